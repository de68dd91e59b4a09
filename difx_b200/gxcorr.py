"""Python binding of the gxcorr C ABI (include/gxcorr.h) via ctypes.

``Correlator`` mirrors the reference's Core-slot contract: one call per
subint with the raw datastream buffers and control words, returning the Core
result array (complex64, the layout of ``procslots[].results``,
mpifxcorr/src/configuration.cpp:2348-2630).

The CUDA library ``difx_b200/libgxcorr.so`` must be built (``python -m
difx_b200.build``); there is no CPU fallback -- loading fails loudly if it is
missing.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from . import capi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libgxcorr.so")
_lib = None


class GxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{capi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    """The loaded libgxcorr.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is missing: build it with `python -m difx_b200.build`")
        L = C.CDLL(LIBPATH)
        L.gx_last_error.restype = C.c_char_p
        L.gx_status_string.restype = C.c_char_p
        L.gx_server_last_error.restype = C.c_char_p
        L.gx_batch_last_error.restype = C.c_char_p
        L.gx_vdifmux_last_error.restype = C.c_char_p
        L.gx_ring_last_error.restype = C.c_char_p
        for name in EXPORTED_SYMBOLS:
            if name not in ("gx_last_error", "gx_status_string", "gx_server_last_error", "gx_batch_last_error",
                            "gx_vdifmux_last_error", "gx_ring_last_error"):
                getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


EXPORTED_SYMBOLS = ("gx_open", "gx_open_input", "gx_close", "gx_last_error", "gx_status_string",
                    "gx_get_layout", "gx_get_offsets", "gx_interpolator", "gx_scan_start_sec", "gx_subint",
                    "gx_subint_device", "gx_synchronize", "gx_spectra", "gx_stage_times", "gx_launch_count",
                    "gx_subint_device_noalloc", "gx_set_tc_scales", "gx_vis_open", "gx_vis_add", "gx_vis_write",
                    "gx_vis_close", "gx_uvw", "gx_server_open", "gx_server_set_executor", "gx_server_attach",
                    "gx_server_submit", "gx_server_set_deadline", "gx_server_wait", "gx_server_stats", "gx_server_close", "gx_device_bytes",
                    "gx_server_last_error", "gx_batch_open", "gx_batch_run", "gx_batch_synchronize",
                    "gx_batch_info", "gx_batch_last_error", "gx_batch_close", "gx_vis_buffer",
                    "gx_vis_set_subints", "gx_vis_clear", "gx_subint_async", "gx_subint_wait", "gx_vdifmux_open",
                    "gx_vdifmux_info", "gx_vdifmux_run", "gx_vdifmux_reset_stats", "gx_vdifmux_last_error",
                    "gx_vdifmux_close", "gx_get_pcal_layout", "gx_vis_pcal_headers", "gx_ring_open",
                    "gx_ring_geometry_get", "gx_ring_buffer", "gx_ring_read", "gx_ring_set_segment",
                    "gx_ring_get_segment", "gx_ring_control_host", "gx_ring_subint_device", "gx_ring_last_control",
                    "gx_ring_reset", "gx_ring_last_error", "gx_ring_close", "gx_set_kurtosis", "gx_kurtosis",
                    "gx_sta", "gx_set_tiles", "gx_get_tiles", "gx_batch_tune_tiles")


def subint_device_noalloc(jd: capi.JobDesc, sd: capi.SubintDesc, dev_results_ptr: int, stream_ptr: int = 0) -> None:
    """One subint without any device allocation (gx_subint_device_noalloc).

    For callers that cannot allocate device memory: sd holds device data
    pointers (host control words and interpolators); results go to the
    caller's device buffer.  Work runs on `stream_ptr` (0 = legacy default
    stream) and is not synchronised.  Calls share one library-wide scratch
    array, so calls must not overlap on the GPU."""
    err = C.create_string_buffer(512)
    st = lib().gx_subint_device_noalloc(jd.ptr(), sd.ptr(), C.c_void_p(dev_results_ptr),
                                        C.c_void_p(stream_ptr) if stream_ptr else None, err, len(err))
    if st != 0:
        raise GxError(st, err.value.decode(errors="replace"))


class Correlator:
    """One correlation configuration on one GPU."""

    def __init__(self, handle: C.c_void_p, keepalive=None):
        self.h = handle
        self._keep = keepalive
        info = capi.gx_layout_info()
        self._check(lib().gx_get_layout(self.h, C.byref(info)))
        self.info = info
        self.result_length = int(info.result_length)

    # ------------------------------------------------------------- opening
    @classmethod
    def from_desc(cls, jd: capi.JobDesc, device: int = 0) -> "Correlator":
        h = C.c_void_p()
        st = lib().gx_open(jd.ptr(), device, C.byref(h))
        if st != 0:
            raise GxError(st, "gx_open failed (see stderr)")
        return cls(h, jd)

    @classmethod
    def from_input(cls, inputfile: str, device: int = 0, xstep: int = capi.GX_XSTEP_FP32) -> "Correlator":
        h = C.c_void_p()
        st = lib().gx_open_input(inputfile.encode(), device, xstep, C.byref(h))
        if st != 0:
            raise GxError(st, f"gx_open_input({inputfile}) failed (see stderr)")
        return cls(h)

    def close(self):
        if self.h:
            lib().gx_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            msg = lib().gx_last_error(self.h).decode() if self.h else ""
            raise GxError(st, msg)

    # ------------------------------------------------------------- queries
    def offsets(self):
        i = self.info
        nfb = max(1, i.nfreqs * i.nbaselines)
        bl = np.zeros(nfb, np.int32)
        bw = np.zeros(nfb, np.int32)
        ac = np.zeros(i.nstations, np.int32)
        acw = np.zeros(i.nstations, np.int32)
        self._check(lib().gx_get_offsets(self.h, bl.ctypes.data_as(C.c_void_p), bw.ctypes.data_as(C.c_void_p),
                                         ac.ctypes.data_as(C.c_void_p), acw.ctypes.data_as(C.c_void_p)))
        return self.result_length, bl, bw, ac, acw

    def pcal_layout(self):
        """(offsets, ntones), each [nstations][GX_MAX_BANDS]: result index of the first
        phase-cal tone of each recorded band (-1: none) and its number of tones."""
        n = self.info.nstations * capi.GX_MAX_BANDS
        off = np.zeros(n, np.int32)
        nt = np.zeros(n, np.int32)
        self._check(lib().gx_get_pcal_layout(self.h, off.ctypes.data_as(C.c_void_p), nt.ctypes.data_as(C.c_void_p)))
        return off.reshape(-1, capi.GX_MAX_BANDS), nt.reshape(-1, capi.GX_MAX_BANDS)

    def interpolator(self, station: int, scan: int, sec: int, ns: int) -> np.ndarray:
        out = np.zeros(3, np.float64)
        self._check(lib().gx_interpolator(self.h, station, scan, sec, ns, out.ctypes.data_as(C.c_void_p)))
        return out

    def uvw(self, scan: int, offset_s: float, ds1: int, ds2: int) -> np.ndarray:
        """(u, v, w) in metres of baseline ds1 - ds2, offset_s after the scan start (gx_uvw)."""
        out = np.zeros(3, np.float64)
        self._check(lib().gx_uvw(self.h, scan, C.c_double(offset_s), ds1, ds2, out.ctypes.data_as(C.c_void_p)))
        return out

    def scan_start_sec(self, scan: int) -> float:
        v = C.c_double(0)
        self._check(lib().gx_scan_start_sec(self.h, scan, C.byref(v)))
        return v.value

    def stage_times(self) -> np.ndarray:
        ms = (C.c_float * 3)()
        self._check(lib().gx_stage_times(self.h, ms))
        return np.array(list(ms))

    def device_bytes(self) -> int:
        """Device memory the handle holds (gx_device_bytes)."""
        n = C.c_longlong(0)
        self._check(lib().gx_device_bytes(self.h, C.byref(n)))
        return n.value

    def launch_count(self) -> int:
        n = C.c_int(0)
        self._check(lib().gx_launch_count(self.h, C.byref(n)))
        return n.value

    # ------------------------------------------------------------- work
    def subint(self, sd: capi.SubintDesc, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Host buffers in, Core result array (complex64) out."""
        if out is None:
            out = np.zeros(self.result_length, np.complex64)
        self._check(lib().gx_subint(self.h, sd.ptr(), out.ctypes.data_as(C.c_void_p)))
        return out

    def subint_device(self, sd: capi.SubintDesc, dev_results_ptr: int, stream_ptr: int = 0):
        """Device buffers in (sd holds device pointers), device results out; asynchronous."""
        self._check(lib().gx_subint_device(self.h, sd.ptr(), C.c_void_p(dev_results_ptr),
                                           C.c_void_p(stream_ptr) if stream_ptr else None))

    def synchronize(self):
        self._check(lib().gx_synchronize(self.h))

    def subint_async(self, sd: capi.SubintDesc, out: np.ndarray) -> None:
        """Pipelined gx_subint: returns once the subint is enqueued (at most two in
        flight); `sd`'s buffers and `out` (complex64, pinned for overlap) must stay
        alive until the matching wait()."""
        self._check(lib().gx_subint_async(self.h, sd.ptr(), out.ctypes.data_as(C.c_void_p)))
        if not hasattr(self, "_inflight"):
            self._inflight = []
        self._inflight.append((sd, out))

    def wait(self) -> np.ndarray:
        """Waits for the oldest gx_subint_async call; returns its result array."""
        st = lib().gx_subint_wait(self.h)
        sd, out = self._inflight.pop(0) if getattr(self, "_inflight", None) else (None, None)
        self._check(st)
        return out

    def set_tiles(self, xmac_variant: int, fstep_items: int) -> None:
        """Launch shapes (results do not depend on them)."""
        self._check(lib().gx_set_tiles(self.h, xmac_variant, fstep_items))

    def tiles(self):
        x, f = C.c_int(0), C.c_int(0)
        self._check(lib().gx_get_tiles(self.h, C.byref(x), C.byref(f)))
        return x.value, f.value

    def set_kurtosis(self, dump_channels: int) -> None:
        """Spectral kurtosis accumulation on (dump channels) or off (0)."""
        self._check(lib().gx_set_kurtosis(self.h, dump_channels))
        self._kdump = dump_channels

    def kurtosis(self):
        """(sk [nstations, GX_MAX_BANDS, dump], nchan [nstations, GX_MAX_BANDS], valid [nstations])
        of the last subint."""
        n = self.info.nstations
        d = self._kdump
        sk = np.zeros((n, capi.GX_MAX_BANDS, d), np.float32)
        nch = np.zeros((n, capi.GX_MAX_BANDS), np.int32)
        valid = np.zeros(n, np.int32)
        self._check(lib().gx_kurtosis(self.h, sk.ctypes.data_as(C.c_void_p), nch.ctypes.data_as(C.c_void_p),
                                      valid.ctypes.data_as(C.c_void_p)))
        return sk, nch, valid

    def sta(self, results: np.ndarray, dump_channels: int):
        """STA dump of a Core result array (complex64, host): (sta, nchan, sent)."""
        n = self.info.nstations
        res = np.ascontiguousarray(results, dtype=np.complex64)
        out = np.zeros((n, capi.GX_MAX_BANDS, dump_channels), np.float32)
        nch = np.zeros((n, capi.GX_MAX_BANDS), np.int32)
        sent = np.zeros((n, capi.GX_MAX_BANDS), np.int32)
        self._check(lib().gx_sta(self.h, res.ctypes.data_as(C.c_void_p), dump_channels, out.ctypes.data_as(C.c_void_p),
                                 nch.ctypes.data_as(C.c_void_p), sent.ctypes.data_as(C.c_void_p)))
        return out, nch, sent

    def set_tc_scales(self, station: int, band: int, scales) -> None:
        """Per-channel operand scales of the tensor-core X-step for one station band
        (rounded to powers of two by the library)."""
        a = np.ascontiguousarray(scales, dtype=np.float32)
        self._check(lib().gx_set_tc_scales(self.h, station, band, a.ctypes.data_as(C.c_void_p)))

    def spectra(self, station: int, block: int, nbands: int):
        out = np.zeros(nbands * self.info.nchan, np.complex64)
        w = C.c_float(0)
        self._check(lib().gx_spectra(self.h, station, block, out.ctypes.data_as(C.c_void_p), C.byref(w)))
        return out.reshape(nbands, self.info.nchan), w.value


class Visibility:
    """Device integration buffer and DIFX/SWIN writer of one Correlator
    (gx_vis_*, mpifxcorr's Visibility).  The Correlator must come from
    ``Correlator.from_input``."""

    def __init__(self, corr: Correlator, outdir: str):
        self.corr = corr
        self.v = C.c_void_p()
        corr._check(lib().gx_vis_open(corr.h, outdir.encode(), C.byref(self.v)))

    def add(self, dev_results_ptr: int, stream_ptr: int = 0) -> None:
        """Adds one subint's Core result array (device pointer) to the integration."""
        self.corr._check(lib().gx_vis_add(self.v, C.c_void_p(dev_results_ptr),
                                          C.c_void_p(stream_ptr) if stream_ptr else None))

    def write(self, scan: int, sec: int, ns: int) -> int:
        """Normalises and appends the integration that started at (scan, sec, ns); returns the records written."""
        n = C.c_int(0)
        self.corr._check(lib().gx_vis_write(self.v, scan, sec, ns, C.byref(n)))
        return n.value

    def buffer(self):
        """(device pointer, float count, subints added) of the integration buffer (gx_vis_buffer)."""
        p, n, k = C.c_void_p(), C.c_longlong(0), C.c_int(0)
        self.corr._check(lib().gx_vis_buffer(self.v, C.byref(p), C.byref(n), C.byref(k)))
        return p.value, n.value, k.value

    def set_subints(self, nsub: int) -> None:
        self.corr._check(lib().gx_vis_set_subints(self.v, int(nsub)))

    def clear(self) -> None:
        self.corr._check(lib().gx_vis_clear(self.v))

    def pcal_headers(self) -> None:
        """The comment lines at the top of the PCAL files (once per job)."""
        self.corr._check(lib().gx_vis_pcal_headers(self.v))

    def close(self) -> None:
        if self.v:
            lib().gx_vis_close(self.v)
            self.v = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LatencyStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("failed", C.c_longlong), ("p50_ms", C.c_double),
                ("p95_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double)]


EXECUTOR = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p)


class Server:
    """Request loop over resident jobs on one GPU (gx_server_*): continuous
    batching of subint requests under an HBM budget, with latency statistics."""

    def __init__(self, slots: int, hbm_budget_bytes: int, device_inputs: bool = False):
        self.s = C.c_void_p()
        self._check(lib().gx_server_open(int(slots), C.c_longlong(int(hbm_budget_bytes)), 1 if device_inputs else 0,
                                         C.byref(self.s)))
        self._keep = []   # descriptors and buffers of requests in flight

    def _check(self, st: int):
        if st != 0:
            msg = lib().gx_server_last_error(self.s).decode() if getattr(self, "s", None) else ""
            raise GxError(st, msg or "gx_server call failed")

    def set_executor(self, fn) -> None:
        """fn(job, sub_ptr, results_ptr) -> status; replaces the default executor."""
        cb = EXECUTOR(lambda ctx, h, job, sub, res: int(fn(job, sub, res)))
        self._cb = cb
        self._check(lib().gx_server_set_executor(self.s, cb, None))

    def attach(self, corr: Optional[Correlator] = None, resident_bytes: int = -1) -> int:
        job = C.c_int(-1)
        self._check(lib().gx_server_attach(self.s, corr.h if corr else None, C.c_longlong(int(resident_bytes)),
                                           C.byref(job)))
        return job.value

    def set_deadline(self, job: int, deadline_ms: float) -> None:
        """Relative deadline of the job's requests (default: its subint duration; <= 0: none)."""
        self._check(lib().gx_server_set_deadline(self.s, job, C.c_double(deadline_ms)))

    def submit(self, job: int, sd: capi.SubintDesc, results_ptr: int = 0, request_bytes: int = -1,
               keep=None) -> int:
        t = C.c_longlong(0)
        self._check(lib().gx_server_submit(self.s, job, sd.ptr(), C.c_void_p(results_ptr) if results_ptr else None,
                                           C.c_longlong(int(request_bytes)), C.byref(t)))
        self._keep.append((t.value, sd, keep))
        return t.value

    def wait(self, ticket: int) -> float:
        ms = C.c_double(0)
        st = lib().gx_server_wait(self.s, C.c_longlong(ticket), C.byref(ms))
        self._keep = [k for k in self._keep if k[0] != ticket]
        self._check(st)
        return ms.value

    def stats(self, reset: bool = False) -> LatencyStats:
        out = LatencyStats()
        self._check(lib().gx_server_stats(self.s, 1 if reset else 0, C.byref(out)))
        return out

    def close(self) -> None:
        if self.s:
            lib().gx_server_close(self.s)
            self.s = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


BATCH_MODES = {"serial": 0, "streams": 1, "graph": 2}


class Batch:
    """One subint of each of several resident jobs per step (gx_batch_*):
    per-job launches on one stream ("serial"), jobs spread over branch
    streams ("streams") or that schedule replayed as one CUDA graph
    ("graph"); nstreams 0 tunes the branch count on the first steps."""

    def __init__(self, corrs: Sequence[Correlator], dev_results_ptrs: Sequence[int], mode: str = "graph",
                 nstreams: int = 0):
        n = len(corrs)
        hs = (C.c_void_p * n)(*[c.h for c in corrs])
        rs = (C.c_void_p * n)(*[int(p) for p in dev_results_ptrs])
        self.b = C.c_void_p()
        self.n = n
        self._corrs = list(corrs)
        st = lib().gx_batch_open(hs, rs, n, BATCH_MODES[mode], int(nstreams), C.byref(self.b))
        if st != 0:
            raise GxError(st, "gx_batch_open failed")
        self._subs = None

    def _check(self, st: int):
        if st != 0:
            raise GxError(st, lib().gx_batch_last_error(self.b).decode() if self.b else "")

    def run(self, subs: Sequence[capi.SubintDesc]) -> None:
        """Starts one step: subs[j] is job j's subint (device data pointers)."""
        arr = (C.c_void_p * self.n)(*[C.addressof(sd.desc) for sd in subs])
        self._subs = (list(subs), arr)   # alive until the step has been staged and run
        self._check(lib().gx_batch_run(self.b, arr))

    def synchronize(self) -> float:
        """Waits for the step; returns its device time in ms."""
        ms = C.c_float(0)
        self._check(lib().gx_batch_synchronize(self.b, C.byref(ms)))
        return ms.value

    def tune_tiles(self, subs: Sequence[capi.SubintDesc], reps: int = 2) -> int:
        """Per shape class, the fastest launch shapes (gx_batch_tune_tiles); returns the class count."""
        arr = (C.c_void_p * self.n)(*[C.addressof(sd.desc) for sd in subs])
        n = C.c_int(0)
        self._check(lib().gx_batch_tune_tiles(self.b, arr, int(reps), C.byref(n)))
        return n.value

    def info(self):
        """(branch streams in use (0 while tuning), tuning, kernel launches of the last step)."""
        k, t, l = C.c_int(0), C.c_int(0), C.c_int(0)
        self._check(lib().gx_batch_info(self.b, C.byref(k), C.byref(t), C.byref(l)))
        return k.value, bool(t.value), l.value

    def close(self) -> None:
        if self.b:
            lib().gx_batch_close(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VdifMuxStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in (
        "valid_frames", "invalid_frames", "discarded_frames", "wrong_thread_frames", "skipped_bytes", "fill_bytes",
        "duplicate_frames", "bytes_processed", "good_output_frames", "partial_output_frames", "filler_output_frames",
        "calls", "src_bytes", "src_used", "dest_bytes", "dest_used", "output_frames", "start_frame",
        "returned_bytes")] + [("epoch", C.c_int)]


class VdifMux:
    """Multi-thread VDIF -> multi-channel single-thread VDIF on the device (gx_vdifmux_*)."""

    def __init__(self, frame_bytes: int, frames_per_second: int, bits: int, thread_ids: Sequence[int],
                 nsort: int = 32, ngap: int = 1000, flags: int = 0, channels_per_thread: int = 1, device: int = 0):
        ids = (C.c_int * len(thread_ids))(*thread_ids)
        self.m = C.c_void_p()
        st = lib().gx_vdifmux_open(frame_bytes, frames_per_second, bits, len(thread_ids), ids, channels_per_thread,
                                   nsort, ngap, flags, device, C.byref(self.m))
        if st != 0:
            raise GxError(st, "gx_vdifmux_open failed")
        ofb, nch, gran = C.c_int(0), C.c_int(0), C.c_int(0)
        lib().gx_vdifmux_info(self.m, C.byref(ofb), C.byref(nch), C.byref(gran))
        self.output_frame_bytes, self.output_channels, self.frame_granularity = ofb.value, nch.value, gran.value

    def run(self, src_ptr: int, src_bytes: int, dest_ptr: int, dest_bytes: int, start_frame: int = -1,
            stream_ptr: int = 0) -> VdifMuxStats:
        stats = VdifMuxStats()
        st = lib().gx_vdifmux_run(self.m, C.c_void_p(src_ptr), C.c_longlong(src_bytes), C.c_void_p(dest_ptr),
                                  C.c_longlong(dest_bytes), C.c_longlong(start_frame), C.byref(stats),
                                  C.c_void_p(stream_ptr) if stream_ptr else None)
        if st != 0:
            raise GxError(st, lib().gx_vdifmux_last_error(self.m).decode())
        return stats

    def reset_stats(self) -> None:
        lib().gx_vdifmux_reset_stats(self.m)

    def close(self) -> None:
        if self.m:
            lib().gx_vdifmux_close(self.m)
            self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RingGeometry(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "bufferbytes", "readbytes", "numsegments", "overflowbytes", "sendbytes", "blockspersend", "controllength",
        "blockbytes", "bytespersamplenum", "bytespersampledenom", "bytesbetweenintegerns", "nsinc", "framebytes",
        "payloadbytes", "framespersecond", "framegranularity", "intclockseconds")] + [
        ("sampletimens", C.c_double), ("dataspanns", C.c_longlong)]


class RingSegment(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("scan", "scanseconds", "scanns", "validbytes", "readto", "configindex")]

    def astuple(self):
        return (self.scan, self.scanseconds, self.scanns, self.validbytes, self.readto, self.configindex)


class Ring:
    """Per-station data rings of a Correlator with control words computed on
    the device (gx_ring_*): the DataStream's segmented buffer, filled by the
    device multiplexer, walked by a kernel for every subint."""

    def __init__(self, corr: Correlator, databufferfactor: int = 0, numdatasegments: int = 0):
        self.corr = corr
        self.r = C.c_void_p()
        st = lib().gx_ring_open(corr.h, databufferfactor, numdatasegments, C.byref(self.r))
        if st != 0:
            raise GxError(st, lib().gx_last_error(corr.h).decode())
        self.nst = corr.info.nstations if hasattr(corr, "info") else None

    def _check(self, st: int):
        if st != 0:
            raise GxError(st, lib().gx_ring_last_error(self.r).decode())

    def geometry(self, station: int) -> RingGeometry:
        g = RingGeometry()
        self._check(lib().gx_ring_geometry_get(self.r, station, C.byref(g)))
        return g

    def buffer_ptr(self, station: int) -> int:
        p = C.c_void_p()
        self._check(lib().gx_ring_buffer(self.r, station, C.byref(p)))
        return p.value

    def read(self, station: int, segment: int, scan: int, raw_ptr: int, raw_bytes: int, stream_ptr: int = 0) -> int:
        used = C.c_longlong(0)
        self._check(lib().gx_ring_read(self.r, station, segment, scan, C.c_void_p(raw_ptr), C.c_longlong(raw_bytes),
                                       C.byref(used), C.c_void_p(stream_ptr) if stream_ptr else None))
        return used.value

    def set_segment(self, station: int, segment: int, seg) -> None:
        s = RingSegment(*seg) if not isinstance(seg, RingSegment) else seg
        self._check(lib().gx_ring_set_segment(self.r, station, segment, C.byref(s)))

    def segment(self, station: int, segment: int) -> RingSegment:
        s = RingSegment()
        self._check(lib().gx_ring_get_segment(self.r, station, segment, C.byref(s)))
        return s

    def control_host(self, station: int, scan: int, sec: int, ns: int):
        n = self.geometry(station).controllength
        cw = np.zeros(n, np.int32)
        sp = C.c_int(0)
        st = lib().gx_ring_control_host(self.r, station, scan, sec, ns, cw.ctypes.data_as(C.c_void_p), C.byref(sp))
        if st not in (0, 8):
            self._check(st)
        return cw, sp.value, st == 8

    def subint_device(self, scan: int, sec: int, ns: int, scan_start_sec: float, dev_results_ptr: int,
                      stream_ptr: int = 0) -> None:
        st = lib().gx_ring_subint_device(self.corr.h, self.r, scan, sec, ns, C.c_double(scan_start_sec),
                                         C.c_void_p(dev_results_ptr), C.c_void_p(stream_ptr) if stream_ptr else None)
        if st != 0:
            raise GxError(st, lib().gx_last_error(self.corr.h).decode())

    def last_control(self, nstations: int):
        n = self.geometry(0).controllength
        cw = np.zeros((nstations, n), np.int32)
        sp = np.zeros(nstations, np.int32)
        st = lib().gx_ring_last_control(self.r, cw.ctypes.data_as(C.c_void_p), sp.ctypes.data_as(C.c_void_p))
        if st not in (0, 8):
            self._check(st)
        return cw, sp, st == 8

    def reset(self) -> None:
        self._check(lib().gx_ring_reset(self.r))

    def close(self) -> None:
        if self.r:
            lib().gx_ring_close(self.r)
            self.r = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
