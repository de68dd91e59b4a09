"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

* :class:`Oracle` -- the C restatement in gxoracle.c (``_ref/libgxoracle.so``).
* :class:`Reference` -- the reference correlator's own hot path compiled from
  its sources with the harness in ref_harness.cpp (``_ref/libdifxref.so``).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from difx_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_LIB = os.path.join(REF_DIR, "libgxoracle.so")
REFERENCE_LIB = os.path.join(REF_DIR, "libdifxref.so")
# Where the reference tree lies in the build container (DIFX_REFERENCE); the
# GPU box has no tree and uses the prebuilt _ref/ libraries.
REFERENCE_SRC = os.environ.get("DIFX_REFERENCE", "/root/reference")


def build(reference: bool = True) -> None:
    """Build the oracle (and, where the reference tree exists, the reference harness)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if reference and os.path.isdir(REFERENCE_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "-j8", f"REF={REFERENCE_SRC}"], check=True)
        subprocess.run(["make", "-s", "-C", HERE, "vmux", f"REF={REFERENCE_SRC}"], check=True)
        subprocess.run(["make", "-s", "-C", HERE, "shim", "-j8", f"REF={REFERENCE_SRC}"], check=True)


def reference_available() -> bool:
    return os.path.exists(REFERENCE_LIB)


class gxo_params(C.Structure):
    _fields_ = [("precision", C.c_int), ("nthreads", C.c_int), ("num_buffered_ffts", C.c_int),
                ("xc_avg_ns", C.c_longlong), ("ac_avg_ns", C.c_longlong)]


FP32_REF = 0
FP64 = 1


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_LIB):
            build(reference=False)
        self.lib = C.CDLL(ORACLE_LIB)
        self.lib.gxo_layout.restype = C.c_longlong
        self.lib.gxo_unpack.restype = C.c_int

    def layout(self, jd: capi.JobDesc):
        d = jd.desc
        nfb = max(1, d.nfreqs * d.nbaselines)
        bl = np.zeros(nfb, np.int32)
        bw = np.zeros(nfb, np.int32)
        ac = np.zeros(d.nstations, np.int32)
        acw = np.zeros(d.nstations, np.int32)
        rl = self.lib.gxo_layout(jd.ptr(), bl.ctypes.data_as(C.c_void_p), bw.ctypes.data_as(C.c_void_p),
                                 ac.ctypes.data_as(C.c_void_p), acw.ctypes.data_as(C.c_void_p))
        return int(rl), bl, bw, ac, acw

    def params(self, precision=FP32_REF, nthreads=1, num_buffered_ffts=10,
               xc_avg_ns=2_000_000_000, ac_avg_ns=2_000_000_000):
        return gxo_params(precision, nthreads, num_buffered_ffts, xc_avg_ns, ac_avg_ns)

    def subint(self, jd: capi.JobDesc, sd: capi.SubintDesc, params: gxo_params) -> np.ndarray:
        rl = self.layout(jd)[0]
        out = np.zeros(2 * rl, np.float64)
        self.lib.gxo_subint(jd.ptr(), sd.ptr(), C.byref(params), out.ctypes.data_as(C.c_void_p))
        return out[0::2] + 1j * out[1::2]

    def station_block(self, jd: capi.JobDesc, sd: capi.SubintDesc, station: int, block: int,
                      params: gxo_params):
        st = jd.desc.stations[station]
        n = jd.desc.freqs[st.recfreq[0]].nchan
        out = np.zeros(2 * st.nbands * n, np.float64)
        w = C.c_double(0)
        self.lib.gxo_station_block(jd.ptr(), sd.ptr(), station, block, C.byref(params),
                                   out.ctypes.data_as(C.c_void_p), C.byref(w))
        return (out[0::2] + 1j * out[1::2]).reshape(st.nbands, n), w.value

    def unpack(self, jd: capi.JobDesc, station: int, data: np.ndarray, offset: int, nsamp: int):
        st = jd.desc.stations[station]
        fs = (st.framebytes - 32) * 8 // (st.nbits * st.nbands)
        if st.is_complex:
            fs //= 2
        per = nsamp * (2 if st.is_complex else 1)
        out = np.zeros(st.nbands * per, np.float32)
        good = self.lib.gxo_unpack(C.byref(st), fs, data.ctypes.data_as(C.c_void_p), C.c_longlong(len(data)),
                                   offset, nsamp, out.ctypes.data_as(C.c_void_p))
        return out.reshape(st.nbands, per), good


class Reference:
    """The reference's own Configuration/Mode/Core, driven through ref_harness.cpp."""

    def __init__(self, inputfile: str):
        if not os.path.exists(REFERENCE_LIB):
            raise RuntimeError("reference harness not built (oracle/_ref/libdifxref.so)")
        self.lib = C.CDLL(REFERENCE_LIB)
        self.lib.ref_open.restype = C.c_void_p
        h = self.lib.ref_open(inputfile.encode())
        if not h:
            raise RuntimeError(f"reference could not open {inputfile}")
        self.h = C.c_void_p(h)
        self.result_length = self.lib.ref_result_length(self.h)
        self.blocks_per_send = self.lib.ref_blocks_per_send(self.h)
        self.nthreads = self.lib.ref_num_threads(self.h)

    def close(self) -> None:
        """Free the reference's Core, Modes and Configuration (many GB for large jobs)."""
        if getattr(self, "h", None) is not None:
            self.lib.ref_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def layout(self, nfreqs: int, nbaselines: int, nstations: int):
        bl = np.zeros(max(1, nfreqs * nbaselines), np.int32)
        bw = np.zeros_like(bl)
        ac = np.zeros(nstations, np.int32)
        acw = np.zeros(nstations, np.int32)
        self.lib.ref_layout(self.h, bl.ctypes.data_as(C.c_void_p), bw.ctypes.data_as(C.c_void_p),
                            ac.ctypes.data_as(C.c_void_p), acw.ctypes.data_as(C.c_void_p))
        return self.result_length, bl, bw, ac, acw

    def interpolator(self, station: int, scan: int, sec: int, ns: int) -> np.ndarray:
        out = np.zeros(3, np.float64)
        self.lib.ref_interpolator(self.h, station, scan, sec, ns, out.ctypes.data_as(C.c_void_p))
        return out

    def process(self, si) -> np.ndarray:
        n = len(si.data)
        datap = (C.c_void_p * n)(*[d.ctypes.data for d in si.data])
        lens = (C.c_int * n)(*[len(d) for d in si.data])
        ctrl = (C.c_void_p * n)(*[c.ctypes.data for c in si.control])
        res = np.zeros(2 * self.result_length, np.float32)
        self.lib.ref_process(self.h, si.scan, si.sec, si.ns, datap, lens, ctrl, len(si.control[0]),
                             res.ctypes.data_as(C.c_void_p))
        return res[0::2] + 1j * res[1::2]

    def vis_write(self, results, scan: int, sec: int, ns: int, outdir: str) -> None:
        """The reference's Visibility integrating `results` (complex64 Core result
        arrays) for the integration starting at (scan, sec, ns), written to outdir."""
        arrs = [np.ascontiguousarray(r, dtype=np.complex64) for r in results]
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        os.makedirs(outdir, exist_ok=True)
        st = self.lib.ref_vis_write(self.h, len(arrs), ptrs, scan, sec, ns, outdir.encode())
        if st != 0:
            raise RuntimeError(f"ref_vis_write failed ({st})")

    def set_monitor(self, sta: bool, kurtosis: bool, channels: int) -> None:
        """STA / kurtosis dumps on for the following process() calls."""
        self.lib.ref_set_monitor(self.h, int(sta), int(kurtosis), channels)

    def take_monitor_records(self):
        """The STA and kurtosis records (DifxMessageSTARecord, difxmessage.h:637-652)
        the reference sent since the last call: a list of dicts with the type
        (STA_AUTOCORRELATION 1, STA_KURTOSIS 3), datastream,
        band, nChan, times and the float data."""
        buf = (C.c_char * (1 << 22))()
        n = self.lib.ref_take_messages(self.h, buf, len(buf))
        raw = bytes(buf[:n])
        out, o = [], 0
        hdr = 10 * 4 + 32
        while o + hdr <= n:
            v = np.frombuffer(raw[o:o + 40], "<i4")
            nchan = int(v[9])
            data = np.frombuffer(raw[o + hdr:o + hdr + 4 * nchan], "<f4").copy()
            out.append(dict(type=int(v[0]), scan=int(v[1]), sec=int(v[2]), ns=int(v[3]), nswidth=int(v[4]),
                            ds=int(v[5]), core=int(v[6]), thread=int(v[7]), band=int(v[8]), nchan=nchan,
                            ident=raw[o + 40:o + hdr].split(b"\0")[0].decode(), data=data))
            o += hdr + 4 * nchan
        return out

    def uvw(self, scan: int, offset_s: float, ds1: int, ds2: int) -> np.ndarray:
        out = np.zeros(3, np.float64)
        if self.lib.ref_uvw(self.h, scan, C.c_double(offset_s), ds1, ds2, out.ctypes.data_as(C.c_void_p)) != 0:
            raise RuntimeError("no (u, v, w) model at this time")
        return out

    def mode_block(self, si, station: int, block: int, nbands: int, nchan: int):
        sp = np.zeros(2 * nbands * nchan, np.float32)
        w = C.c_float(0)
        self.lib.ref_mode_block(self.h, station, si.data[station].ctypes.data_as(C.c_void_p),
                                len(si.data[station]), si.control[station].ctypes.data_as(C.c_void_p),
                                len(si.control[station]), si.scan, si.sec, si.ns, block,
                                sp.ctypes.data_as(C.c_void_p), C.byref(w))
        return (sp[0::2] + 1j * sp[1::2]).reshape(nbands, nchan), w.value

    def mode_blocks(self, si, station: int, nblocks: int, nbands: int, nchan: int):
        """Mode::process of one datastream over blocks 0..nblocks-1: (spectra
        [nblocks][nbands][nchan], data weights [nblocks], autocorrelations
        [2][nbands][nchan], weights [2][nbands])."""
        return _mode_blocks(self.lib.ref_mode_blocks, self.h, nblocks, nbands, nchan,
                            (si.data[station].ctypes.data_as(C.c_void_p), len(si.data[station]),
                             si.control[station].ctypes.data_as(C.c_void_p), len(si.control[station]),
                             si.scan, si.sec, si.ns), station)

    def set_interpolator(self, station: int, interp=None) -> None:
        """Replaces the delay interpolator Mode::setOffsets computes for
        `station` in later mode_blocks calls (None: the model's again)."""
        arr = None if interp is None else np.ascontiguousarray(interp, np.float64)
        st = self.lib.ref_set_interpolator(self.h, station, None if arr is None else arr.ctypes.data_as(C.c_void_p))
        if st != 0:
            raise RuntimeError(f"ref_set_interpolator failed ({st})")

    def unpack(self, station: int, data: np.ndarray, offset: int, nbands: int, per: int):
        out = np.zeros(nbands * per * 2, np.float32)
        w = C.c_float(0)
        us = C.c_int(0)
        n = self.lib.ref_unpack(self.h, station, data.ctypes.data_as(C.c_void_p), len(data), offset,
                                out.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(us))
        return out, w.value, us.value, n


class RefDataStream:
    """The reference's VDIF DataStream of one datastream of a Reference
    (ds_harness.cpp): raw frames of one scan file, dataRead per segment,
    calculateControlParams per subint."""

    GEOM = ("bufferbytes", "readbytes", "numsegments", "overflowbytes", "sendbytes", "blockspersend",
            "controllength", "bytespersamplenum", "bytespersampledenom", "bytesbetweenintegerns", "nsinc",
            "framegranularity", "slotbytes", "framespersecond")

    def __init__(self, ref: "Reference", ds: int, raw: bytes):
        self.ref = ref
        self.lib = ref.lib
        self.lib.ref_ds_open.restype = C.c_void_p
        self.lib.ref_ds_buffer.restype = C.c_void_p
        self._raw = (C.c_ubyte * len(raw)).from_buffer_copy(raw)
        p = self.lib.ref_ds_open(ref.h, ds, self._raw, C.c_longlong(len(raw)))
        if not p:
            raise RuntimeError("reference DataStream could not take these bytes")
        self.p = C.c_void_p(p)
        g = (C.c_longlong * 14)()
        d = (C.c_double * 1)()
        self.lib.ref_ds_geometry(self.p, g, d)
        self.geometry = dict(zip(self.GEOM, list(g)))
        self.geometry["sampletimens"] = d[0]

    def read(self, segment: int):
        """dataRead(segment): ((raw offset, window bytes, dest bytes, start
        frame), (scan, scanseconds, scanns, validbytes, readto)), or None once
        the data has ended."""
        win = (C.c_longlong * 4)()
        seg = (C.c_int * 5)()
        if self.lib.ref_ds_read(self.p, segment, win, seg) != 0:
            return None
        return tuple(win), tuple(seg)

    def set_segment(self, segment: int, seg) -> None:
        a = (C.c_int * 5)(*seg[:5])
        self.lib.ref_ds_set_segment(self.p, segment, a)

    def control(self, scan: int, sec: int, ns: int):
        """calculateControlParams + the wrap copy: (control words, send start,
        segment, bytes sent)."""
        n = self.geometry["controllength"]
        cw = np.zeros(n, np.int32)
        info = (C.c_int * 3)()
        self.lib.ref_ds_control(self.p, scan, sec, ns, cw.ctypes.data_as(C.c_void_p), info)
        return cw, info[0], info[1], info[2]

    def data(self, start: int, nbytes: int) -> np.ndarray:
        """A copy of the data buffer's bytes [start, start + nbytes)."""
        base = self.lib.ref_ds_buffer(self.p)
        return np.ctypeslib.as_array((C.c_ubyte * nbytes).from_address(base + start)).copy()

    def close(self) -> None:
        if getattr(self, "p", None) is not None:
            self.lib.ref_ds_close(self.p)
            self.p = None

    def __del__(self):
        self.close()


def _mode_blocks(fn, h, nblocks, nbands, nchan, mid_args, station):
    sp = np.zeros(2 * nblocks * nbands * nchan, np.float32)
    dw = np.zeros(nblocks, np.float32)
    au = np.zeros(2 * 2 * nbands * nchan, np.float32)
    wt = np.zeros(2 * nbands, np.float32)
    tail = (nblocks, sp.ctypes.data_as(C.c_void_p), dw.ctypes.data_as(C.c_void_p), au.ctypes.data_as(C.c_void_p),
            wt.ctypes.data_as(C.c_void_p))
    st = fn(h, station, *mid_args, *tail)
    if st != 0:
        raise RuntimeError(f"mode_blocks failed ({st})")
    c = lambda a: a[0::2] + 1j * a[1::2]
    return (c(sp).reshape(nblocks, nbands, nchan), dw, c(au).reshape(2, nbands, nchan), wt.reshape(2, nbands))


SHIM_LIB = os.path.join(REF_DIR, "libgxshim.so")


def shim_available() -> bool:
    return os.path.exists(SHIM_LIB)


class Binding:
    """The DiFX-side binding (difx_b200/mpifxcorr: GpuCore, GpuMode) over the
    reference's Configuration, driven through shim_harness.cpp."""

    def __init__(self, inputfile: str, device: int = 0, xstep: int = 0):
        if not shim_available():
            raise RuntimeError("binding harness not built (oracle/_ref/libgxshim.so)")
        self.lib = C.CDLL(SHIM_LIB)
        self.lib.shim_open.restype = C.c_void_p
        self.lib.shim_last_error.restype = C.c_char_p
        h = self.lib.shim_open(inputfile.encode(), device, xstep)
        if not h:
            raise RuntimeError(f"binding could not open {inputfile}")
        self.h = C.c_void_p(h)

    def process(self, si, result_length: int) -> np.ndarray:
        n = len(si.data)
        datap = (C.c_void_p * n)(*[d.ctypes.data for d in si.data])
        lens = (C.c_int * n)(*[len(d) for d in si.data])
        ctrl = (C.c_void_p * n)(*[c.ctypes.data for c in si.control])
        res = np.zeros(2 * result_length, np.float32)
        st = self.lib.shim_process(self.h, si.scan, si.sec, si.ns, datap, lens, ctrl, len(si.control[0]),
                                   res.ctypes.data_as(C.c_void_p))
        if st != 0:
            raise RuntimeError(f"GpuCore slot failed ({st}): {self.lib.shim_last_error(self.h).decode()}")
        return res[0::2] + 1j * res[1::2]

    def mode_blocks(self, station: int, nblocks: int, nbands: int, nchan: int):
        """GpuMode over blocks 0..nblocks-1 of the slot process() last correlated
        (same outputs as Reference.mode_blocks)."""
        return _mode_blocks(self.lib.shim_mode_blocks, self.h, nblocks, nbands, nchan, (), station)

    def close(self) -> None:
        if getattr(self, "h", None) is not None:
            self.lib.shim_close(self.h)
            self.h = None

    def __del__(self):
        self.close()


VMUX_LIB = os.path.join(HERE, "_ref", "libvdifmuxref.so")


def vmux_available() -> bool:
    return os.path.exists(VMUX_LIB)


def ref_vdifmux(src: bytes, dest_bytes: int, frame_bytes: int, fps: int, bits: int, thread_ids, nsort: int,
                ngap: int, flags: int, start_frame: int = -1, dest_init: int = 0, channels_per_thread: int = 1):
    """The reference's vdifmux on host buffers: (output bytes, array of 23
    values in the order of vdifmux_harness.c: statistics, return value, output
    frame bytes, nanoseconds of the call)."""
    lib = C.CDLL(VMUX_LIB)
    dest = (C.c_ubyte * dest_bytes)(*([dest_init] * dest_bytes)) if dest_init else (C.c_ubyte * dest_bytes)()
    srcb = (C.c_ubyte * len(src)).from_buffer_copy(src)
    ids = (C.c_int * len(thread_ids))(*thread_ids)
    out = (C.c_longlong * 23)()
    rv = lib.ref_vdifmux_channels(dest, dest_bytes, srcb, len(src), frame_bytes, fps, bits, len(thread_ids), ids,
                                  nsort, ngap, flags, C.c_longlong(start_frame), channels_per_thread, out)
    if rv < 0:
        raise RuntimeError(f"reference vdifmux failed: {rv}")
    return bytes(dest), list(out)
