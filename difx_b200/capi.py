"""ctypes mirror of include/gxcorr.h and descriptor builders.

The structs here are byte-for-byte the C ABI's; :func:`job_desc_from_spec`
fills a ``gx_job_desc`` the way ``Configuration::getMode`` and the baseline
table parser derive a Mode's parameters from the ``.input`` tables
(mpifxcorr/src/configuration.cpp:932-998, 1033-1180, 1397-1850).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import List, Optional, Sequence

import numpy as np

from .jobfiles import JobSpec, baseline_plan

GX_MAX_LOCAL_FREQS = 64
GX_MAX_BANDS = 128
GX_MAX_POLPRODUCTS = 4
GX_MAX_MUX_THREADS = 64

GX_XSTEP_FP32 = 0
GX_XSTEP_TC_FP16 = 1
GX_XSTEP_TC_FP16_HILO = 2
GX_XSTEP_AUTO = 3

STATUS_NAMES = {0: "GX_OK", 1: "GX_ERR_ARG", 2: "GX_ERR_UNSUPPORTED", 3: "GX_ERR_CUDA", 4: "GX_ERR_NOMEM",
                5: "GX_ERR_IO", 6: "GX_ERR_MODEL", 7: "GX_ERR_TIMEOUT", 8: "GX_ERR_STATE"}


class gx_freq_desc(C.Structure):
    _fields_ = [("freq_mhz", C.c_double), ("bw_mhz", C.c_double),
                ("lower_sideband", C.c_int), ("nchan", C.c_int), ("chans_to_average", C.c_int)]


class gx_station_desc(C.Structure):
    _fields_ = [("nbits", C.c_int), ("is_complex", C.c_int), ("framebytes", C.c_int),
                ("nrecfreqs", C.c_int),
                ("recfreq", C.c_int * GX_MAX_LOCAL_FREQS),
                ("clock_offset_us", C.c_double * GX_MAX_LOCAL_FREQS),
                ("clock_offset_delta_us", C.c_double * GX_MAX_LOCAL_FREQS),
                ("lo_offset_hz", C.c_double * GX_MAX_LOCAL_FREQS),
                ("nbands", C.c_int),
                ("band_localfreq", C.c_int * GX_MAX_BANDS),
                ("band_pol", C.c_char * GX_MAX_BANDS),
                ("clock_int_seconds", C.c_int),
                ("phase_cal_interval_hz", C.c_longlong), ("phase_cal_base_hz", C.c_longlong),
                ("interlaced", C.c_int),
                ("nzoomfreqs", C.c_int),
                ("zoomfreq", C.c_int * GX_MAX_LOCAL_FREQS),
                ("nzoombands", C.c_int),
                ("zoomband_localfreq", C.c_int * GX_MAX_BANDS),
                ("zoomband_pol", C.c_char * GX_MAX_BANDS),
                ("nmuxthreads", C.c_int),
                ("muxthread", C.c_int * GX_MAX_MUX_THREADS)]


class gx_baseline_desc(C.Structure):
    _fields_ = [("ds1", C.c_int), ("ds2", C.c_int), ("nfreqs", C.c_int),
                ("freq", C.c_int * GX_MAX_LOCAL_FREQS),
                ("npolprod", C.c_int * GX_MAX_LOCAL_FREQS),
                ("band1", (C.c_int * GX_MAX_POLPRODUCTS) * GX_MAX_LOCAL_FREQS),
                ("band2", (C.c_int * GX_MAX_POLPRODUCTS) * GX_MAX_LOCAL_FREQS)]


class gx_job_desc(C.Structure):
    _fields_ = [("nstations", C.c_int), ("stations", C.POINTER(gx_station_desc)),
                ("nfreqs", C.c_int), ("freqs", C.POINTER(gx_freq_desc)),
                ("nbaselines", C.c_int), ("baselines", C.POINTER(gx_baseline_desc)),
                ("subint_ns", C.c_int), ("guard_ns", C.c_int),
                ("fringe_rotation_order", C.c_int), ("array_stride", C.c_int),
                ("xmac_stride", C.c_int), ("write_autocorrs", C.c_int),
                ("max_data_bytes", C.c_int64), ("xstep", C.c_int), ("block_chunk", C.c_int),
                ("spectra_budget_bytes", C.c_int64)]


class gx_subint_desc(C.Structure):
    _fields_ = [("scan", C.c_int), ("sec", C.c_int), ("ns", C.c_int),
                ("scan_start_sec", C.c_double),
                ("interp", C.POINTER(C.c_double)),
                ("data", C.POINTER(C.c_void_p)),
                ("datalen", C.POINTER(C.c_int64)),
                ("control", C.POINTER(C.c_void_p)),
                ("controllen", C.c_int)]


class gx_layout_info(C.Structure):
    _fields_ = [("result_length", C.c_int64), ("nfreqs", C.c_int), ("nbaselines", C.c_int),
                ("nstations", C.c_int), ("blocks_per_send", C.c_int), ("xmac_stride", C.c_int),
                ("array_stride", C.c_int), ("fftchannels", C.c_int), ("nchan", C.c_int), ("xstep", C.c_int),
                ("block_chunk", C.c_int), ("chans_to_average", C.c_int)]


class JobDesc:
    """Owns the ctypes arrays behind a gx_job_desc."""

    def __init__(self, stations, freqs, baselines, **kw):
        self._st = (gx_station_desc * len(stations))(*stations)
        self._fr = (gx_freq_desc * len(freqs))(*freqs)
        nbl = max(1, len(baselines))
        self._bl = (gx_baseline_desc * nbl)(*baselines) if baselines else (gx_baseline_desc * 1)()
        self.desc = gx_job_desc()
        self.desc.nstations = len(stations)
        self.desc.stations = C.cast(self._st, C.POINTER(gx_station_desc))
        self.desc.nfreqs = len(freqs)
        self.desc.freqs = C.cast(self._fr, C.POINTER(gx_freq_desc))
        self.desc.nbaselines = len(baselines)
        self.desc.baselines = C.cast(self._bl, C.POINTER(gx_baseline_desc))
        for k, v in kw.items():
            setattr(self.desc, k, v)

    def ptr(self):
        return C.byref(self.desc)


def job_desc_from_spec(spec: JobSpec, xstep: int = GX_XSTEP_FP32, max_data_bytes: int = 0,
                       block_chunk: int = 0, spectra_budget_bytes: int = 0) -> JobDesc:
    """gx_job_desc for a JobSpec: the freq table is its subbands then its zoom
    freqs; each station records its subbands (all of them by default) in every
    polarisation and has the zoom freqs that lie within them."""
    spec.validate()
    freqs = []
    for sb in list(spec.subbands) + list(spec.zooms):
        f = gx_freq_desc()
        f.freq_mhz = sb.freq_mhz
        f.bw_mhz = sb.bw_mhz
        f.lower_sideband = 1 if sb.sideband.upper().startswith("L") else 0
        f.nchan = sb.nchan
        f.chans_to_average = spec.chans_to_avg
        freqs.append(f)
    nsb = len(spec.subbands)
    stations = []
    for s in range(spec.nstations):
        st = gx_station_desc()
        st.nbits = spec.nbits
        st.is_complex = 1 if spec.is_complex else 0
        st.framebytes = spec.framebytes
        sbs = spec.station_sb(s)
        st.nrecfreqs = len(sbs)
        for j, g in enumerate(sbs):
            st.recfreq[j] = g
            st.clock_offset_us[j] = 0.0
            st.clock_offset_delta_us[j] = 0.0
            st.lo_offset_hz[j] = 0.0
        st.nbands = spec.nbands
        b = 0
        pols = b""
        for j in range(len(sbs)):
            for p in spec.pols:
                st.band_localfreq[b] = j
                pols += p.encode()
                b += 1
        st.band_pol = pols
        zl = spec.station_zooms(s)
        st.nzoomfreqs = len(zl)
        b = 0
        pols = b""
        for j, (k, _) in enumerate(zl):
            st.zoomfreq[j] = nsb + k
            for p in spec.zpols:
                st.zoomband_localfreq[b] = j
                pols += p.encode()
                b += 1
        st.nzoombands = b
        st.zoomband_pol = pols
        c0 = spec.clock_us[s] if s < len(spec.clock_us) else 0.0
        st.clock_int_seconds = int(math.floor(c0 / 1e6 + 0.5))
        st.phase_cal_interval_hz = int(1e6 * spec.pcal_interval_mhz)
        st.interlaced = 1 if spec.mux_threads > 0 else 0
        st.nmuxthreads = spec.mux_threads
        for t in range(spec.mux_threads):
            st.muxthread[t] = t
        stations.append(st)
    baselines = []
    for a, bb, fl in baseline_plan(spec):
        bl = gx_baseline_desc()
        bl.ds1, bl.ds2 = a, bb
        bl.nfreqs = len(fl)
        for j, (f, pairs) in enumerate(fl):
            bl.freq[j] = f
            bl.npolprod[j] = len(pairs)
            for k, (b1, b2) in enumerate(pairs):
                bl.band1[j][k] = b1
                bl.band2[j][k] = b2
        baselines.append(bl)
    return JobDesc(stations, freqs, baselines,
                   subint_ns=spec.subint_ns, guard_ns=spec.guard_ns,
                   fringe_rotation_order=spec.fringe_rot_order, array_stride=spec.array_stride,
                   xmac_stride=spec.xmac_stride, write_autocorrs=1 if spec.write_autocorrs else 0,
                   max_data_bytes=max_data_bytes, xstep=xstep, block_chunk=block_chunk,
                   spectra_budget_bytes=spectra_budget_bytes)


class SubintDesc:
    """Owns the ctypes arrays behind a gx_subint_desc (host or device pointers)."""

    def __init__(self, scan: int, sec: int, ns: int, scan_start_sec: float,
                 data_ptrs: Sequence[int], datalens: Sequence[int], control_ptrs: Sequence[int],
                 controllen: int, interp: Optional[np.ndarray] = None):
        n = len(data_ptrs)
        self._data = (C.c_void_p * n)(*data_ptrs)
        self._len = (C.c_int64 * n)(*datalens)
        self._ctrl = (C.c_void_p * n)(*control_ptrs)
        self.desc = gx_subint_desc()
        self.desc.scan, self.desc.sec, self.desc.ns = scan, sec, ns
        self.desc.scan_start_sec = scan_start_sec
        if interp is not None:
            self._interp = np.ascontiguousarray(interp, dtype=np.float64).reshape(-1)
            self.desc.interp = self._interp.ctypes.data_as(C.POINTER(C.c_double))
        else:
            self._interp = None
            self.desc.interp = None
        self.desc.data = C.cast(self._data, C.POINTER(C.c_void_p))
        self.desc.datalen = C.cast(self._len, C.POINTER(C.c_int64))
        self.desc.control = C.cast(self._ctrl, C.POINTER(C.c_void_p))
        self.desc.controllen = controllen

    def ptr(self):
        return C.byref(self.desc)


def subint_desc_host(si, interp: Optional[np.ndarray], scan_start_sec: float = 0.0) -> SubintDesc:
    """SubintDesc over a synth.SubintInput's host arrays (kept alive by `si`)."""
    return SubintDesc(si.scan, si.sec, si.ns, scan_start_sec,
                      [d.ctypes.data for d in si.data], [len(d) for d in si.data],
                      [c.ctypes.data for c in si.control], len(si.control[0]), interp)
