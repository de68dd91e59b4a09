"""Small seeded correlation jobs shared by the tests.

Shapes follow the benchmark configurations (2-bit real VDIF with 2 pols per
subband; 8-bit complex VDIF) at sizes the oracle finishes in seconds."""
from __future__ import annotations

import dataclasses
import os
import tempfile
from typing import List, Optional

import numpy as np

from difx_b200 import capi, synth
from difx_b200.jobfiles import JobSpec, Subband, write_job

_TMP = os.environ.get("GX_TEST_TMP") or tempfile.mkdtemp(prefix="gxtests_")


def spec_c1(**kw) -> JobSpec:
    """C1 shape: 4 stations, 4 x 16 MHz USB subbands, 2 pols, 128 channels, 2-bit real."""
    base = dict(name="c1", nstations=4, subbands=[Subband(8400.0 + 16 * i, 16.0, "U", 128) for i in range(4)],
                nbits=2, subint_ns=8_000_000, execute_seconds=2, max_delay_us=200.0, seed=3)
    base.update(kw)
    return JobSpec(**base)


def spec_lsb(**kw) -> JobSpec:
    base = dict(name="lsb", nstations=3, subbands=[Subband(8432.0, 16.0, "L", 128), Subband(8448.0, 16.0, "L", 128)],
                nbits=2, subint_ns=4_000_000, execute_seconds=2, max_delay_us=300.0, seed=5)
    base.update(kw)
    return JobSpec(**base)


def spec_cplx8(**kw) -> JobSpec:
    """Complex 8-bit (C3 sample format) at a small size."""
    base = dict(name="cx8", nstations=3, subbands=[Subband(6000.0 + 16 * i, 16.0, "U", 256) for i in range(2)],
                nbits=8, sampling="COMPLEX", subint_ns=4_096_000, execute_seconds=2, max_delay_us=150.0, seed=7)
    base.update(kw)
    return JobSpec(**base)


def spec_c2small(**kw) -> JobSpec:
    """C2 shape: 16 stations, 8 x 32 MHz, 2 pols, 256 channels, 2-bit real (short subint)."""
    base = dict(name="c2s", nstations=16, subbands=[Subband(8200.0 + 32 * i, 32.0, "U", 256) for i in range(8)],
                nbits=2, subint_ns=2_048_000, execute_seconds=2, max_delay_us=400.0, seed=11)
    base.update(kw)
    return JobSpec(**base)


def spec_long(name: str, nbits: int, sampling: str, sideband: str, nchan: int, seed: int, **kw) -> JobSpec:
    """Long transforms (2048- to 8192-point FFTs): 3 stations, 2 x 16 MHz subbands, 2 pols, 64 FFT blocks."""
    f0 = 6000.0 if sampling == "COMPLEX" else 8400.0
    if sideband == "L":
        f0 += 16.0
    fft_us = nchan / 16.0 if sampling == "COMPLEX" else 2 * nchan / 32.0
    base = dict(name=name, nstations=3, subbands=[Subband(f0 + 16 * i, 16.0, sideband, nchan) for i in range(2)],
                nbits=nbits, sampling=sampling, subint_ns=int(64 * fft_us * 1000), execute_seconds=2,
                max_delay_us=200.0, seed=seed)
    base.update(kw)
    return JobSpec(**base)


@dataclasses.dataclass
class Prepared:
    spec: JobSpec
    paths: dict
    jd: capi.JobDesc
    subs: List[synth.SubintInput]
    interps: List[np.ndarray]
    sds: List[capi.SubintDesc]


def prepare(spec: JobSpec, sub_starts_ns: List[int], rho: float = 0.05, invalid_frac: float = 0.0,
            fill_frac: float = 0.0, bad_blocks=None, interp_source=None) -> Prepared:
    """Write the job files, synthesise VDIF, slice subints, and compute the
    interpolators with the reference harness when available, else with the
    host model of libgxcorr (device -1 handle)."""
    d = os.path.join(_TMP, spec.name + f"_{spec.seed}")
    paths = write_job(spec, d)
    streams = synth.streams_for_job(spec, sub_starts_ns, rho=rho, seed=spec.seed, invalid_frac=invalid_frac,
                                    fill_frac=fill_frac)
    subs = [synth.build_subint(spec, streams, t, bad_blocks) for t in sub_starts_ns]
    interps = []
    for si in subs:
        interps.append(interpolators(paths["input"], spec, si, interp_source))
    sds = [capi.subint_desc_host(si, ip) for si, ip in zip(subs, interps)]
    return Prepared(spec, paths, capi.job_desc_from_spec(spec), subs, interps, sds)


def interpolators(inputfile: str, spec: JobSpec, si, source=None) -> np.ndarray:
    from oracle import pyoracle
    if source != "host" and pyoracle.reference_available():
        ref = reference_for(inputfile)
        return np.array([ref.interpolator(s, 0, si.sec, si.ns) for s in range(spec.nstations)])
    from difx_b200.gxcorr import Correlator
    c = Correlator.from_input(inputfile, device=-1)
    out = np.array([c.interpolator(s, 0, si.sec, si.ns) for s in range(spec.nstations)])
    c.close()
    return out


_refs = {}


def reference_for(inputfile: str):
    from oracle import pyoracle
    if inputfile not in _refs:
        _refs[inputfile] = pyoracle.Reference(inputfile)
    return _refs[inputfile]


def record_metric(a: np.ndarray, b: np.ndarray, offsets, nchan: int) -> float:
    """Largest per-record mean|a-b| / mean|b| over the visibility records
    (the metric of utilities/vis2screen/diffDiFX.py:146-151)."""
    worst = 0.0
    for o in offsets:
        ra, rb = a[o:o + nchan], b[o:o + nchan]
        den = np.mean(np.abs(rb))
        if den == 0:
            if np.any(ra != 0):
                return float("inf")
            continue
        worst = max(worst, float(np.mean(np.abs(ra - rb)) / den))
    return worst


def record_offsets(jd: capi.JobDesc, blofs, acofs, spec: JobSpec, nchan: int = 0):
    """Start offsets of every cross and auto record (one per polproduct / band)
    of records of nchan channels (default: the job's output channels)."""
    nchan = nchan or spec.nchan // spec.chans_to_avg
    out = []
    d = jd.desc
    nbl = d.nbaselines
    for f in range(d.nfreqs):
        for j in range(nbl):
            o = blofs[f * nbl + j]
            if o < 0:
                continue
            lf = [d.baselines[j].freq[k] for k in range(d.baselines[j].nfreqs)].index(f)
            for p in range(d.baselines[j].npolprod[lf]):
                out.append(o + p * nchan)
    nauto = spec.nbands * (2 if len(spec.pols) > 1 and spec.full_pol else 1)
    for s in range(d.nstations):
        for b in range(nauto):
            out.append(acofs[s] + b * nchan)
    return out
