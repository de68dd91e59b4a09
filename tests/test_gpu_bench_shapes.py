"""Parity at the benchmarked shapes, through the bench's own job descriptors.

The bench times C3 (64 stations x 2 pol, 4 x 64 MHz, 4096 channels, 8-bit
complex VDIF), its 2-bit real variant (8192-point real transforms) and C2
(16 stations, 16 x 32 MHz bands, 256 channels) with descriptors built by
``bench.workload_spec`` and ``capi.job_desc_from_spec``; the device picks the
pass length, the K-split and (tensor-core form) the 4-D TMA map from those
shapes.  These cases run the same descriptors over short subints (32 FFT
blocks for C3; two passes of 4100 blocks for C2) on the bench's tiled,
seeded input with 1 % invalid frames, so that the tiling of the timed runs is
the tiling checked here:

  split-FP16 tensor cores vs the FP64 oracle   every visibility <= 1e-3
                                               relative (floored at its
                                               record's mean |V|), every
                                               record <= 1e-5
  single-FP16 tensor cores vs the FP64 oracle  every record <= 1e-3
  FP32 plain vs the compiled reference         every record <= 1e-5
  (Core::processdata on all host cores)        (diffDiFX metric), weights 1e-6
Record error = mean |gpu - ref| / mean |ref| (utilities/vis2screen/
diffDiFX.py:146-151); element error = |gpu - ref| / |ref| per channel."""
import os

import numpy as np
import pytest

import bench
from difx_b200 import capi
from difx_b200.gxcorr import Correlator
from difx_b200.jobfiles import write_job
from oracle import pyoracle
from tests import jobs

pytestmark = pytest.mark.gpu

ELEM_TOL_HILO = 1e-3
REC_TOL = 1e-5
REC_TOL_FP16 = 1e-3
W_TOL = 1e-6

# workload: (subint ns, block_chunk for the FP32 form: 0 = the library's choice)
SHAPES = {
    "c3": (32 * 64_000, 0),
    "c3_2bit": (32 * 64_000, 0),
    # two passes of the library's own FP32 pass length (4096 blocks at most per 2 GB of spectra)
    "c2": (8200 * 8_000, 0),
}

_cache = {}


def _prepared(name):
    if name not in _cache:
        subint_ns, _ = SHAPES[name]
        spec = bench.workload_spec(name, subint_ns=subint_ns)
        d = os.path.join(jobs._TMP, f"bench_shape_{name}")
        paths = write_job(spec, d)
        with open(paths["threads"], "w") as f:
            f.write(f"{'NUMBER OF CORES:':<20}1\n{os.cpu_count() or 1}\n")
        si = bench.build_input(spec, 200_000_000, rho=bench.RHO[name])
        m = Correlator.from_input(paths["input"], device=-1)
        interp = np.array([m.interpolator(s, 0, si.sec, si.ns) for s in range(spec.nstations)])
        m.close()
        sd = capi.subint_desc_host(si, interp)
        maxbytes = max(len(x) for x in si.data)
        _cache[name] = dict(spec=spec, paths=paths, si=si, sd=sd, maxbytes=maxbytes, jd=capi.job_desc_from_spec(spec))
    return _cache[name]


def _run_gpu(name, xstep):
    p = _prepared(name)
    jd = capi.job_desc_from_spec(p["spec"], xstep=xstep, max_data_bytes=p["maxbytes"])
    c = Correlator.from_desc(jd)
    info = c.info
    g = c.subint(p["sd"])
    c.close()
    return g, info


def _fp64(name, orc):
    key = ("fp64", name)
    if key not in _cache:
        p = _prepared(name)
        spec = p["spec"]
        prm = orc.params(precision=pyoracle.FP64, nthreads=1, num_buffered_ffts=spec.num_buffered_ffts,
                         xc_avg_ns=spec.uvshift_interval_ns, ac_avg_ns=spec.ac_avg_interval_ns)
        _cache[key] = orc.subint(p["jd"], p["sd"], prm)
    return _cache[key]


def _reference(name):
    key = ("ref", name)
    if key not in _cache:
        p = _prepared(name)
        with pyoracle.Reference(p["paths"]["input"]) as ref:
            _cache[key] = ref.process(p["si"])
    return _cache[key]


def _weight_rel(g, ref, jd, spec, orc):
    rl, bl, bw, ac, acw = orc.layout(jd)
    d = jd.desc
    idx = []
    for f in range(d.nfreqs):
        for j in range(d.nbaselines):
            o = bw[f * d.nbaselines + j]
            if o >= 0:
                idx += [2 * o + q for q in range(d.baselines[j].npolprod[0])]
    nw = spec.nbands * (2 if spec.full_pol and len(spec.pols) > 1 else 1)
    for s in range(d.nstations):
        idx += [2 * acw[s] + k for k in range(nw)]
    idx = np.array(idx)
    gf, rf = g.view(np.float32), ref.astype(np.complex64).view(np.float32)
    return float(np.max(np.abs(gf[idx] - rf[idx]) / np.maximum(np.abs(rf[idx]), 1e-30)))


def _errors(g, ref, name, orc):
    """(record error, largest element error, zero-reference magnitude, weight
    error, element statistics): element error |g - ref| / |ref| per channel,
    and |g - ref| / max(|ref|, mean |ref| of its record) (relative, floored at
    the record's mean magnitude)."""
    p = _prepared(name)
    spec, jd = p["spec"], p["jd"]
    rl, bl, bw, ac, acw = orc.layout(jd)
    offs = jobs.record_offsets(jd, bl, ac, spec)
    rec = jobs.record_metric(g, ref, offs, spec.nchan)
    idx = np.stack([np.arange(o, o + spec.nchan) for o in offs])
    gv, rv = g[idx].astype(np.complex128), ref[idx].astype(np.complex128)
    err, mag = np.abs(gv - rv), np.abs(rv)
    mean = mag.mean(axis=1, keepdims=True)
    nz = mag > 0
    rel = np.where(nz, err / np.where(nz, mag, 1.0), 0.0)
    floored = err / np.maximum(mag, np.maximum(mean, 1e-300))
    k = np.unravel_index(np.argmax(rel), rel.shape)
    stats = dict(elem_max=float(rel.max()), floored_max=float(floored.max()),
                 n_over_1e3=int((rel > 1e-3).sum()), n_vis=int(rel.size),
                 worst_mag_over_mean=float(mag[k] / mean[k[0], 0]) if mean[k[0], 0] > 0 else 0.0,
                 abs_over_mean_max=float((err / np.maximum(mean, 1e-300)).max()))
    zero_abs = float(err[~nz].max()) if (~nz).any() else 0.0
    return rec, stats, zero_abs, _weight_rel(g, ref, jd, spec, orc)


@pytest.mark.parametrize("name", ["c3", "c3_2bit"])
def test_bench_shape_tc_hilo_vs_fp64(name, oracle_lib):
    """Split FP16 against FP64.  Every visibility within 1e-3 relative of
    FP64, relative to max(|V|, the mean |V| of its record): at 1.3e8
    noise-dominated visibilities a few channels have |V| near 1e-4 of their
    record's mean, where any FP32-accumulated form (the FP32 plain form
    measured beside it here included) exceeds 1e-3 of |V| itself.  Those
    counts are printed for both forms."""
    g, info = _run_gpu(name, capi.GX_XSTEP_TC_FP16_HILO)
    assert info.block_chunk == _prepared(name)["spec"].blocks_per_send  # one pass, as in the timed runs
    ref = _fp64(name, oracle_lib)
    rec, st, zero_abs, wrel = _errors(g, ref, name, oracle_lib)
    g32, _ = _run_gpu(name, capi.GX_XSTEP_FP32)
    rec32, st32, _, _ = _errors(g32, ref, name, oracle_lib)
    print(f"\n{name} split FP16 vs FP64: record {rec:.3g}, weights {wrel:.3g}, {st}")
    print(f"{name} FP32 plain vs FP64: record {rec32:.3g}, {st32}")
    assert st["floored_max"] <= ELEM_TOL_HILO, st
    assert rec <= REC_TOL, rec
    assert zero_abs == 0.0, zero_abs
    assert wrel < W_TOL, wrel


@pytest.mark.parametrize("name", ["c3", "c3_2bit"])
def test_bench_shape_tc_fp16_vs_fp64(name, oracle_lib):
    g, _ = _run_gpu(name, capi.GX_XSTEP_TC_FP16)
    rec, st, zero_abs, wrel = _errors(g, _fp64(name, oracle_lib), name, oracle_lib)
    print(f"\n{name} FP16 vs FP64: record {rec:.3g}, {st}")
    assert rec <= REC_TOL_FP16, rec
    assert zero_abs == 0.0, zero_abs
    assert wrel < W_TOL, wrel


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("name", ["c3", "c3_2bit", "c2"])
def test_bench_shape_fp32_vs_reference(name, oracle_lib):
    g, info = _run_gpu(name, capi.GX_XSTEP_FP32)
    if name == "c2":
        assert _prepared(name)["spec"].blocks_per_send > info.block_chunk  # several passes
    rec, st, zero_abs, wrel = _errors(g, _reference(name), name, oracle_lib)
    print(f"\n{name} FP32 vs reference: record {rec:.3g}, weights {wrel:.3g}, pass {info.block_chunk} blocks, {st}")
    assert rec <= REC_TOL, rec
    assert wrel < W_TOL, wrel
