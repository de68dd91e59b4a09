"""Tensor-core X-step (tcgen05, FP16 and split FP16) against the FP64 oracle.

Every case runs the same subint through libgxcorr with the tensor-core X-step
and through the oracle evaluated in FP64 (precision GXO_FP64), and measures
  record error   mean |tc - ref| / mean |ref| per visibility record
                 (the metric of utilities/vis2screen/diffDiFX.py:146-151);
  element error  |tc - ref| / |ref| per visibility (one channel of one record).
Bounds:
  split FP16 (hi + lo, three products): every visibility within 1e-3 relative
    of FP64 (ELEM_TOL_HILO), every record within 1e-5;
  single FP16: every record within 1e-3 (REC_TOL_FP16).  One FP16 rounding
    per operand leaves ~3e-4 r.m.s. relative error on noise-dominated cross
    products, so single channels can pass 1e-3; their largest element error
    is printed, not bounded.
Weights come from the same weight kernel as the FP32 path and must match the
oracle within 1e-6 relative."""
import numpy as np
import pytest

from difx_b200 import capi
from difx_b200.jobfiles import JobSpec, Subband
from oracle import pyoracle
from tests import jobs

pytestmark = pytest.mark.gpu

ELEM_TOL_HILO = 1e-3
REC_TOL_HILO = 1e-5
REC_TOL_FP16 = 1e-3
W_TOL = 1e-6


def spec_c3small(**kw) -> JobSpec:
    """C3 shape (64 stations x 2 pols = 128 inputs, 8-bit complex) at 64 channels, 256 blocks."""
    base = dict(name="c3s", nstations=64, subbands=[Subband(6000.0, 16.0, "U", 64)], nbits=8, sampling="COMPLEX",
                subint_ns=1_024_000, execute_seconds=2, max_delay_us=150.0, seed=31)
    base.update(kw)
    return JobSpec(**base)


def spec_c3small_2bit(**kw) -> JobSpec:
    """The 2-bit real variant: 64 stations x 2 pols, 2-bit real, 2 subbands of 64 channels."""
    base = dict(name="c3s2", nstations=64, subbands=[Subband(6000.0 + 16 * i, 16.0, "U", 64) for i in range(2)],
                nbits=2,
                subint_ns=1_024_000, execute_seconds=2, max_delay_us=150.0, seed=37)
    base.update(kw)
    return JobSpec(**base)


CASES = {
    # name: (spec factory, prepare kwargs, block_chunk)
    "c3small": (spec_c3small, dict(rho=0.01), 0),
    "c3small_2bit": (spec_c3small_2bit, dict(rho=0.02, invalid_frac=0.01), 0),
    "c1_padded_chunked": (jobs.spec_c1, dict(), 40),
    "lsb_ksplit_chunked": (jobs.spec_lsb, dict(invalid_frac=0.03), 200),
    "cplx8": (jobs.spec_cplx8, dict(invalid_frac=0.05), 0),
    # FFT lengths of the register-resident F-step
    "cplx8_4096": (lambda: jobs.spec_long("tcx4k", 8, "COMPLEX", "U", 4096, 61), dict(invalid_frac=0.03), 0),
    "real2_8192_lsb": (lambda: jobs.spec_long("tcr8k", 2, "REAL", "L", 4096, 67), dict(invalid_frac=0.03), 0),
    # 64 stations x 2 pols at 512 channels, chunks of 24 blocks (partial K-tiles, accumulation over chunks)
    "c3_512_chunked": (lambda: spec_c3small(name="c3p", subbands=[Subband(6000.0, 16.0, "U", 512)],
                                            subint_ns=2_048_000, seed=71), dict(rho=0.01), 24),
    # single polarisation
    "cplx8_2048_singlepol": (lambda: jobs.spec_long("tcsp", 8, "COMPLEX", "U", 2048, 73, pols=("R",)),
                             dict(invalid_frac=0.03), 0),
}

_prepared = {}


def _prepared_case(name):
    if name not in _prepared:
        factory, kw, chunk = CASES[name]
        spec = factory()
        prep = jobs.prepare(spec, [100_000_000], **kw)
        _prepared[name] = (spec, prep, chunk)
    return _prepared[name]


_fp64 = {}


def _fp64_ref(name, orc):
    if name not in _fp64:
        spec, prep, _ = _prepared_case(name)
        p = orc.params(precision=pyoracle.FP64, nthreads=1, num_buffered_ffts=spec.num_buffered_ffts,
                       xc_avg_ns=spec.uvshift_interval_ns, ac_avg_ns=spec.ac_avg_interval_ns)
        _fp64[name] = orc.subint(prep.jd, prep.sds[0], p)
    return _fp64[name]


def _errors(g, ref, offs, nchan):
    rec = jobs.record_metric(g, ref, offs, nchan)
    idx = np.concatenate([np.arange(o, o + nchan) for o in offs])
    gv, rv = g[idx].astype(np.complex128), ref[idx].astype(np.complex128)
    nz = np.abs(rv) > 0
    elem = float(np.max(np.abs(gv[nz] - rv[nz]) / np.abs(rv[nz]))) if nz.any() else 0.0
    zero_abs = float(np.max(np.abs(gv[~nz]))) if (~nz).any() else 0.0
    return rec, elem, zero_abs


def _weights_rel(g, ref, jd, spec, orc):
    rl, bl, bw, ac, acw = orc.layout(jd)
    d = jd.desc
    idx = []
    for f in range(d.nfreqs):
        for j in range(d.nbaselines):
            o = bw[f * d.nbaselines + j]
            if o >= 0:
                idx += [2 * o + p for p in range(d.baselines[j].npolprod[0])]
    nw = spec.nbands * (2 if spec.full_pol and len(spec.pols) > 1 else 1)
    for s in range(d.nstations):
        idx += [2 * acw[s] + k for k in range(nw)]
    idx = np.array(idx)
    gf, rf = g.view(np.float32), ref.astype(np.complex64).view(np.float32)
    return float(np.max(np.abs(gf[idx] - rf[idx]) / np.maximum(np.abs(rf[idx]), 1e-30)))


def _run(name, xstep, orc):
    from difx_b200 import gxcorr
    spec, prep, chunk = _prepared_case(name)
    jd = capi.job_desc_from_spec(spec, xstep=xstep, block_chunk=chunk)
    c = gxcorr.Correlator.from_desc(jd)
    g = c.subint(prep.sds[0])
    c.close()
    ref = _fp64_ref(name, orc)
    rl, bl, bw, ac, acw = orc.layout(prep.jd)
    offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    return g, ref, offs, spec, prep


@pytest.mark.parametrize("case", sorted(CASES))
def test_tc_hilo_every_visibility_within_1e3(case, oracle_lib):
    g, ref, offs, spec, prep = _run(case, capi.GX_XSTEP_TC_FP16_HILO, oracle_lib)
    rec, elem, zero_abs = _errors(g, ref, offs, spec.nchan)
    print(f"{case} hi+lo: record {rec:.3g} element max {elem:.3g}")
    assert elem <= ELEM_TOL_HILO, elem
    assert rec <= REC_TOL_HILO, rec
    assert zero_abs == 0.0, zero_abs
    assert _weights_rel(g, ref, prep.jd, spec, oracle_lib) < W_TOL


@pytest.mark.parametrize("case", sorted(CASES))
def test_tc_fp16_records_within_1e3(case, oracle_lib):
    g, ref, offs, spec, prep = _run(case, capi.GX_XSTEP_TC_FP16, oracle_lib)
    rec, elem, zero_abs = _errors(g, ref, offs, spec.nchan)
    print(f"{case} fp16: record {rec:.3g} element max {elem:.3g}")
    assert rec <= REC_TOL_FP16, rec
    assert zero_abs == 0.0, zero_abs
    assert _weights_rel(g, ref, prep.jd, spec, oracle_lib) < W_TOL


def test_tc_matches_fp32_path(oracle_lib):
    """Split-FP16 tensor-core and FP32 plain X-steps agree with each other as
    closely as each agrees with FP64."""
    g_tc, ref, offs, spec, prep = _run("c3small", capi.GX_XSTEP_TC_FP16_HILO, oracle_lib)
    g_fp, _, _, _, _ = _run("c3small", capi.GX_XSTEP_FP32, oracle_lib)
    rec_fp, elem_fp, _ = _errors(g_fp, ref, offs, spec.nchan)
    rec_x = jobs.record_metric(g_tc, g_fp, offs, spec.nchan)
    print(f"fp32 vs fp64: record {rec_fp:.3g} element {elem_fp:.3g}; tc vs fp32 record {rec_x:.3g}")
    assert rec_fp <= 1e-5
    assert rec_x <= 2e-5


def test_tc_scales_change_nothing(oracle_lib):
    """Per-station/per-channel power-of-two operand scales are divided out exactly."""
    from difx_b200 import gxcorr
    spec, prep, _ = _prepared_case("cplx8")
    jd = capi.job_desc_from_spec(spec, xstep=capi.GX_XSTEP_TC_FP16_HILO)
    c = gxcorr.Correlator.from_desc(jd)
    base = c.subint(prep.sds[0])
    rng = np.random.default_rng(5)
    for s in range(spec.nstations):
        for b in range(spec.nbands):
            c.set_tc_scales(s, b, 2.0 ** rng.integers(-4, 5, spec.nchan))
    scaled = c.subint(prep.sds[0])
    c.close()
    ref = _fp64_ref("cplx8", oracle_lib)
    rl, bl, bw, ac, acw = oracle_lib.layout(prep.jd)
    offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    rec, elem, _ = _errors(scaled, ref, offs, spec.nchan)
    assert elem <= ELEM_TOL_HILO and rec <= REC_TOL_HILO, (rec, elem)
    assert jobs.record_metric(scaled, base, offs, spec.nchan) <= 1e-5
