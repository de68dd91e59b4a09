"""The DiFX-side binding (difx_b200/mpifxcorr: GpuCore, GpuMode), compiled
against the reference's own headers and Configuration, against the
reference's Core::processdata and Mode::process on the same slot.

GpuCore builds the gxcorr job from the reference Configuration (not from the
test's job description) and computes the delay interpolators as
Mode::setOffsets does, so these cases check the descriptor mapping, the
interpolators (complex data included: half the time span) and the result
layout of the integration as a maintainer would build it.  Tolerances as the
other parity tests: records within 1e-5 (diffDiFX metric), weights within
1e-6; per-block spectra within 1e-5 per band, data weights exact."""
import numpy as np
import pytest

from oracle import pyoracle
from tests import jobs

pytestmark = pytest.mark.gpu

REC_TOL = 1e-5
W_TOL = 1e-6

CASES = {
    "c1": lambda: (jobs.spec_c1(name="bind_c1", seed=41), dict(invalid_frac=0.02)),
    "cplx8_lsb": lambda: (jobs.spec_long("bind_cx", 8, "COMPLEX", "L", 1024, 43), dict(invalid_frac=0.03)),
    "real2_usb": lambda: (jobs.spec_long("bind_r2", 2, "REAL", "U", 1024, 45), dict(invalid_frac=0.03)),
}

needs = pytest.mark.skipif(not (pyoracle.reference_available() and pyoracle.shim_available()),
                           reason="reference or binding harness not built")


def _weights(g, r, prep, orc):
    rl, bl, bw, ac, acw = orc.layout(prep.jd)
    d = prep.jd.desc
    idx = []
    for f in range(d.nfreqs):
        for j in range(d.nbaselines):
            o = bw[f * d.nbaselines + j]
            if o >= 0:
                idx += [2 * o + p for p in range(d.baselines[j].npolprod[0])]
    nw = prep.spec.nbands * (2 if prep.spec.full_pol and len(prep.spec.pols) > 1 else 1)
    for s in range(d.nstations):
        idx += [2 * acw[s] + k for k in range(nw)]
    gf, rf = g.astype(np.complex64).view(np.float32), r.astype(np.complex64).view(np.float32)
    idx = np.array(idx)
    return float(np.max(np.abs(gf[idx] - rf[idx]) / np.maximum(np.abs(rf[idx]), 1e-30)))


@needs
@pytest.mark.parametrize("case", sorted(CASES))
def test_gpucore_slot_matches_core_processdata(case, oracle_lib):
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    ref = jobs.reference_for(prep.paths["input"])
    r = ref.process(prep.subs[0])
    b = pyoracle.Binding(prep.paths["input"])
    g = b.process(prep.subs[0], ref.result_length)
    b.close()
    rl, bl, bw, ac, acw = oracle_lib.layout(prep.jd)
    offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    m = jobs.record_metric(g, r, offs, spec.nchan)
    w = _weights(g, r, prep, oracle_lib)
    print(f"{case}: GpuCore vs Core::processdata record {m:.3g}, weights {w:.3g}")
    assert m < REC_TOL, m
    assert w < W_TOL, w


@needs
@pytest.mark.parametrize("case", ["c1", "cplx8_lsb"])
def test_gpumode_matches_mode_process(case, oracle_lib):
    """GpuMode::process over the first blocks of a slot against Mode::process:
    spectra, data weights, autocorrelations (parallel and cross-hand) and
    their weights, read through Mode's own accessors."""
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    ref = jobs.reference_for(prep.paths["input"])
    b = pyoracle.Binding(prep.paths["input"])
    b.process(prep.subs[0], ref.result_length)
    nblk = min(24, spec.blocks_per_send)
    for s in range(spec.nstations):
        gs, gw, ga, gwt = b.mode_blocks(s, nblk, spec.nbands, spec.nchan)
        rs, rw, ra, rwt = ref.mode_blocks(prep.subs[0], s, nblk, spec.nbands, spec.nchan)
        assert np.array_equal(gw, rw), (s, gw, rw)
        for k in range(nblk):
            for band in range(spec.nbands):
                den = np.mean(np.abs(rs[k, band]))
                if den == 0:
                    assert not np.any(gs[k, band]), (s, k, band)
                    continue
                e = np.mean(np.abs(gs[k, band] - rs[k, band])) / den
                assert e < REC_TOL, (s, k, band, e)
        for x in range(2):
            for band in range(spec.nbands):
                den = np.mean(np.abs(ra[x, band]))
                if den > 0:
                    assert np.mean(np.abs(ga[x, band] - ra[x, band])) / den < REC_TOL, (s, x, band)
        assert np.allclose(gwt, rwt, rtol=W_TOL, atol=0), (s, gwt, rwt)
    b.close()
