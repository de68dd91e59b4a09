"""Multiple phase centres (Core::uvshiftAndAverage, core.cpp:1431-1938;
Configuration, configuration.cpp:2366-2373, 2455-2566): the cross products
of each uv-shift interval are rotated by every phase centre's differential
delay against the pointing centre and added into that centre's records; the
shift decorrelation factors (time smearing and delay window) are summed per
baseline, freq and centre; Mode correlates at the pointing centre.

Cases (2-bit real, 4 x 16 MHz, 128 channels, 3 stations, seeded phase-centre
offsets of up to 20 ns and rates of up to 2 ns/s):
  pc3        3 phase centres, 2 ms uv-shift interval (4 intervals of 250 blocks)
  pc2_ragged 2 phase centres, 3 ms interval (370, 370 and 260 blocks)
  pc3_lsb    lower sideband
  pc2_avg    with channel averaging (CHANS TO AVG 4)

Layout on the CPU against the compiled reference's Configuration; on the GPU
the Core result array against Core::processdata of the compiled reference
(one process thread): every record within 1e-5 (the diffDiFX metric),
baseline and autocorrelation weights and shift decorrelation factors within
1e-6."""
import os

import numpy as np
import pytest

from difx_b200.jobfiles import baseline_plan, write_job
from oracle import pyoracle
from tests import jobs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")


def _case(name):
    if name == "pc3":
        return jobs.spec_c1(name="pc3", nstations=3, phase_centres=3, uvshift_interval_ns=2_000_000, seed=61)
    if name == "pc2_ragged":
        return jobs.spec_c1(name="pc2r", nstations=3, phase_centres=2, uvshift_interval_ns=3_000_000, seed=63)
    if name == "pc3_lsb":
        return jobs.spec_lsb(name="pc3l", phase_centres=3, uvshift_interval_ns=1_000_000, seed=65)
    if name == "pc2_avg":
        return jobs.spec_c1(name="pc2a", nstations=3, phase_centres=2, uvshift_interval_ns=2_000_000,
                            chans_to_avg=4, seed=67)
    raise ValueError(name)


CASES = ["pc3", "pc2_ragged", "pc3_lsb", "pc2_avg"]


def _records(spec, offsets):
    """(offset, channels) of every record: each baseline-freq's records for
    every phase centre and polarisation product, then the autocorrelations."""
    _, bl, _, ac, _ = offsets
    n = spec.nchan // spec.chans_to_avg
    plan = baseline_plan(spec)
    nbl = len(plan)
    out = []
    for f in range(len(spec.subbands)):
        for j, (_, _, fl) in enumerate(plan):
            o = bl[f * nbl + j]
            if o < 0:
                continue
            npp = [len(p) for g, p in fl if g == f][0]
            out += [(o + q * n, n) for q in range(spec.phase_centres * npp)]
    nauto = spec.nbands * (2 if len(spec.pols) > 1 and spec.full_pol else 1)
    for s in range(spec.nstations):
        out += [(ac[s] + b * n, n) for b in range(nauto)]
    return out


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_phase_centre_layout_matches_reference(name):
    from difx_b200.gxcorr import Correlator
    spec = _case(name)
    paths = write_job(spec, os.path.join(jobs._TMP, "pclayout_" + name))
    c = Correlator.from_input(paths["input"], device=-1)
    try:
        g = c.offsets()
    finally:
        c.close()
    nbl = spec.nstations * (spec.nstations - 1) // 2
    with pyoracle.Reference(paths["input"]) as ref:
        r = ref.layout(len(spec.subbands), nbl, spec.nstations)
    assert g[0] == r[0]
    for a, b in zip(g[1:], r[1:]):
        np.testing.assert_array_equal(a, b)


@needs_ref
def test_phase_centre_decorrelation_section_in_reference():
    """The reference fills exactly the floats the layout reserves for the
    shift decorrelation factors between the baseline weights and the
    autocorrelations: one per phase centre, each the sum over the subint's
    intervals of nswidth x smearing factors (close to the subint length)."""
    from difx_b200.gxcorr import Correlator
    spec = _case("pc3")
    prep = jobs.prepare(spec, [100_000_000])
    ref = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    c = Correlator.from_input(prep.paths["input"], device=-1)
    rl, bl, bw, ac, acw = c.offsets()
    c.close()
    fl = ref.view(np.float32)
    # the section: after the last baseline's weights (4 products: 2 complex floats), before the autocorrelations
    bw_end = max(int(x) for x in bw if x >= 0) + 2
    lo, hi = 2 * bw_end, 2 * int(ac[0])
    sec = fl[lo:hi]
    assert sec.size > 0
    v = sec[sec != 0]
    # 3 centres per baseline-freq, padded to whole complex floats
    assert v.size == 3 * 4 * 3, v.size
    assert np.all(np.abs(v - spec.subint_ns) < 0.01 * spec.subint_ns), v


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_gpu_phase_centres_match_reference(name):
    from difx_b200 import gxcorr
    spec = _case(name)
    prep = jobs.prepare(spec, [100_000_000])
    ref = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    c = gxcorr.Correlator.from_input(prep.paths["input"])
    g = c.subint(prep.sds[0])
    offsets = c.offsets()
    c.close()
    recs = _records(spec, offsets)
    mask = np.ones(len(ref), bool)
    worst = 0.0
    for o, n in recs:
        r, q = ref[o:o + n], g[o:o + n]
        mask[o:o + n] = False
        m = np.mean(np.abs(r))
        assert m > 0, (o, n)
        worst = max(worst, float(np.mean(np.abs(q - r)) / m))
    rw, gw = ref[mask].view(np.float32), g[mask].view(np.float32)
    assert np.count_nonzero(rw) > 0
    wrel = float(np.max(np.abs(gw - rw) / np.maximum(np.abs(rw), 1e-30)))
    print(f"\n{name}: {len(recs)} records, worst record {worst:.3g}, weights and decorrelation {wrel:.3g}")
    assert worst <= 1e-5, worst
    assert wrel <= 1e-6, wrel
