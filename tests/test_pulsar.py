"""Pulsar binning (Core::processdata, core.cpp:803-811, 913-958, 1079-1086;
Core::uvshiftAndAverage, core.cpp:1439-1470; Polyco, polyco.cpp;
Configuration::processPulsarConfig, configuration.cpp:3400-3520): every
channel of every FFT block goes to the bin of its pulse phase (the block's
mean phase from the polyco plus the channel's dispersion offset); cross
products and baseline weights are accumulated per bin, or summed with the
bin weights when the output is scrunched.

Cases (2-bit real, 4 x 16 MHz, 128 channels, 3 stations; a 503.7 Hz pulsar,
DM 500, polyco centred on the job):
  bins8        8 bins of equal phase width
  bins5_lsb    5 bins, lower sideband
  scrunch4     4 bins scrunched with weights 1, 0.5, -0.25, 0

Layout on the CPU against the compiled reference's Configuration; on the GPU
the Core result array against Core::processdata of the compiled reference
(one process thread): every record within 1e-5 (the diffDiFX metric; the
binned crosses accumulate in the reference's order, the spectra differ from
the reference's by FP32 FFT rounding), baseline and autocorrelation weights
within 1e-6 (they come out identical)."""
import os

import numpy as np
import pytest

from difx_b200.jobfiles import baseline_plan, write_job
from oracle import pyoracle
from tests import jobs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")


def _case(name):
    if name == "bins8":
        return jobs.spec_c1(name="psr8", nstations=3, pulsar_bins=8, seed=71)
    if name == "bins5_lsb":
        return jobs.spec_lsb(name="psr5l", pulsar_bins=5, seed=73)
    if name == "scrunch4":
        return jobs.spec_c1(name="psrs4", nstations=3, pulsar_bins=4, pulsar_scrunch=True,
                            pulsar_bin_weights=[1.0, 0.5, -0.25, 0.0], seed=75)
    raise ValueError(name)


CASES = ["bins8", "bins5_lsb", "scrunch4"]


def _records(spec, offsets):
    """(offset, channels) of every record: per baseline-freq the records of
    every bin (one when scrunched) and product, then the autocorrelations."""
    _, bl, _, ac, _ = offsets
    n = spec.nchan // spec.chans_to_avg
    binloop = 1 if spec.pulsar_scrunch else spec.pulsar_bins
    plan = baseline_plan(spec)
    nbl = len(plan)
    out = []
    for f in range(len(spec.subbands)):
        for j, (_, _, fl) in enumerate(plan):
            o = bl[f * nbl + j]
            if o < 0:
                continue
            npp = [len(p) for g, p in fl if g == f][0]
            out += [(o + q * n, n) for q in range(binloop * npp)]
    nauto = spec.nbands * (2 if len(spec.pols) > 1 and spec.full_pol else 1)
    for s in range(spec.nstations):
        out += [(ac[s] + b * n, n) for b in range(nauto)]
    return out


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_pulsar_layout_matches_reference(name):
    from difx_b200.gxcorr import Correlator
    spec = _case(name)
    paths = write_job(spec, os.path.join(jobs._TMP, "psrlayout_" + name))
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
def test_pulsar_bins_are_all_used_in_reference():
    """The synthetic pulsar turns several times per subint, so every bin of
    the reference's binned output holds data."""
    from difx_b200.gxcorr import Correlator
    spec = _case("bins8")
    prep = jobs.prepare(spec, [100_000_000])
    ref = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    c = Correlator.from_input(prep.paths["input"], device=-1)
    recs = _records(spec, c.offsets())
    c.close()
    nz = [np.count_nonzero(ref[o:o + n]) for o, n in recs]
    assert min(nz) > 0


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_gpu_pulsar_binning_matches_reference(name):
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
    ident = 0
    for o, n in recs:
        r, q = ref[o:o + n], g[o:o + n]
        mask[o:o + n] = False
        m = np.mean(np.abs(r))
        assert m > 0, (o, n)
        worst = max(worst, float(np.mean(np.abs(q - r)) / m))
        ident += int(np.array_equal(q, r))
    rw, gw = ref[mask].view(np.float32), g[mask].view(np.float32)
    assert np.count_nonzero(rw) > 0
    wrel = float(np.max(np.abs(gw - rw) / np.maximum(np.abs(rw), 1e-30)))
    print(f"\n{name}: {len(recs)} records ({ident} bit-identical), worst record {worst:.3g}, weights {wrel:.3g}")
    assert worst <= 1e-5, worst
    assert wrel <= 1e-6, wrel
