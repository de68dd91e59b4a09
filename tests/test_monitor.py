"""Monitoring spectra: the STA dump (Core::averageAndSendAutocorrs,
core.cpp:1180-1255) and the spectral kurtosis (Mode, mode.cpp:1237-1254,
1403-1454; Core::averageAndSendKurtosis, core.cpp:1378-1430) against the
records the compiled reference sends on its message bus (captured by the
oracle's difxmessage stand-in).

CPU: gx_sta over the reference's own Core result array equals the
reference's STA records bit for bit (the same autocorrelations, weights and
FP32 operations), with and without channel averaging.  GPU: the kurtosis
accumulated from the device spectra within 1e-4 (absolute) of the
reference's records, and the STA dump of the GPU result array within 1e-5
(relative) of the reference's."""
import numpy as np
import pytest

from oracle import pyoracle
from tests import jobs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")

STA, KURT = 1, 3


def _cases():
    return {
        "c1": lambda: jobs.spec_c1(name="mon_c1", nstations=3, seed=91),
        "c1_avg4": lambda: jobs.spec_c1(name="mon_a4", nstations=3, chans_to_avg=4, seed=92),
        "lsb": lambda: jobs.spec_lsb(name="mon_l", seed=93),
        "cplx8": lambda: jobs.spec_cplx8(name="mon_cx", seed=94),
    }


def _ref_records(spec, prep, dump, sta, kurt):
    ref = pyoracle.Reference(prep.paths["input"])
    ref.set_monitor(sta, kurt, dump)
    r = ref.process(prep.subs[0])
    recs = ref.take_monitor_records()
    ref.close()
    return r, recs


@needs_ref
@pytest.mark.parametrize("case", sorted(_cases()))
@pytest.mark.parametrize("dump", [32, 16])
def test_sta_from_reference_result_matches_reference_records(case, dump):
    from difx_b200.gxcorr import Correlator
    spec = _cases()[case]()
    prep = jobs.prepare(spec, [100_000_000], invalid_frac=0.03)
    r, recs = _ref_records(spec, prep, dump, True, False)
    stas = [x for x in recs if x["type"] == STA]
    assert stas
    c = Correlator.from_input(prep.paths["input"], device=-1)
    out, nch, sent = c.sta(r, dump)
    c.close()
    want = {(x["ds"], x["band"]): x for x in stas}
    for s in range(spec.nstations):
        for b in range(spec.nbands):
            x = want.get((s, b))
            assert bool(sent[s, b]) == (x is not None), (s, b)
            if x is None:
                continue
            assert nch[s, b] == x["nchan"]
            assert np.array_equal(out[s, b, :x["nchan"]], x["data"]), (case, s, b)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("case", sorted(_cases()))
def test_gpu_kurtosis_and_sta_match_reference_records(case):
    from difx_b200.gxcorr import Correlator
    spec = _cases()[case]()
    dump = 32
    prep = jobs.prepare(spec, [100_000_000], invalid_frac=0.03)
    r, recs = _ref_records(spec, prep, dump, True, True)
    c = Correlator.from_input(prep.paths["input"], device=0)
    c.set_kurtosis(dump)
    g = c.subint(prep.sds[0])
    sk, nch, valid = c.kurtosis()
    out, snch, sent = c.sta(g, dump)
    c.close()
    kur = [x for x in recs if x["type"] == KURT]
    assert kur
    worst = 0.0
    for x in kur:
        s, b = x["ds"], x["band"]
        assert valid[s] and nch[s, b] == x["nchan"]
        worst = max(worst, float(np.max(np.abs(sk[s, b, :x["nchan"]] - x["data"]))))
    assert {x["ds"] for x in kur} == {s for s in range(spec.nstations) if valid[s]}
    swor = 0.0
    for x in (x for x in recs if x["type"] == STA):
        s, b = x["ds"], x["band"]
        assert sent[s, b] and snch[s, b] == x["nchan"]
        swor = max(swor, float(np.max(np.abs(out[s, b, :x["nchan"]] - x["data"]) / np.abs(x["data"]))))
    print(f"\n{case}: kurtosis worst |diff| {worst:.3g}, STA worst relative {swor:.3g}")
    assert worst <= 1e-4, worst
    assert swor <= 1e-5, swor
