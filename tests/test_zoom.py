"""Zoom bands (Configuration, configuration.cpp:1701-1753, 2774-2880; Mode,
mode.cpp:184-196, 379-391; Core, core.cpp:1273-1370): a zoom freq is a
channel range of the recorded freq that contains it, and its visibilities,
autocorrelations and weights are those of its parent bands' channels.

Cases (2-bit real, 16 MHz subbands of 128 channels):
  shifted   stations record shifted subbands, so one zoom freq has a
            different parent and channel offset per station (80 or 16);
            zoom freqs only
  mixed     recorded freqs and two zoom freqs correlated together
  onepol    zoom bands of one polarisation (their cross-pol
            autocorrelations are slices of the parent's)
  lsb       lower-sideband subbands and zoom freq
  avg       zoom freqs with channel averaging (CHANS TO AVG 4)

The layout (offsets of every record) is compared with the compiled
reference's Configuration on the CPU; on the GPU the Core result array of
one subint is compared with Core::processdata of the compiled reference
(all records within 1e-5, the diffDiFX metric; weights within 1e-6)."""
import numpy as np
import pytest

from difx_b200.jobfiles import Subband
from oracle import pyoracle
from tests import jobs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")

_SB = [Subband(8400.0, 16.0, "U", 128), Subband(8408.0, 16.0, "U", 128), Subband(8416.0, 16.0, "U", 128)]
_SBL = [Subband(8432.0, 16.0, "L", 128), Subband(8424.0, 16.0, "L", 128), Subband(8448.0, 16.0, "L", 128)]


def _case(name):
    base = dict(name="z_" + name, nstations=3, subbands=_SB, station_subbands=[[0, 2], [1, 2], [0, 2]], seed=51)
    if name == "shifted":
        base.update(zooms=[Subband(8410.0, 4.0, "U", 32)], zoom_only=True)
    elif name == "mixed":
        base.update(zooms=[Subband(8410.0, 4.0, "U", 32), Subband(8420.0, 4.0, "U", 32)])
    elif name == "onepol":
        base.update(zooms=[Subband(8410.0, 4.0, "U", 32)], zoom_pols=("L",))
    elif name == "lsb":
        base.update(subbands=_SBL, zooms=[Subband(8422.0, 4.0, "L", 32)], zoom_only=True)
    elif name == "avg":
        base.update(zooms=[Subband(8410.0, 4.0, "U", 32), Subband(8420.0, 4.0, "U", 32)], chans_to_avg=4)
    else:
        raise ValueError(name)
    return jobs.spec_c1(**base)


CASES = ["shifted", "mixed", "onepol", "lsb", "avg"]


def _records(spec, offsets):
    """(offset, channels) of every cross and autocorrelation record of the
    Core result array, from the layout offsets (rl, bl, bw, ac, acw)."""
    from difx_b200.jobfiles import baseline_plan
    _, bl, _, ac, _ = offsets
    freqs = list(spec.subbands) + list(spec.zooms)
    nout = [f.nchan // spec.chans_to_avg for f in freqs]
    plan = baseline_plan(spec)
    nbl = len(plan)
    out = []
    used = set()
    for j, (_, _, fl) in enumerate(plan):
        for f, pairs in fl:
            used.add(f)
    for f in range(len(freqs)):
        for j, (_, _, fl) in enumerate(plan):
            o = bl[f * nbl + j]
            if o < 0:
                continue
            npp = [len(p) for g, p in fl if g == f][0]
            out += [(o + p * nout[f], nout[f]) for p in range(npp)]
    maxprod = max(len(p) for _, _, fl in plan for _, p in fl)
    bpa = 2 if maxprod > 2 else 1
    nsb = len(spec.subbands)
    for s in range(spec.nstations):
        bands = [g for g in spec.station_sb(s) for _ in spec.pols]
        bands += [nsb + k for k, _ in spec.station_zooms(s) for _ in spec.zpols]
        rows = [nout[f] for f in bands if f in used]
        o = ac[s]
        for _ in range(bpa):
            for n in rows:
                out.append((o, n))
                o += n
    return out


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_zoom_layout_matches_reference(name):
    from difx_b200.gxcorr import Correlator
    from difx_b200.jobfiles import write_job
    import os
    spec = _case(name)
    paths = write_job(spec, os.path.join(jobs._TMP, "zoomlayout_" + name))
    nf = len(spec.subbands) + len(spec.zooms)
    nbl = spec.nstations * (spec.nstations - 1) // 2
    c = Correlator.from_input(paths["input"], device=-1)
    try:
        g = c.offsets()
    finally:
        c.close()
    with pyoracle.Reference(paths["input"]) as ref:
        r = ref.layout(nf, nbl, spec.nstations)
    assert g[0] == r[0]
    for a, b in zip(g[1:], r[1:]):
        np.testing.assert_array_equal(a, b)


@needs_ref
def test_zoom_descriptor_matches_input():
    """The descriptor built from the job spec and the one read from its .input
    give the same layout."""
    from difx_b200 import capi
    from difx_b200.gxcorr import Correlator
    from difx_b200.jobfiles import write_job
    import os
    for name in CASES:
        spec = _case(name)
        paths = write_job(spec, os.path.join(jobs._TMP, "zoomdesc_" + name))
        a = Correlator.from_input(paths["input"], device=-1)
        b = Correlator.from_desc(capi.job_desc_from_spec(spec), device=-1)
        try:
            x, y = a.offsets(), b.offsets()
            assert x[0] == y[0]
            for u, v in zip(x[1:], y[1:]):
                np.testing.assert_array_equal(u, v)
        finally:
            a.close()
            b.close()


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_gpu_zoom_matches_reference(name):
    from difx_b200 import gxcorr as gx
    spec = _case(name)
    prep = jobs.prepare(spec, [100_000_000])
    ref = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    for xs in (0, 2):   # the FP32 form, and the split-FP16 tensor-core form for the recorded freqs
        c = gx.Correlator.from_input(prep.paths["input"], xstep=xs)
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
        # the rest: baseline and autocorrelation weights
        rw, gw = ref[mask].view(np.float32), g[mask].view(np.float32)
        wrel = float(np.max(np.abs(gw - rw) / np.maximum(np.abs(rw), 1e-30)))
        print(f"\n{name} xstep {xs}: {len(recs)} records, worst record {worst:.3g}, weights {wrel:.3g}")
        assert worst <= 1e-5, (name, xs, worst)
        assert wrel <= 1e-6, (name, xs, wrel)


@pytest.mark.gpu
@pytest.mark.skipif(not (pyoracle.reference_available() and pyoracle.shim_available()),
                    reason="reference or binding harness not built")
@pytest.mark.parametrize("name", ["shifted", "mixed"])
def test_gpucore_zoom_slot_matches_core_processdata(name):
    """The DiFX-side GpuCore passes the Configuration's zoom freqs and bands
    to the device: a zoom job's slot against Core::processdata."""
    from difx_b200.gxcorr import Correlator
    spec = _case(name)
    prep = jobs.prepare(spec, [100_000_000])
    ref = jobs.reference_for(prep.paths["input"])
    r = ref.process(prep.subs[0])
    b = pyoracle.Binding(prep.paths["input"])
    g = b.process(prep.subs[0], ref.result_length)
    b.close()
    c = Correlator.from_input(prep.paths["input"], device=-1)
    recs = _records(spec, c.offsets())
    c.close()
    worst = max(float(np.mean(np.abs(g[o:o + n] - r[o:o + n])) / np.mean(np.abs(r[o:o + n]))) for o, n in recs)
    print(f"\n{name}: GpuCore vs Core::processdata worst record {worst:.3g}")
    assert worst <= 1e-5, worst
