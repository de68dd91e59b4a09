"""Visibility output on the device (gx_vis_*) against the reference's Visibility.

* Same input, same bytes: the subint result arrays the GPU produced are
  integrated and written by gx_vis (device add, device normalisation, SWIN
  records) and by the reference's Visibility (visibility.cpp, through the
  harness); the two files must be byte-identical (headers, weights, (u, v, w)
  and every normalised channel).
* End to end: raw VDIF -> gx_subint_device -> gx_vis against raw VDIF ->
  the reference's Core -> the reference's Visibility, per record within
  1e-5 by the metric of utilities/vis2screen/diffDiFX.py:146-151, headers
  identical.
"""
import os

import numpy as np
import pytest

from difx_b200 import capi, swin
from oracle import pyoracle
from tests import jobs

pytestmark = pytest.mark.gpu

CASES = {
    "c1": lambda: jobs.spec_c1(name="gvis", seed=17, int_time=0.016),
    "lsb_3st": lambda: jobs.spec_lsb(name="gvisl", seed=19, int_time=0.008),
    "cplx8": lambda: jobs.spec_cplx8(name="gvisc", seed=23, int_time=0.008192),
    "c1_avg4": lambda: jobs.spec_c1(name="gvisa", seed=29, int_time=0.016, chans_to_avg=4),
    "c1_pcal": lambda: jobs.spec_c1(name="gvisp", seed=31, int_time=0.016, pcal_interval_mhz=1),
    "lsb_pcal": lambda: jobs.spec_lsb(name="gvislp", seed=37, int_time=0.008, pcal_interval_mhz=1),
    # a-priori calibration (visibility.cpp:463-484, 505-519, 607-616)
    "c1_tsys": lambda: jobs.spec_c1(name="gvist", seed=41, int_time=0.016, tsys=55.0),
    "cplx8_tsys": lambda: jobs.spec_cplx8(name="gvisct", seed=43, int_time=0.008192, tsys=70.0),
    # zoom freqs: records of their own channel counts, zoom autocorrelations
    # scaled by zoom / parent bandwidth (visibility.cpp:624-633)
    "zoom_shifted": lambda: _zoom("shifted"),
    "zoom_mixed": lambda: _zoom("mixed"),
    "zoom_avg": lambda: _zoom("avg"),
    # multiple phase centres: one file per centre, weights times the shift
    # decorrelation, scales divided by it (visibility.cpp:428-441, 554-557, 860-890)
    "pc3": lambda: _pc("pc3"),
    "pc2_avg": lambda: _pc("pc2_avg"),
    # pulsar binning: one file per bin, baseline weights over the bin's phase
    # width; scrunched: one file, weights over the summed weight x width
    # (visibility.cpp:402-415, 1056-1091, 1376-1393)
    "psr8": lambda: _psr("bins8"),
    "psr_scrunch": lambda: _psr("scrunch4"),
}


def _psr(name):
    from dataclasses import replace
    from tests.test_pulsar import _case
    return replace(_case(name), name="gvispsr_" + name, int_time=0.016)


def _pc(name):
    from dataclasses import replace
    from tests.test_phase_centres import _case
    return replace(_case(name), name="gvispc_" + name, int_time=0.016)


def _zoom(name):
    from dataclasses import replace
    from tests.test_zoom import _case
    return replace(_case(name), name="gvisz_" + name, int_time=0.016)


def _run_gpu(prep, outdir, xstep=capi.GX_XSTEP_FP32):
    import torch
    from difx_b200.gxcorr import Correlator, Visibility
    c = Correlator.from_input(prep.paths["input"], device=0, xstep=xstep)
    v = Visibility(c, outdir)
    dev = []
    for si, ip in zip(prep.subs, prep.interps):
        data = [torch.from_numpy(x).cuda() for x in si.data]
        res = torch.zeros(2 * c.result_length, dtype=torch.float32, device="cuda")
        sd = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in data], [len(x) for x in si.data],
                             [x.ctypes.data for x in si.control], len(si.control[0]), ip)
        c.subint_device(sd, res.data_ptr())
        c.synchronize()
        v.add(res.data_ptr())
        dev.append(res)
    s0 = prep.subs[0]
    n = v.write(s0.scan, s0.sec, s0.ns)
    host = [r.cpu().numpy().view(np.complex64) for r in dev]
    v.close()
    c.close()
    return n, host


def _file(d):
    fs = [f for f in os.listdir(d) if f.startswith("DIFX_")]
    assert len(fs) == 1, fs
    return os.path.join(d, fs[0])


@pytest.mark.parametrize("case", sorted(CASES))
def test_gx_vis_bytes_match_reference_visibility(case, tmp_path):
    spec = CASES[case]()
    nsub = int(round(spec.int_time * 1e9 / spec.subint_ns))
    starts = [100_000_000 + k * spec.subint_ns for k in range(nsub)]
    prep = jobs.prepare(spec, starts, invalid_frac=0.03)
    ours = str(tmp_path / "gx.difx")
    os.makedirs(ours)
    n, host = _run_gpu(prep, ours)
    assert n > 0
    ref = jobs.reference_for(prep.paths["input"])
    theirs = str(tmp_path / "ref.difx")
    s0 = prep.subs[0]
    ref.vis_write(host, s0.scan, s0.sec, s0.ns, theirs)
    fa = sorted(f for f in os.listdir(ours) if f.startswith("DIFX_"))
    fb = sorted(f for f in os.listdir(theirs) if f.startswith("DIFX_"))
    nbinfiles = spec.pulsar_bins if spec.pulsar_bins and not spec.pulsar_scrunch else 1
    assert fa == fb and len(fa) == max(1, spec.phase_centres) * nbinfiles, (fa, fb)
    freqs = list(spec.subbands) + list(spec.zooms)
    nrec = 0
    for f in fa:
        a = np.fromfile(os.path.join(ours, f), np.uint8)
        b = np.fromfile(os.path.join(theirs, f), np.uint8)
        assert a.size == b.size, (f, a.size, b.size)
        assert np.array_equal(a, b), f
        nrec += len(swin.read_records(os.path.join(ours, f), lambda q: freqs[q].nchan // spec.chans_to_avg))
    assert nrec == n


def test_gx_vis_end_to_end_matches_reference(tmp_path):
    spec = jobs.spec_c1(name="gvise", seed=29, int_time=0.016)
    prep = jobs.prepare(spec, [100_000_000, 108_000_000], invalid_frac=0.03)
    ours = str(tmp_path / "gx.difx")
    os.makedirs(ours)
    _run_gpu(prep, ours)
    ref = jobs.reference_for(prep.paths["input"])
    theirs = str(tmp_path / "ref.difx")
    ref.vis_write([ref.process(si) for si in prep.subs], 0, 0, 100_000_000, theirs)
    ra = swin.read_records(_file(ours), spec.nchan // spec.chans_to_avg)
    rb = swin.read_records(_file(theirs), spec.nchan // spec.chans_to_avg)
    assert len(ra) == len(rb)
    worst = 0.0
    for (ha, da), (hb, db) in zip(ra, rb):
        for f in ("baseline", "mjd", "seconds", "source", "freq", "pol", "uvw"):
            assert np.array_equal(ha[f], hb[f]), f
        assert abs(float(ha["weight"]) - float(hb["weight"])) <= 1e-6 * float(hb["weight"])
        worst = max(worst, float(np.mean(np.abs(da - db)) / np.mean(np.abs(db))))
    assert worst < 1e-5, worst


def test_integration_over_ranks_single_gpu(tmp_path):
    """difx_b200.dist.correlate_integration with one rank writes the same file
    as the sequential use of gx_vis, and the integration buffer seen through
    torch (gx_vis_buffer) holds the sum of the subints' result arrays."""
    import torch
    from difx_b200 import dist as gxdist
    from difx_b200.gxcorr import Correlator, Visibility
    spec = CASES["c1"]()
    nsub = int(round(spec.int_time * 1e9 / spec.subint_ns))
    starts = [100_000_000 + k * spec.subint_ns for k in range(nsub)]
    prep = jobs.prepare(spec, starts, invalid_frac=0.03)
    seq = str(tmp_path / "seq")
    os.makedirs(seq)
    _, host = _run_gpu(prep, seq)
    c = Correlator.from_input(prep.paths["input"], device=0)
    v = Visibility(c, str(tmp_path))
    keep, subs = [], []
    for si, ip in zip(prep.subs, prep.interps):
        data = [torch.from_numpy(x).cuda() for x in si.data]
        keep.append(data)
        subs.append(capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in data],
                                    [len(x) for x in si.data], [x.ctypes.data for x in si.control],
                                    len(si.control[0]), ip))
    res = torch.zeros(2 * c.result_length, dtype=torch.float32, device="cuda")
    # the buffer view: add two subints, compare with their sum
    for i in range(2):
        c.subint_device(subs[i], res.data_ptr())
        v.add(res.data_ptr())
    c.synchronize()
    buf = gxdist.integration_tensor(v)
    want = host[0].view(np.float32).astype(np.float64) + host[1].view(np.float32)
    np.testing.assert_allclose(buf.cpu().numpy(), want, rtol=1e-6, atol=1e-6)
    assert v.buffer()[2] == 2
    v.clear()
    assert v.buffer()[2] == 0 and float(buf.abs().max()) == 0.0
    outdir = str(tmp_path / "ranks")
    os.makedirs(outdir)
    v.close()
    v = Visibility(c, outdir)
    s0 = prep.subs[0]
    n = gxdist.correlate_integration(c, v, subs, res, s0.scan, s0.sec, s0.ns)
    assert n > 0
    assert np.array_equal(np.fromfile(_file(outdir), np.uint8), np.fromfile(_file(seq), np.uint8))
    v.close()
    c.close()


@pytest.mark.parametrize("case", ["c1_pcal", "lsb_pcal"])
def test_pcal_files_match_reference(case, tmp_path):
    """PCAL_<mjd>_<sec>_<station> lines (tones scaled as the band's
    autocorrelation, USB imaginary parts negated) equal the reference
    Visibility's for the same result arrays; the header lines come from
    gx_vis_pcal_headers as FxManager writes them once per job."""
    spec = CASES[case]()
    nsub = int(round(spec.int_time * 1e9 / spec.subint_ns))
    starts = [100_000_000 + k * spec.subint_ns for k in range(nsub)]
    prep = jobs.prepare(spec, starts, invalid_frac=0.03)
    ours = str(tmp_path / "gx.difx")
    os.makedirs(ours)
    n, host = _run_gpu(prep, ours)
    theirs = str(tmp_path / "ref.difx")
    s0 = prep.subs[0]
    jobs.reference_for(prep.paths["input"]).vis_write(host, s0.scan, s0.sec, s0.ns, theirs)
    pa = sorted(f for f in os.listdir(ours) if f.startswith("PCAL_"))
    pb = sorted(f for f in os.listdir(theirs) if f.startswith("PCAL_"))
    assert pa == pb and len(pa) == spec.nstations, (pa, pb)
    for f in pa:
        a = open(os.path.join(ours, f)).read()
        b = open(os.path.join(theirs, f)).read()
        assert a == b, f
        assert len(a.splitlines()) == 1 and len(a.split()) == 6 + 4 * spec.nbands * 16
    # the header lines
    from difx_b200.gxcorr import Correlator, Visibility
    c = Correlator.from_input(prep.paths["input"], device=0)
    hd = str(tmp_path / "hdr")
    os.makedirs(hd)
    v = Visibility(c, hd)
    v.pcal_headers()
    v.close()
    c.close()
    for f in os.listdir(hd):
        lines = open(os.path.join(hd, f)).read().splitlines()
        assert lines[0] == "# DiFX-derived pulse cal data" and lines[1] == "# File version = 1"
        assert lines[4] == "# Telescope name = " + f.split("_", 3)[3]
