"""CUDA path (libgxcorr through its C ABI) against the oracle and the reference.

Tolerances: visibility and autocorrelation records within 1e-5 by the
per-record metric of utilities/vis2screen/diffDiFX.py:146-151
(mean |gpu - ref| / mean |ref|); weights within 1e-6 relative; per-block
data weights bit-exact."""
import numpy as np
import pytest

from oracle import pyoracle
from tests import jobs

pytestmark = pytest.mark.gpu

REC_TOL = 1e-5
W_TOL = 1e-6


def _params(orc, spec, precision=pyoracle.FP32_REF):
    return orc.params(precision=precision, nthreads=1, num_buffered_ffts=spec.num_buffered_ffts,
                      xc_avg_ns=spec.uvshift_interval_ns, ac_avg_ns=spec.ac_avg_interval_ns)


def _weight_slots(jd, bw, acw, spec):
    """Float indices of every weight in the result array."""
    d = jd.desc
    idx = []
    nbl = d.nbaselines
    for f in range(d.nfreqs):
        for j in range(nbl):
            o = bw[f * nbl + j]
            if o < 0:
                continue
            for p in range(d.baselines[j].npolprod[0]):
                idx.append(2 * o + p)
    nw = spec.nbands * (2 if spec.full_pol and len(spec.pols) > 1 else 1)
    for s in range(d.nstations):
        idx += [2 * acw[s] + k for k in range(nw)]
    return np.array(idx)


def _compare(gpu, ref, jd, spec, orc, layout=None):
    rl, bl, bw, ac, acw = layout if layout is not None else orc.layout(jd)
    offs = jobs.record_offsets(jd, bl, ac, spec)
    m = jobs.record_metric(gpu, ref, offs, spec.nchan // spec.chans_to_avg)
    wi = _weight_slots(jd, bw, acw, spec)
    gf = gpu.view(np.float32) if gpu.dtype == np.complex64 else gpu.astype(np.complex64).view(np.float32)
    rf = ref.astype(np.complex64).view(np.float32)
    wrel = np.max(np.abs(gf[wi] - rf[wi]) / np.maximum(np.abs(rf[wi]), 1e-30))
    return m, wrel


CASES = {
    "c1": lambda: (jobs.spec_c1(), dict()),
    "c1_invalid_fill": lambda: (jobs.spec_c1(name="c1bad", seed=21), dict(invalid_frac=0.05, fill_frac=0.03)),
    "lsb": lambda: (jobs.spec_lsb(), dict()),
    "cplx8": lambda: (jobs.spec_cplx8(), dict()),
    "cplx8_invalid": lambda: (jobs.spec_cplx8(name="cx8bad", seed=23), dict(invalid_frac=0.08)),
    "c2small": lambda: (jobs.spec_c2small(), dict(invalid_frac=0.01)),
    # long transforms (register-resident radix-16 F-step)
    "cplx8_4096": lambda: (jobs.spec_long("cx8l", 8, "COMPLEX", "U", 4096, 41), dict(invalid_frac=0.03)),
    "cplx8_4096_lsb": lambda: (jobs.spec_long("cx8ll", 8, "COMPLEX", "L", 4096, 43), dict(invalid_frac=0.03)),
    "real2_8192": lambda: (jobs.spec_long("r2x", 2, "REAL", "U", 4096, 47), dict(invalid_frac=0.03)),
    "real2_2048_lsb": lambda: (jobs.spec_long("r2m", 2, "REAL", "L", 1024, 53), dict(invalid_frac=0.03)),
    # other bit depths: 1-bit real (8 bands so that a time sample fills a byte), 4-bit real and complex
    "real1_256": lambda: (jobs.spec_long("r1p", 1, "REAL", "U", 128, 57, subbands=[
        jobs.Subband(8400.0 + 16 * i, 16.0, "U", 128) for i in range(4)]), dict(invalid_frac=0.03)),
    "real4_1024": lambda: (jobs.spec_long("r4p", 4, "REAL", "U", 512, 59), dict(invalid_frac=0.03)),
    "cplx4_512": lambda: (jobs.spec_long("cx4p", 4, "COMPLEX", "U", 512, 61), dict(invalid_frac=0.03)),
    "cplx2_128": lambda: (jobs.spec_long("cx2p", 2, "COMPLEX", "U", 128, 63), dict(invalid_frac=0.03)),
}


@pytest.fixture(scope="module")
def gx():
    from difx_b200 import gxcorr
    return gxcorr


@pytest.mark.parametrize("case", sorted(CASES))
def test_gpu_matches_oracle(case, gx, oracle_lib):
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    g = c.subint(prep.sds[0])
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec))
    m, wrel = _compare(g, o, prep.jd, spec, oracle_lib)
    assert m < REC_TOL, m
    assert wrel < W_TOL, wrel
    c.close()


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("case", ["c1", "cplx8_invalid"])
def test_gpu_matches_reference(case, gx, oracle_lib):
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    g = c.subint(prep.sds[0])
    r = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    m, wrel = _compare(g, r, prep.jd, spec, oracle_lib)
    assert m < REC_TOL, m
    assert wrel < W_TOL, wrel
    c.close()


@pytest.mark.parametrize("case", ["c1_invalid_fill", "cplx8_invalid", "lsb"])
def test_gpu_block_spectra_and_weights(case, gx, oracle_lib):
    """Station-stage output of single blocks (Mode::getFreqs after process())."""
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    c.subint(prep.sds[0])
    p = _params(oracle_lib, spec)
    for st in range(spec.nstations):
        for blk in (0, 3, 101, spec.blocks_per_send // 2, spec.blocks_per_send - 1):
            gs, gw = c.spectra(st, blk, spec.nbands)
            os_, ow = oracle_lib.station_block(prep.jd, prep.sds[0], st, blk, p)
            assert np.float32(gw) == np.float32(ow)          # data weight bit-exact
            scale = np.sqrt(np.mean(np.abs(os_) ** 2)) if ow > 0 else 1.0
            assert np.max(np.abs(gs - os_)) <= 1e-5 * max(scale, 1e-30) * np.sqrt(spec.fftchannels), (st, blk)
    c.close()


def test_gpu_bad_blocks_and_host_model(gx, oracle_lib):
    """Per-block valid flags (mode.cpp:656-669) and the handle's own delay model
    (gx_open_input, interpolators from its .im reader) on two subints."""
    spec = jobs.spec_c1(name="c1flags", seed=31)
    nb = spec.blocks_per_send
    bad = [np.array([0, 5, 6, 7, nb - 1]), np.array([]), np.arange(100, 160), np.array([999])]
    prep = jobs.prepare(spec, [100_000_000, 108_000_000], bad_blocks=bad)
    c = gx.Correlator.from_input(prep.paths["input"])
    c2 = gx.Correlator.from_desc(prep.jd)
    from difx_b200 import capi
    for i, si in enumerate(prep.subs):
        own = capi.subint_desc_host(si, None)          # handle computes the interpolators
        g_own = c.subint(own)
        g_exp = c2.subint(prep.sds[i])
        np.testing.assert_array_equal(g_own, g_exp)
        o = oracle_lib.subint(prep.jd, prep.sds[i], _params(oracle_lib, spec))
        m, wrel = _compare(g_own, o, prep.jd, spec, oracle_lib)
        assert m < REC_TOL and wrel < W_TOL, (m, wrel)
    c.close()
    c2.close()


def test_gpu_device_entry_point(gx, oracle_lib):
    """gx_subint_device on device-resident buffers equals the host entry point."""
    import torch
    from difx_b200 import capi
    spec = jobs.spec_c1(name="c1dev", seed=41)
    prep = jobs.prepare(spec, [100_000_000])
    c = gx.Correlator.from_desc(prep.jd)
    g_host = c.subint(prep.sds[0])
    si = prep.subs[0]
    dev = [torch.from_numpy(d).cuda() for d in si.data]
    torch.cuda.synchronize()
    sd = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in dev], [len(d) for d in si.data],
                         [x.ctypes.data for x in si.control], len(si.control[0]), prep.interps[0])
    out = torch.zeros(2 * c.result_length, dtype=torch.float32, device="cuda")
    c.subint_device(sd, out.data_ptr())
    c.synchronize()
    g_dev = out.cpu().numpy().view(np.complex64)
    np.testing.assert_array_equal(g_dev, g_host)
    c.close()


@pytest.mark.parametrize("case", ["c2small", "real2_2048_lsb"])
def test_gpu_fstep_kernel_choices_agree(case, gx, oracle_lib, monkeypatch):
    """Each F-step kernel a transform length can be routed to (radix-16
    register kernel, warp kernel for <= 1024 points, CTA-slot kernel above)
    matches the oracle on the same subint."""
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec))
    for r16_min in ("512", "1000000"):
        monkeypatch.setenv("GX_FSTEP_R16_MIN", r16_min)
        c = gx.Correlator.from_desc(prep.jd)
        g = c.subint(prep.sds[0])
        c.close()
        m, wrel = _compare(g, o, prep.jd, spec, oracle_lib)
        assert m < REC_TOL and wrel < W_TOL, (r16_min, m, wrel)


def test_gpu_async_pipeline_matches_sync(gx):
    """gx_subint_async / gx_subint_wait (two subints in flight, uploads on a
    copy stream) give the same result arrays as gx_subint, in order; a third
    subint in flight and a blocking call meanwhile are refused."""
    import torch
    from difx_b200 import capi
    spec = jobs.spec_c1(name="c1async", seed=43)
    starts = [100_000_000 + k * spec.subint_ns for k in range(4)]
    prep = jobs.prepare(spec, starts)
    c = gx.Correlator.from_desc(prep.jd)
    want = [c.subint(sd).copy() for sd in prep.sds]
    pinned = []
    sds = []
    for si, ip in zip(prep.subs, prep.interps):
        data = [torch.from_numpy(x).pin_memory() for x in si.data]
        pinned.append(data)
        sds.append(capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in data],
                                   [len(x) for x in si.data], [x.ctypes.data for x in si.control],
                                   len(si.control[0]), ip))
    outs = [torch.zeros(2 * c.result_length, dtype=torch.float32).pin_memory().numpy().view(np.complex64)
            for _ in range(4)]
    c.subint_async(sds[0], outs[0])
    c.subint_async(sds[1], outs[1])
    with pytest.raises(gx.GxError) as ei:
        c.subint_async(sds[2], outs[2])
    assert ei.value.status == 8
    with pytest.raises(gx.GxError) as ei:
        c.subint(prep.sds[0])
    assert ei.value.status == 8
    np.testing.assert_array_equal(c.wait(), want[0])
    c.subint_async(sds[2], outs[2])
    np.testing.assert_array_equal(c.wait(), want[1])
    c.subint_async(sds[3], outs[3])
    np.testing.assert_array_equal(c.wait(), want[2])
    np.testing.assert_array_equal(c.wait(), want[3])
    with pytest.raises(gx.GxError) as ei:
        c.wait()
    assert ei.value.status == 8
    np.testing.assert_array_equal(c.subint(prep.sds[1]), want[1])   # blocking calls work again
    c.close()


ORDER_CASES = {
    # fractional-MHz LOs exercise the integer-delay term of the post-F phase
    "c1_postf": lambda: (jobs.spec_c1(name="c1pf", seed=91, fringe_rot_order=0, subbands=[
        jobs.Subband(8400.25 + 16 * i, 16.0, "U", 128) for i in range(4)]), dict(invalid_frac=0.02)),
    "lsb_postf": lambda: (jobs.spec_lsb(name="lsbpf", seed=92, fringe_rot_order=0), dict(invalid_frac=0.02)),
    "long_postf": lambda: (jobs.spec_long("r2pf", 2, "REAL", "U", 1024, 93, fringe_rot_order=0),
                           dict(invalid_frac=0.02)),
    # FRINGE ROTN ORDER 2 (quadratic, pre-F)
    "c1_quad": lambda: (jobs.spec_c1(name="c1q", seed=94, fringe_rot_order=2, subbands=[
        jobs.Subband(8400.25 + 16 * i, 16.0, "U", 128) for i in range(4)]), dict(invalid_frac=0.02)),
    "lsb_quad": lambda: (jobs.spec_lsb(name="lsbq", seed=95, fringe_rot_order=2), dict(invalid_frac=0.02)),
    "cplx8_quad": lambda: (jobs.spec_cplx8(name="cx8q", seed=96, fringe_rot_order=2), dict(invalid_frac=0.02)),
    "cplx8_4096_quad": lambda: (jobs.spec_long("cx8lq", 8, "COMPLEX", "U", 4096, 97, fringe_rot_order=2),
                                dict(invalid_frac=0.02)),
}


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("case", sorted(ORDER_CASES))
def test_gpu_fringe_rotation_orders_match_reference(case, gx, oracle_lib):
    """FRINGE ROTN ORDER 0 (post-F): no rotation before the FFT, the fringe
    phase at the block centre added to the fractional-sample rotator's first
    stride (mode.cpp:778-780, 1038-1049, 1131-1159).  ORDER 2 (quadratic):
    delay, slope and curvature at the block start (800-825), rotator
    sub[k] quad[k]^j step[j] with the powers as repeated FP32 products
    (956-1005).  Against the compiled reference reading the same .input, two
    subints."""
    spec, kw = ORDER_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000, 108_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    for i, sd in enumerate(prep.sds):
        g = c.subint(sd)
        r = jobs.reference_for(prep.paths["input"]).process(prep.subs[i])
        assert g.shape == r.shape
        m, wrel = _compare(g, r, prep.jd, spec, oracle_lib, layout=c.offsets())
        assert m < REC_TOL and wrel < W_TOL, (m, wrel)
    c.close()


MUX_CASES = {
    "real2_mux": lambda: (jobs.spec_c1(name="c1mx", seed=101, mux_threads=8, edv4_partial_frac=0.3),
                          dict(invalid_frac=0.02)),
    # 8-bit: a blanked sample whose code decodes to 0.0 does not count as invalid
    "real8_mux": lambda: (jobs.spec_c1(name="r8mx", seed=102, nbits=8, mux_threads=8, edv4_partial_frac=0.3),
                          dict(invalid_frac=0.02)),
    # complex: the blanker's header geometry spans two data frames per header frame
    "cplx8_mux": lambda: (jobs.spec_cplx8(name="cx8mx", seed=103, mux_threads=4, edv4_partial_frac=0.3),
                          dict(invalid_frac=0.02)),
    "lsb_mux": lambda: (jobs.spec_lsb(name="lsbmx", seed=104, mux_threads=4, edv4_partial_frac=0.3),
                        dict(invalid_frac=0.02)),
}


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("case", sorted(MUX_CASES))
def test_gpu_interlaced_vdif_matches_reference(case, gx, oracle_lib):
    """INTERLACEDVDIF: multiplexed frames whose EDV4 validity masks lack some
    threads; those bands' samples are blanked and every band gets its own
    weight (mk5mode.cpp:142-163, format_vdif.c:8486-8660), used for the
    baseline, autocorrelation and cross-pol weights (core.cpp:911-912,
    1039-1044; mode.cpp:1277-1284, 1342-1351).  Against the compiled
    reference reading the same .input, two subints."""
    spec, kw = MUX_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000, 108_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    for i, sd in enumerate(prep.sds):
        g = c.subint(sd)
        r = jobs.reference_for(prep.paths["input"]).process(prep.subs[i])
        assert g.shape == r.shape
        m, wrel = _compare(g, r, prep.jd, spec, oracle_lib, layout=c.offsets())
        assert m < REC_TOL and wrel < W_TOL, (m, wrel)
    c.close()


GRAN_CASES = {
    # time samples narrower than a byte (mark5access sample granularity 8 / bits)
    "real2_2band": lambda: (jobs.spec_c1(name="g_r2x2", seed=111, subbands=[jobs.Subband(8400.0, 16.0, "U", 128)]),
                            dict(invalid_frac=0.03)),
    "real1_2band": lambda: (jobs.spec_c1(name="g_r1x2", seed=112, nbits=1,
                                         subbands=[jobs.Subband(8400.0, 16.0, "U", 128)]), dict(invalid_frac=0.03)),
    "real2_1band": lambda: (jobs.spec_c1(name="g_r2x1", seed=113, pols=("R",),
                                         subbands=[jobs.Subband(8400.0, 16.0, "U", 128)]), dict(invalid_frac=0.03)),
    "real2_2band_long": lambda: (jobs.spec_long("g_r2l", 2, "REAL", "U", 1024, 115, pols=("R", "L"),
                                                subbands=[jobs.Subband(8400.0, 16.0, "U", 1024)]),
                                 dict(invalid_frac=0.03)),
}


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("case", sorted(GRAN_CASES))
def test_gpu_sub_byte_time_samples_match_reference(case, gx, oracle_lib):
    """Time samples of 1, 2 or 4 bits (several per byte): the unpack starts on
    a granularity boundary and the samples outside the FFT window are erased
    from the weight (mk5mode.cpp:100, 118-141); the range check uses bytes per
    block numerator / denominator (mode.cpp:131-143, 688).  Against the
    compiled reference reading the same .input, two subints."""
    spec, kw = GRAN_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000, 108_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    for i, sd in enumerate(prep.sds):
        g = c.subint(sd)
        r = jobs.reference_for(prep.paths["input"]).process(prep.subs[i])
        assert g.shape == r.shape
        m, wrel = _compare(g, r, prep.jd, spec, oracle_lib, layout=c.offsets())
        assert m < REC_TOL and wrel < W_TOL, (m, wrel)
    c.close()


AVG_CASES = {
    "c1_avg4": lambda: (jobs.spec_c1(name="c1avg", seed=61, chans_to_avg=4), dict(invalid_frac=0.03)),
    "cplx8_avg8": lambda: (jobs.spec_cplx8(name="cx8avg", seed=62, chans_to_avg=8), dict(invalid_frac=0.03)),
}


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("case", sorted(AVG_CASES))
def test_gpu_channel_averaging_matches_reference(case, gx, oracle_lib):
    """CHANS TO AVG (core.cpp:1819-1869, mode.cpp:1376-1401): the averaged
    Core result array against the compiled reference reading the same .input,
    and against the full-resolution oracle averaged here."""
    spec, kw = AVG_CASES[case]()
    L = spec.chans_to_avg
    prep = jobs.prepare(spec, [100_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    assert c.info.chans_to_average == L
    g = c.subint(prep.sds[0])
    r = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    assert g.shape == r.shape
    m, wrel = _compare(g, r, prep.jd, spec, oracle_lib, layout=c.offsets())
    assert m < REC_TOL and wrel < W_TOL, (m, wrel)
    # the oracle at full resolution, averaged over groups of L channels
    full_spec = jobs.JobSpec(**{**spec.__dict__, "chans_to_avg": 1})
    jd_full = capi_job_desc(full_spec)
    o = oracle_lib.subint(jd_full, prep.sds[0], _params(oracle_lib, full_spec))
    rl_f, bl_f, bw_f, ac_f, acw_f = oracle_lib.layout(jd_full)
    _, bl, bw, ac, acw = c.offsets()
    full_offs = jobs.record_offsets(jd_full, bl_f, ac_f, full_spec)
    out_offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    n = spec.nchan // L
    worst = 0.0
    for fo, oo in zip(full_offs, out_offs):
        want = o[fo:fo + spec.nchan].reshape(n, L).mean(axis=1)
        got = g[oo:oo + n]
        den = np.mean(np.abs(want))
        if den > 0:
            worst = max(worst, float(np.mean(np.abs(got - want)) / den))
    assert worst < REC_TOL, worst
    c.close()


def capi_job_desc(spec):
    from difx_b200 import capi
    return capi.job_desc_from_spec(spec)


PCAL_CASES = {
    "c1_pcal": lambda: (jobs.spec_c1(name="c1pc", seed=81, pcal_interval_mhz=1), dict(invalid_frac=0.03)),
    "lsb_pcal": lambda: (jobs.spec_lsb(name="lsbpc", seed=82, pcal_interval_mhz=1), dict(invalid_frac=0.03)),
    "cplx8_pcal": lambda: (jobs.spec_cplx8(name="cx8pc", seed=83, pcal_interval_mhz=1), dict(invalid_frac=0.03)),
    # 8 complex 8-bit bands: 16-byte time samples (the C3 sample format)
    "cplx8_8band_pcal": lambda: (jobs.spec_cplx8(name="cx8pc8", seed=84, pcal_interval_mhz=1,
                                                 subbands=[jobs.Subband(6000.0 + 16 * i, 16.0, "U", 256)
                                                           for i in range(4)]), dict(invalid_frac=0.03)),
    # 4-bit real and 2-bit complex: the decode width read at run time
    "real4_pcal": lambda: (jobs.spec_long("r4pc", 4, "REAL", "U", 512, 86, pcal_interval_mhz=1),
                           dict(invalid_frac=0.03)),
    "cplx2_pcal": lambda: (jobs.spec_long("cx2pc", 2, "COMPLEX", "U", 128, 87, pcal_interval_mhz=1),
                           dict(invalid_frac=0.03)),
    # the C3 sample format (8 complex 8-bit bands, 16-byte time samples) with
    # 4096-point transforms: the station-block F-step forms the bin sums
    # (16 bins divide its 256 threads per transform); real4_pcal takes that
    # path with four transform groups per CTA (32 bins, 64 threads)
    "cplx8_4096_pcal": lambda: (jobs.spec_long("cx8pcl", 8, "COMPLEX", "U", 4096, 91, pcal_interval_mhz=1,
                                               subbands=[jobs.Subband(6000.0 + 16 * i, 16.0, "U", 4096)
                                                         for i in range(4)]), dict(invalid_frac=0.03)),
    # multiplexed frames with EDV4 masks: phase-cal of the blanked samples
    "mux_pcal": lambda: (jobs.spec_c1(name="c1mxpc", seed=105, pcal_interval_mhz=1, mux_threads=8,
                                      edv4_partial_frac=0.3), dict(invalid_frac=0.02)),
    # 16 2-bit real bands: 32-bit time samples
    "real2_16band_pcal": lambda: (jobs.spec_c1(name="c1pc16", seed=85, nstations=3, pcal_interval_mhz=1,
                                               subbands=[jobs.Subband(8400.0 + 16 * i, 16.0, "U", 128)
                                                         for i in range(8)]), dict(invalid_frac=0.03)),
    # 3 MHz tones: the subbands' first-tone offsets (1, 2 and 3 MHz) make the
    # reference pick the implicit-shift extractor for some bands and the
    # shifting one (the samples mixed down by the offset, pcal.cpp:583-1025)
    # for others: real USB, real LSB, complex
    "c1_pcal3": lambda: (jobs.spec_c1(name="c1pc3", seed=88, pcal_interval_mhz=3), dict(invalid_frac=0.03)),
    "lsb_pcal3": lambda: (jobs.spec_lsb(name="lsbpc3", seed=89, pcal_interval_mhz=3), dict(invalid_frac=0.03)),
    "cplx8_pcal3": lambda: (jobs.spec_cplx8(name="cx8pc3", seed=90, pcal_interval_mhz=3), dict(invalid_frac=0.03)),
}
PCAL_TOL = 1e-4   # FP32 bin sums (tens of thousands of samples per bin) formed in another order


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("case", sorted(PCAL_CASES))
def test_gpu_phase_cal_matches_reference(case, gx, oracle_lib):
    """Phase-cal tones (PHASE CAL INT 1 or 3 MHz; the reference's
    implicit-shift and shifting extractors, pcal.cpp:583-1600, called from
    mode.cpp:759-774 and copied by core.cpp:1131-1164) in the Core result
    array, against the compiled reference reading the same .input; the rest
    of the array as usual."""
    spec, kw = PCAL_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000, 108_000_000], **kw)
    c = gx.Correlator.from_desc(prep.jd)
    off, nt = c.pcal_layout()
    for i, sd in enumerate(prep.sds):
        g = c.subint(sd)
        r = jobs.reference_for(prep.paths["input"]).process(prep.subs[i])
        assert g.shape == r.shape
        m, wrel = _compare(g, r, prep.jd, spec, oracle_lib, layout=c.offsets())
        assert m < REC_TOL and wrel < W_TOL, (m, wrel)
        worst, nbands = 0.0, 0
        for s in range(spec.nstations):
            for b in range(spec.nbands):
                o, n = int(off[s, b]), int(nt[s, b])
                assert o >= 0 and n > 0
                ga, ra = g[o:o + n], r[o:o + n]
                den = np.mean(np.abs(ra))
                if den > 0:
                    worst = max(worst, float(np.mean(np.abs(ga - ra)) / den))
                    nbands += 1
                else:
                    assert np.all(ga == 0)
        assert nbands > 0 and worst < PCAL_TOL, (i, worst)
    c.close()
