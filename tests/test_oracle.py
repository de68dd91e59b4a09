"""The oracle pinned against the reference correlator itself (CPU).

The reference's own hot path (Configuration, Mk5Mode/Mode, Core::processdata,
mark5access) is compiled from its sources into oracle/_ref/libdifxref.so; the
C restatement in oracle/gxoracle.c must reproduce it bit for bit when the
reference runs one process thread (a deterministic accumulation order)."""
import os

import numpy as np
import pytest

from oracle import pyoracle
from tests import jobs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")


def _params(orc, spec, precision=pyoracle.FP32_REF):
    return orc.params(precision=precision, nthreads=1, num_buffered_ffts=spec.num_buffered_ffts,
                      xc_avg_ns=spec.uvshift_interval_ns, ac_avg_ns=spec.ac_avg_interval_ns)


CASES = {
    "c1": lambda: (jobs.spec_c1(), dict()),
    "c1_invalid_fill": lambda: (jobs.spec_c1(name="c1bad", seed=21), dict(invalid_frac=0.05, fill_frac=0.03)),
    "lsb": lambda: (jobs.spec_lsb(), dict()),
    "cplx8": lambda: (jobs.spec_cplx8(), dict()),
    "cplx8_invalid": lambda: (jobs.spec_cplx8(name="cx8bad", seed=23), dict(invalid_frac=0.08)),
    "c1_flush": lambda: (jobs.spec_c1(name="c1fl", uvshift_interval_ns=1_000_000, ac_avg_interval_ns=2_000_000,
                                      num_buffered_ffts=7), dict()),
}


@needs_ref
@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_bitexact_vs_reference(case, oracle_lib):
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    ref = jobs.reference_for(prep.paths["input"])
    assert ref.nthreads == 1
    r = ref.process(prep.subs[0])
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec))
    assert r.shape == o.shape
    np.testing.assert_array_equal(o.astype(np.complex64), r)


@needs_ref
@pytest.mark.parametrize("case", ["c1", "lsb", "cplx8", "c1_invalid_fill"])
def test_layout_matches_reference(case, oracle_lib):
    spec, _ = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000])
    ref = jobs.reference_for(prep.paths["input"])
    nbl = spec.nstations * (spec.nstations - 1) // 2
    rl, *lr = ref.layout(len(spec.subbands), nbl, spec.nstations)
    ol, *lo = oracle_lib.layout(prep.jd)
    assert rl == ol
    for a, b in zip(lr, lo):
        np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("case", ["c1", "lsb", "cplx8"])
def test_host_reader_matches_reference(case):
    """libgxcorr's own .input/.calc/.im reader and delay model (host-only
    handle) against Configuration and Model::calculateDelayInterpolator."""
    from difx_b200.gxcorr import Correlator
    from difx_b200.jobfiles import write_job
    spec, _ = CASES[case]()
    paths = write_job(spec, os.path.join(jobs._TMP, "reader_" + spec.name))
    ref = pyoracle.Reference(paths["input"])
    c = Correlator.from_input(paths["input"], device=-1)
    nbl = spec.nstations * (spec.nstations - 1) // 2
    rl, *lr = ref.layout(len(spec.subbands), nbl, spec.nstations)
    gl, *lg = c.offsets()
    assert rl == gl
    for a, b in zip(lr, lg):
        np.testing.assert_array_equal(a, b)
    assert c.info.blocks_per_send == ref.blocks_per_send
    for sec, ns in [(0, 0), (0, 100_000_000), (1, 300_000_000), (1, 996_000_000)]:
        for s in range(spec.nstations):
            np.testing.assert_array_equal(c.interpolator(s, 0, sec, ns), ref.interpolator(s, 0, sec, ns))
    c.close()


@needs_ref
@pytest.mark.parametrize("case", ["c1_invalid_fill", "cplx8_invalid"])
def test_unpack_bitexact_vs_reference(case, oracle_lib):
    """Mk5Mode::unpack (samples and weight) at many offsets across invalid and fill-pattern frames."""
    spec, kw = CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    ref = jobs.reference_for(prep.paths["input"])
    data = prep.subs[0].data[1]
    per = spec.fftchannels * (2 if spec.is_complex else 1)
    nframes = len(data) // spec.framebytes
    rng = np.random.default_rng(0)
    offs = list(rng.integers(0, (nframes - 2) * spec.frame_samples, 40))
    offs += [f * spec.frame_samples - 3 for f in range(1, min(nframes - 2, 12))]
    for off in offs:
        out, w, us, n = ref.unpack(1, data, int(off), spec.nbands, per)
        o, good = oracle_lib.unpack(prep.jd, 1, data, int(off), spec.fftchannels)
        assert us == off
        np.testing.assert_array_equal(o.reshape(-1), out[:spec.nbands * per].reshape(spec.nbands, per).reshape(-1))
        assert np.float32(good) / np.float32(spec.fftchannels) == np.float32(w)


@needs_ref
def test_mode_block_vs_oracle(oracle_lib):
    """Mode::process spectra of single blocks (after fractional-sample correction)."""
    spec, kw = CASES["c1_invalid_fill"]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    ref = jobs.reference_for(prep.paths["input"])
    p = _params(oracle_lib, spec)
    for st in range(spec.nstations):
        for blk in (0, 1, 17, 500, spec.blocks_per_send - 1):
            rs, rw = ref.mode_block(prep.subs[0], st, blk, spec.nbands, spec.nchan)
            os_, ow = oracle_lib.station_block(prep.jd, prep.sds[0], st, blk, p)
            assert np.float32(ow) == np.float32(rw)
            np.testing.assert_array_equal(os_.astype(np.complex64), rs)


def test_fp64_oracle_agrees_with_fp32(oracle_lib):
    """The FP64 precision oracle and the FP32 reference-order restatement agree
    to FP32 rounding (per-record mean |diff| / mean |value| < 1e-5)."""
    spec, _ = CASES["c1"]()
    prep = jobs.prepare(spec, [100_000_000])
    o32 = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec))
    o64 = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec, pyoracle.FP64))
    rl, bl, bw, ac, acw = oracle_lib.layout(prep.jd)
    offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    assert jobs.record_metric(o32, o64, offs, spec.nchan) < 1e-5


def test_correlation_is_detected(oracle_lib):
    """The synthetic signal model gives a coherent correlation (flat phase across
    channels) on every parallel-hand baseline after delay/fringe correction."""
    spec, _ = CASES["c1"]()
    prep = jobs.prepare(spec, [100_000_000], rho=0.2)
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec, pyoracle.FP64))
    rl, bl, bw, ac, acw = oracle_lib.layout(prep.jd)
    nbl = prep.jd.desc.nbaselines
    for j in range(nbl):
        v = o[bl[j]: bl[j] + spec.nchan]   # freq 0, RR
        coh = abs(v.mean()) / np.abs(v).mean()
        assert coh > 0.8, (j, coh)


FORMAT_CASES = {
    "real1": lambda: (jobs.spec_long("r1p", 1, "REAL", "U", 128, 57, subbands=[
        jobs.Subband(8400.0 + 16 * i, 16.0, "U", 128) for i in range(4)]), dict(invalid_frac=0.03)),
    "real4": lambda: (jobs.spec_long("r4p", 4, "REAL", "U", 512, 59), dict(invalid_frac=0.03)),
    "cplx4": lambda: (jobs.spec_long("cx4p", 4, "COMPLEX", "U", 512, 61), dict(invalid_frac=0.03)),
    "cplx2": lambda: (jobs.spec_long("cx2p", 2, "COMPLEX", "U", 128, 63), dict(invalid_frac=0.03)),
}


@needs_ref
@pytest.mark.parametrize("case", sorted(FORMAT_CASES))
def test_oracle_bitexact_other_bit_depths(case, oracle_lib):
    """1-bit and 4-bit real, 2- and 4-bit complex VDIF: the oracle's Core
    result array equals the reference's bit for bit."""
    spec, kw = FORMAT_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    r = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec))
    assert r.shape == o.shape
    np.testing.assert_array_equal(o.astype(np.complex64), r)


FEATURE_CASES = {
    # FRINGE ROTN ORDER 2 (quadratic rotator as repeated FP32 stride products)
    "quad_real": lambda: (jobs.spec_c1(name="oq", seed=94, fringe_rot_order=2, subbands=[
        jobs.Subband(8400.25 + 16 * i, 16.0, "U", 128) for i in range(4)]), dict(invalid_frac=0.02)),
    "quad_cplx": lambda: (jobs.spec_cplx8(name="oqc", seed=96, fringe_rot_order=2), dict(invalid_frac=0.02)),
    # real time samples narrower than a byte (sample granularity 2 and 4)
    "real2_2band": lambda: (jobs.spec_c1(name="og22", seed=111, subbands=[jobs.Subband(8400.0, 16.0, "U", 128)]),
                            dict(invalid_frac=0.03)),
    "real1_2band": lambda: (jobs.spec_c1(name="og12", seed=112, nbits=1,
                                         subbands=[jobs.Subband(8400.0, 16.0, "U", 128)]), dict(invalid_frac=0.03)),
    # INTERLACEDVDIF: EDV4 per-band blanking and per-band weights
    "mux_real2": lambda: (jobs.spec_c1(name="omx2", seed=101, mux_threads=8, edv4_partial_frac=0.3),
                          dict(invalid_frac=0.02)),
    "mux_real8": lambda: (jobs.spec_c1(name="omx8", seed=102, nbits=8, mux_threads=8, edv4_partial_frac=0.3),
                          dict(invalid_frac=0.02)),
    "mux_cplx8": lambda: (jobs.spec_cplx8(name="omxc", seed=103, mux_threads=4, edv4_partial_frac=0.3),
                          dict(invalid_frac=0.02)),
}


@needs_ref
@pytest.mark.parametrize("case", sorted(FEATURE_CASES))
def test_oracle_bitexact_fringe_orders_and_granularity(case, oracle_lib):
    """Quadratic fringe rotation, sub-byte time samples and INTERLACEDVDIF
    with EDV4 masks: the oracle's Core result array equals the reference's
    bit for bit."""
    spec, kw = FEATURE_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    r = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec))
    assert r.shape == o.shape
    np.testing.assert_array_equal(o.astype(np.complex64), r)


POSTF_CASES = {
    "postf_usb": lambda: (jobs.spec_c1(name="opf", seed=91, fringe_rot_order=0, subbands=[
        jobs.Subband(8400.25 + 16 * i, 16.0, "U", 128) for i in range(4)]), dict(invalid_frac=0.02)),
    "postf_lsb": lambda: (jobs.spec_lsb(name="opfl", seed=92, fringe_rot_order=0), dict(invalid_frac=0.02)),
}


@needs_ref
@pytest.mark.parametrize("case", sorted(POSTF_CASES))
def test_oracle_post_f_rotation_vs_reference(case, oracle_lib):
    """Post-F fringe rotation: the reference transforms with a real-to-complex
    FFT (mode.cpp:1135-1159), the oracle with a complex FFT of the same real
    samples; records agree to 1e-6 (mean |difference| / mean |reference|)."""
    spec, kw = POSTF_CASES[case]()
    prep = jobs.prepare(spec, [100_000_000], **kw)
    r = jobs.reference_for(prep.paths["input"]).process(prep.subs[0])
    o = oracle_lib.subint(prep.jd, prep.sds[0], _params(oracle_lib, spec)).astype(np.complex64)
    assert r.shape == o.shape
    rl, bl, bw, ac, acw = oracle_lib.layout(prep.jd)
    offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    assert jobs.record_metric(o, r, offs, spec.nchan) < 1e-6


@pytest.mark.skipif(not pyoracle.shim_available(), reason="binding harness not built")
def test_binding_library_builds_a_gpucore_from_the_reference_configuration():
    """The DiFX-side binding (GpuCore over the reference's Configuration and
    Core) loads and opens a job on the CPU; its handle opens on first use."""
    spec = jobs.spec_c1(name="bind_cpu", seed=47)
    prep = jobs.prepare(spec, [100_000_000])
    b = pyoracle.Binding(prep.paths["input"])
    b.close()
