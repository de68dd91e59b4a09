"""The two places where gxcorr deliberately differs from the reference, each
asserted.

1. ``Model::calculateDelayInterpolator`` (mpifxcorr/src/model.cpp:282-286)
   divides the quadratic term by ``numincrements*numincrements`` formed in
   ``int``.  Above 46 340 FFT blocks per subint the product wraps, so the
   reference's quadratic coefficient is the true one times N^2 / int32(N^2)
   (for the 0.5 s subints of 2-bit 16 MHz data with 128 channels, N = 62 500:
   about -10 times the true value, a delay error of some picoseconds at the
   end of the subint).  gxcorr's host model forms N^2 in 64 bits: its linear
   and constant terms equal the reference's, its quadratic term is the
   reference's times int32(N^2) / N^2.  Below the limit the two agree bit for
   bit (tests/test_oracle.py).

2. ``Mode::process`` (mode.cpp:642-709) resets a block's data weight to 0 and
   sets it again only when it unpacks, which it does only when the block's
   nearest sample differs from the start of the window it unpacked last
   (Mk5Mode: ``unpacksamples`` equals the FFT length, mk5mode.cpp:36-41); a
   block left at weight 0 gets zero spectra (mode.cpp:743-753).  So a block
   whose nearest sample equals the previous block's (the delay grows by one
   whole FFT over one block) drops out of the reference's subint.  The window
   is reset at ``Mode::setData`` (mode.cpp:1541-1550), which each process
   thread calls for its own block range, so in the reference the outcome also
   depends on how many threads share the subint.  The device computes every
   block from its own samples and gives it the weight of its good samples.
"""
import os

import numpy as np
import pytest

from difx_b200 import capi
from difx_b200.gxcorr import Correlator
from difx_b200.jobfiles import write_job
from oracle import pyoracle
from tests import jobs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")


def _int32(x: int) -> int:
    return (x + 2 ** 31) % 2 ** 32 - 2 ** 31


@needs_ref
def test_numincrements_squared_in_64_bits():
    spec = jobs.spec_c1(name="c1_halfsec", subint_ns=500_000_000, int_time=1.0)
    n = spec.blocks_per_send
    assert n == 62_500 and n * n > 2 ** 31 - 1
    paths = write_job(spec, os.path.join(jobs._TMP, "div_numinc"))
    c = Correlator.from_input(paths["input"], device=-1)
    with pyoracle.Reference(paths["input"]) as ref:
        for s in range(spec.nstations):
            for sec, ns in ((0, 0), (1, 500_000_000)):
                g = c.interpolator(s, 0, sec, ns)
                r = ref.interpolator(s, 0, sec, ns)
                assert g[2] == r[2] and g[1] == r[1], (s, sec, g, r)
                assert g[0] != 0.0
                # the reference's quadratic term is divided by the wrapped product
                np.testing.assert_allclose(g[0], r[0] * _int32(n * n) / (n * n), rtol=1e-12)
                assert r[0] / g[0] < -9.0
    c.close()


def _same_sample_case():
    """C1-shaped job (2-bit real, 256-point transforms) whose station 0 delay
    grows by one FFT (8 us) per block, so every block has nearest sample 100."""
    spec = jobs.spec_c1(name="c1_jump", seed=41)
    prep = jobs.prepare(spec, [100_000_000])
    t_fft = spec.fftchannels / spec.samples_per_second * 1e6        # microseconds per block
    sampletime = 1e6 / spec.samples_per_second
    jump = np.array([0.0, t_fft, -0.5 * t_fft - 100 * sampletime])  # starttime = 100 samples for every block
    interp = np.array(prep.interps[0])
    interp[0] = jump
    si = prep.subs[0]
    return spec, prep, si, interp, jump


NBLK = 6


@needs_ref
def test_same_nearest_sample_block_weight():
    """The reference's Mode drops blocks 1.. (weight 0, zero spectra); the
    oracle's single-block form (the device's semantics: each block on its
    own) gives each the weight and the transform of its own samples, block 0
    equal to the reference's."""
    spec, prep, si, interp, jump = _same_sample_case()
    orc = pyoracle.Oracle()
    sd = capi.subint_desc_host(si, interp)
    p = orc.params(precision=pyoracle.FP32_REF, nthreads=1, num_buffered_ffts=spec.num_buffered_ffts,
                   xc_avg_ns=spec.uvshift_interval_ns, ac_avg_ns=spec.ac_avg_interval_ns)
    ref = jobs.reference_for(prep.paths["input"])
    ref.set_interpolator(0, jump)
    try:
        sp, dw, _, _ = ref.mode_blocks(si, 0, NBLK, spec.nbands, spec.nchan)
    finally:
        ref.set_interpolator(0, None)
    assert dw[0] > 0.0
    assert np.all(dw[1:] == 0.0), dw
    assert not np.any(sp[1:]), "the reference zeroes the spectra of a weight-0 block"
    for b in range(NBLK):
        os_, ow = orc.station_block(prep.jd, sd, 0, b, p)
        assert np.float32(ow) == np.float32(dw[0]), (b, ow)
        scale = np.sqrt(np.mean(np.abs(os_) ** 2))
        assert scale > 0
        if b == 0:
            assert np.max(np.abs(sp[0] - os_)) <= 1e-5 * scale * np.sqrt(spec.fftchannels)


@pytest.mark.gpu
def test_gpu_same_nearest_sample_block_weight(oracle_lib):
    """The device gives every block of the delay jump its own weight and the
    spectra of its own samples (the oracle's single-block form)."""
    spec, prep, si, interp, _ = _same_sample_case()
    sd = capi.subint_desc_host(si, interp)
    p = oracle_lib.params(precision=pyoracle.FP32_REF, nthreads=1, num_buffered_ffts=spec.num_buffered_ffts,
                          xc_avg_ns=spec.uvshift_interval_ns, ac_avg_ns=spec.ac_avg_interval_ns)
    c = Correlator.from_desc(prep.jd)
    c.subint(sd)
    for b in range(NBLK):
        gs, gw = c.spectra(0, b, spec.nbands)
        os_, ow = oracle_lib.station_block(prep.jd, sd, 0, b, p)
        assert gw > 0.0 and np.float32(gw) == np.float32(ow), (b, gw, ow)
        scale = np.sqrt(np.mean(np.abs(os_) ** 2))
        assert np.max(np.abs(gs - os_)) <= 1e-5 * scale * np.sqrt(spec.fftchannels), b
    c.close()
