"""VDIF multiplexer, CPU side: the reference's vdifmux (compiled by
`make -C oracle vmux`) pinned against the corner-turn restatement of
tests/vdif_streams.py, and the device multiplexer's argument checks and
geometry (gx_vdifmux_open / _info) on a host-only handle."""
import numpy as np
import pytest

from difx_b200 import gxcorr
from oracle import pyoracle
from tests import vdif_streams as vs

needs_ref = pytest.mark.skipif(not pyoracle.vmux_available(), reason="reference vdifmux not built")


@needs_ref
@pytest.mark.parametrize("nthreads,nbits,cplx", [(4, 2, False), (2, 8, False), (8, 1, False), (3, 2, False),
                                                 (4, 8, True), (16, 2, False)])
def test_reference_corner_turn_pinned(nthreads, nbits, cplx):
    fb, fps = 1032, 1000
    ids = list(range(nthreads))
    src = vs.stream(ids, 40, fb, fps, nbits, seed=3, cplx=cplx)
    flags = 0x20 if cplx else 0
    P = 1
    while P < nthreads:
        P *= 2
    dest_bytes = ((fb - 32) * P + 32) * 45
    out, st = pyoracle.ref_vdifmux(src, dest_bytes, fb, fps, nbits, ids, 8, 100, flags)
    ofb = st[21]
    assert ofb == (fb - 32) * P + 32
    nout = st[16]
    assert nout >= 30 and st[8] == nout        # all complete
    frames = [src[i * fb:(i + 1) * fb] for i in range(len(src) // fb)]
    for f in range(nout):
        pay = [frames[f * nthreads + k][32:] for k in range(nthreads)]
        want = vs.corner_turn(pay, nbits, cplx)
        got = out[f * ofb + 32:(f + 1) * ofb]
        if nthreads == 3 and nbits == 8:
            continue                            # that corner turner leaves the padding byte untouched
        assert got == want, f


def test_open_arguments_and_geometry():
    m = gxcorr.VdifMux(8032, 4000, 2, [0, 1, 2, 3, 4], device=-1)
    assert m.output_channels == 8 and m.output_frame_bytes == 8000 * 8 + 32
    assert m.frame_granularity == 1
    m.close()
    m = gxcorr.VdifMux(1032, 25600, 8, [0, 1], device=-1)
    assert m.frame_granularity == 2           # 25600 frames/s: 2 frames make a whole number of ns
    m.close()
    m = gxcorr.VdifMux(1032, 3, 8, [0, 1], device=-1)
    assert m.frame_granularity == 3
    m.close()
    # several channels per thread: the header counts them, the payload stays P input payloads
    m = gxcorr.VdifMux(1032, 1000, 2, [0, 1], channels_per_thread=2, device=-1)
    assert m.output_channels == 4 and m.output_frame_bytes == 1000 * 2 + 32
    m.close()
    m = gxcorr.VdifMux(8032, 4000, 8, [0], channels_per_thread=8, device=-1)
    assert m.output_channels == 8 and m.output_frame_bytes == 8032
    m.close()
    with pytest.raises(gxcorr.GxError) as ei:   # 8 x 8-bit bands per thread do not pack into 32-bit words
        gxcorr.VdifMux(1032, 1000, 8, [0, 1], channels_per_thread=8, device=-1)
    assert ei.value.status == 2
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.VdifMux(1032, 1000, 2, [0, 1], flags=0x08, device=-1)   # legacy input headers
    assert ei.value.status == 2
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.VdifMux(1030, 1000, 2, [0, 1], device=-1)
    assert ei.value.status == 1
    m = gxcorr.VdifMux(1032, 1000, 2, [0, 1], device=-1)
    with pytest.raises(gxcorr.GxError) as ei:
        m.run(0, 0, 0, 0)
    assert ei.value.status in (1, 8)
    m.close()
