"""Device VDIF multiplexer (gx_vdifmux_*) against the reference's vdifmux on
the same seeded multi-thread streams: every output header, the payload of
every frame the reference corner-turns, the statistics and the bytes
consumed, call after call as the VDIF DataStream chains them
(vdiffile.cpp:742-790: the next call starts where this one stopped, at the
next output frame number)."""
import numpy as np
import pytest

from oracle import pyoracle
from tests import vdif_streams as vs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not pyoracle.vmux_available(), reason="reference vdifmux not built")]

PERTURB = dict(invalid_frac=0.04, drop_frac=0.03, dup_frac=0.03, swap_frac=0.05, fill_frac=0.02, stray_frac=0.02)
DS_FLAGS = 0x02 | 0x40        # the DataStream's: respect granularity, propagate validity (EDV4)

CASES = {
    "4thr_2bit_datastream": dict(ids=[0, 1, 2, 3], nbits=2, flags=DS_FLAGS, pert=PERTURB),
    "4thr_2bit_strict": dict(ids=[0, 1, 2, 3], nbits=2, flags=0, pert=PERTURB),
    "4thr_2bit_validity": dict(ids=[0, 1, 2, 3], nbits=2, flags=0x04 | 0x40, pert=PERTURB),
    "3thr_8bit_permuted": dict(ids=[5, 2, 9], nbits=8, flags=DS_FLAGS, pert=PERTURB),
    "8thr_1bit": dict(ids=list(range(8)), nbits=1, flags=DS_FLAGS, pert=PERTURB),
    "2thr_8bit_complex": dict(ids=[0, 1], nbits=8, flags=DS_FLAGS | 0x20, pert=PERTURB, cplx=True),
    "16thr_2bit_clean": dict(ids=list(range(16)), nbits=2, flags=DS_FLAGS, pert={}),
    "4thr_4bit_gotoend": dict(ids=[0, 1, 2, 3], nbits=4, flags=0x01 | 0x40, pert=PERTURB),
    # a thread count and sample width outside the register-transpose kernels: the per-word kernel
    # (24 threads: the reference's presence mask is built with int shifts, vdifmux.c:742-750, so it
    # cannot describe thread 31 and above)
    "24thr_1bit": dict(ids=list(range(24)), nbits=1, flags=DS_FLAGS, pert=PERTURB),
    # several recorded bands per thread (setvdifmuxinputchannels, as the VDIF
    # DataStream sets it when bands outnumber threads): one thread of 8 bands
    # (a plain copy) and 2 threads of 2 bands (4-bit time samples per thread)
    "1thr_8ch_2bit": dict(ids=[0], nbits=2, flags=DS_FLAGS, pert=PERTURB, chans=8),
    "2thr_2ch_2bit": dict(ids=[0, 1], nbits=2, flags=DS_FLAGS, pert=PERTURB, chans=2),
}

FIELDS = ["valid_frames", "invalid_frames", "discarded_frames", "wrong_thread_frames", "skipped_bytes", "fill_bytes",
          "duplicate_frames", "bytes_processed", "good_output_frames", "partial_output_frames",
          "filler_output_frames", "calls", "src_bytes", "src_used", "dest_bytes", "dest_used", "output_frames",
          "start_frame"]


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("dest_frames", [70, 23])
def test_device_mux_matches_reference(case, dest_frames):
    import torch
    from difx_b200.gxcorr import VdifMux
    c = CASES[case]
    fb, fps, nsort, ngap = 1032, 1000, 16, 250
    ids, nbits, cplx, chans = c["ids"], c["nbits"], c.get("cplx", False), c.get("chans", 1)
    # enough frames that every perturbation occurs with few threads too
    src = vs.stream(ids, max(60, 240 // len(ids)), fb, fps, nbits, seed=11 + sorted(CASES).index(case), start_frame=7,
                    cplx=cplx, chans=chans, **c["pert"])
    m = VdifMux(fb, fps, nbits, ids, nsort=nsort, ngap=ngap, flags=c["flags"], channels_per_thread=chans)
    ofb = m.output_frame_bytes
    dest_bytes = ofb * dest_frames
    d_src = torch.frombuffer(bytearray(src), dtype=torch.uint8).cuda()
    d_dest = torch.zeros(dest_bytes, dtype=torch.uint8, device="cuda")
    window = len(src) // 2 // fb * fb            # each call sees half the stream, as a read buffer would
    idx, start, acc = 0, -1, None
    P = 1
    while P < len(ids):
        P *= 2
    B = nbits * (2 if cplx else 1) * chans
    pad_bits = P != len(ids)   # some corner turners leave the padding slots untouched (scratch stays there)
    for call in range(4):
        if idx >= len(src) - fb:
            break
        chunk = src[idx:idx + window]
        ref_out, ref = pyoracle.ref_vdifmux(chunk, dest_bytes, fb, fps, nbits, ids, nsort, ngap, c["flags"], start,
                                            channels_per_thread=chans)
        d_dest.zero_()
        st = m.run(d_src.data_ptr() + idx, len(chunk), d_dest.data_ptr(), dest_bytes, start)
        # the reference's statistics accumulate only within its call here
        mine = {f: getattr(st, f) for f in FIELDS}
        if acc is not None:
            for f in FIELDS[:12]:
                mine[f] -= acc[f]
        want = dict(zip(FIELDS, ref[:18]))
        want["calls"] = 1
        assert mine == want, (case, call, mine, want)
        assert st.returned_bytes == ref[20]
        acc = {f: getattr(st, f) for f in FIELDS}
        got = d_dest.cpu().numpy().tobytes()
        for f in range(st.output_frames):
            h, rh = got[f * ofb:f * ofb + 32], ref_out[f * ofb:f * ofb + 32]
            assert h == rh, (case, call, f, "header")
            if np.frombuffer(h[:4], "<u4")[0] >> 31:
                continue                         # filler frame: the reference leaves scratch in its payload
            a = np.frombuffer(got[f * ofb + 32:(f + 1) * ofb], np.uint8)
            b = np.frombuffer(ref_out[f * ofb + 32:(f + 1) * ofb], np.uint8)
            if pad_bits:                         # compare the threads' slots only
                keep = ((np.arange(a.size * 8) // B) % P) < len(ids)
                a = np.unpackbits(a, bitorder="little")[keep]
                b = np.unpackbits(b, bitorder="little")[keep]
            assert np.array_equal(a, b), (case, call, f, "payload")
        idx += st.src_used
        start = st.start_frame + st.output_frames
    # the streams exercised what they were built for
    assert acc["output_frames"] > 0 and acc["calls"] >= 2
    if c["pert"]:
        assert acc["duplicate_frames"] > 0 and acc["fill_bytes"] > 0 and acc["wrong_thread_frames"] > 0
        if c["flags"] & 0x40:
            # one thread: an output frame is whole or absent, never partial
            assert acc["partial_output_frames"] > 0 or len(ids) == 1
        else:
            assert acc["filler_output_frames"] > 0
    m.close()
