"""Station data rings on the device against the reference's VDIF DataStream
and Core, end to end: raw VDIF of every station is multiplexed into the
device ring segment by segment (gx_ring_read) over the same windows the
reference's VDIFDataStream::dataRead hands its multiplexer
(vdiffile.cpp:668-860); then every subint of the span is correlated straight
from the rings (gx_ring_subint_device: the control words and send starts
computed by the device walk) and compared with the reference's
calculateControlParams (datastream.cpp:368-627, vdiffile.cpp:348-470) and,
for a selection of subints, with Core::processdata run on the reference
DataStream's own buffer at the send start it chose.

Checked per case: every segment's time and valid bytes, the ring's bytes
against the reference data buffer, every control word of a valid subint and
the send start, every record within 1e-5 (the diffDiFX metric) and the
weights within 1e-6.  The rings hold 8 segments; the reads continue into
segments 0 and 1 again, so that a send wraps past the buffer's end and reads
the copied overflow (DataStream::execute, datastream.cpp:296-305)."""
import os

import numpy as np
import pytest

from difx_b200 import synth
from oracle import pyoracle
from tests import jobs
from tests.test_phase_centres import _records
from tests.test_ring import INVALID, _spec, raw_stream, same_control

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not pyoracle.reference_available(),
                                                  reason="reference harness not built")]


def _compare(ref, got, recs):
    mask = np.ones(len(ref), bool)
    worst = 0.0
    for o, n in recs:
        r, q = ref[o:o + n], got[o:o + n]
        mask[o:o + n] = False
        m = np.mean(np.abs(r))
        if m == 0:
            assert np.all(q == 0)
            continue
        worst = max(worst, float(np.mean(np.abs(q - r)) / m))
    rw, gw = ref[mask].view(np.float32), got[mask].view(np.float32)
    wrel = float(np.max(np.abs(gw - rw) / np.maximum(np.abs(rw), 1e-30))) if rw.size else 0.0
    return worst, wrel


@pytest.mark.parametrize("name", ["vdif2bit", "mux4"])
def test_gpu_ring_matches_reference_datastream_and_core(name):
    import torch
    from difx_b200.gxcorr import Correlator, Ring
    from difx_b200.jobfiles import write_job
    spec = _spec(name)
    paths = write_job(spec, os.path.join(jobs._TMP, "gring_" + name))
    ref = pyoracle.Reference(paths["input"])
    c = Correlator.from_input(paths["input"], device=0)
    r = Ring(c)
    nst = spec.nstations
    g = r.geometry(0)
    perturb = dict(invalid_frac=0.03, drop_frac=0.01, dup_frac=0.01, swap_frac=0.02) if spec.mux_threads else None
    fb_thread = (spec.payload_bytes // max(1, spec.mux_threads) + 32) * max(1, spec.mux_threads)
    nfr = int(10.1 * g.readbytes / fb_thread)
    rds, draws = [], []
    pad = 3 * 2 * g.readbytes
    for s in range(nst):
        raw = raw_stream(spec, s, nfr, seed=5, perturb=perturb)
        rds.append(pyoracle.RefDataStream(ref, s, raw))
        buf = np.zeros(len(raw) + pad, np.uint8)
        buf[:len(raw)] = np.frombuffer(raw, np.uint8)
        draws.append(torch.from_numpy(buf).cuda())
    res = torch.zeros(2 * ref.result_length, dtype=torch.float32, device="cuda")
    recs = _records(spec, c.offsets())
    nextoff = [0] * nst

    def read(seg):
        for s in range(nst):
            out = rds[s].read(seg)
            assert out is not None, (s, seg)
            (off, size, dest, start), want = out
            assert off == nextoff[s] and dest == g.readbytes, (s, seg, off, nextoff[s])
            used = r.read(s, seg, 0, draws[s].data_ptr() + off, size)
            nextoff[s] = off + used
            got = r.segment(s, seg).astuple()[:5]
            assert got == tuple(want), (s, seg, got, want)
            mine = _dev_bytes(r.buffer_ptr(s) + seg * g.readbytes, want[3])
            theirs = rds[s].data(seg * g.readbytes, want[3])
            assert np.array_equal(mine, theirs), (s, seg, "ring bytes")

    def subint(k, correlate):
        t = k * spec.subint_ns
        sec, ns = t // 10**9, t % 10**9
        r.subint_device(0, sec, ns, c.scan_start_sec(0), res.data_ptr())
        cws, sps, exhausted = r.last_control(nst)
        assert not exhausted, k
        data, ctrl, wrapped = [], [], False
        for s in range(nst):
            cw, sp, _, nbytes = rds[s].control(0, sec, ns)
            assert same_control(cw, cws[s], sp, int(sps[s])), (k, s, cw[:6], cws[s][:6], sp, sps[s])
            data.append(rds[s].data(sp, nbytes))
            ctrl.append(cw)
            wrapped = wrapped or (cw[1] != INVALID and sp + nbytes > g.bufferbytes)
        if correlate or wrapped:
            si = synth.SubintInput(0, sec, ns, data, ctrl)
            want = ref.process(si)
            got = res.cpu().numpy().view(np.complex64)
            worst, wrel = _compare(want, got, recs)
            print(f"\n{name} subint {k}{' (wraps)' if wrapped else ''}: worst record {worst:.3g}, weights {wrel:.3g}")
            assert worst <= 1e-5 and wrel <= 1e-6, (k, worst, wrel)
        return wrapped

    for seg in range(8):
        read(seg)
    span = 8 * g.nsinc
    ka = int((span - 5 * spec.subint_ns) // spec.subint_ns)
    for k in range(ka):
        subint(k, correlate=k in (0, 1, ka // 2))
    read(0)
    read(1)
    kb = int((10 * g.nsinc - 3 * spec.subint_ns) // spec.subint_ns)
    nwrap = 0
    for k in range(ka, kb):
        nwrap += subint(k, correlate=k == kb - 1)
    assert nwrap > 0
    for x in rds:
        x.close()
    r.close()
    c.close()
    ref.close()


def _dev_bytes(ptr, n):
    """n bytes of device memory at ptr (a cudaMemcpy through the CUDA runtime)."""
    import ctypes as C
    import glob
    import torch
    torch.cuda.synchronize()
    libs = glob.glob("/usr/local/cuda/lib64/libcudart.so*") + \
        glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib", "libcudart.so*"))
    cudart = C.CDLL(libs[0])
    out = np.zeros(n, np.uint8)
    rc = cudart.cudaMemcpy(out.ctypes.data_as(C.c_void_p), C.c_void_p(ptr), C.c_size_t(n), 2)   # device to host
    assert rc == 0, rc
    return out
