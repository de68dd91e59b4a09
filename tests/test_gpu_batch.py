"""Batches of uneven jobs (gx_batch_*): every job's results in a batch step
are bit-identical to the same subint run alone through gx_subint_device, in
each mode (per-job launches on one stream, branch streams, one replayed CUDA
graph), and a replayed graph picks up each step's new subint tables."""
import numpy as np
import pytest

from difx_b200 import capi
from difx_b200.jobfiles import Subband
from tests import jobs

pytestmark = pytest.mark.gpu


def _job_set():
    specs = [
        (jobs.spec_c1(name="bt_c1", seed=71), capi.GX_XSTEP_FP32, 0),
        (jobs.spec_cplx8(name="bt_cx8", seed=72), capi.GX_XSTEP_TC_FP16_HILO, 0),
        (jobs.spec_c2small(name="bt_c2", seed=73), capi.GX_XSTEP_FP32, 0),
        (jobs.spec_long("bt_r1", 1, "REAL", "U", 64, 74,
                        subbands=[Subband(8400.0 + 16 * i, 16.0, "U", 64) for i in range(4)]), capi.GX_XSTEP_FP32, 0),
        (jobs.spec_long("bt_cx8l", 8, "COMPLEX", "U", 2048, 75), capi.GX_XSTEP_AUTO, 0),
        (jobs.spec_c1(name="bt_c1chunk", seed=76), capi.GX_XSTEP_TC_FP16_HILO, 100),
    ]
    return specs


@pytest.fixture(scope="module")
def batch_jobs():
    import torch
    from difx_b200 import gxcorr
    out = []
    for spec, xstep, chunk in _job_set():
        t0 = 100_000_000
        prep = jobs.prepare(spec, [t0, t0 + spec.subint_ns])
        jd = capi.job_desc_from_spec(spec, xstep=xstep, block_chunk=chunk)
        subs = []
        for i, si in enumerate(prep.subs):
            dev = [torch.from_numpy(d).cuda() for d in si.data]
            sd = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in dev], [len(d) for d in si.data],
                                 [x.ctypes.data for x in si.control], len(si.control[0]), prep.interps[i])
            subs.append((sd, dev, si))
        out.append((spec, jd, subs))
    torch.cuda.synchronize()
    # each subint alone through gx_subint_device
    alone = []
    for spec, jd, subs in out:
        c = gxcorr.Correlator.from_desc(jd)
        res = []
        for sd, _, _ in subs:
            buf = torch.zeros(2 * c.result_length, dtype=torch.float32, device="cuda")
            c.subint_device(sd, buf.data_ptr())
            c.synchronize()
            res.append(buf.cpu().numpy().view(np.complex64).copy())
        c.close()
        alone.append(res)
    return out, alone


def test_auto_xstep_resolution(batch_jobs):
    from difx_b200 import gxcorr
    out, _ = batch_jobs
    spec, jd, _ = out[4]
    c = gxcorr.Correlator.from_desc(jd)
    assert c.info.xstep == capi.GX_XSTEP_FP32     # 6 inputs per freq: below the tensor-core break-even
    c.close()


@pytest.mark.parametrize("mode,nstreams", [("serial", 1), ("streams", 3), ("graph", 2), ("graph", 0)])
def test_batch_matches_alone(batch_jobs, mode, nstreams):
    import torch
    from difx_b200 import gxcorr
    out, alone = batch_jobs
    corrs = [gxcorr.Correlator.from_desc(jd) for _, jd, _ in out]
    bufs = [torch.full((2 * c.result_length,), float("nan"), dtype=torch.float32, device="cuda") for c in corrs]
    b = gxcorr.Batch(corrs, [x.data_ptr() for x in bufs], mode=mode, nstreams=nstreams)
    steps = 8 if nstreams == 0 else 4   # tuning: 1, 2, 4 branches twice each for six jobs
    for step in range(steps):
        k = step % 2                       # alternate the two subints of every job
        b.run([subs[k][0] for _, _, subs in out])
        ms = b.synchronize()
        assert ms > 0
        for j in range(len(out)):
            got = bufs[j].cpu().numpy().view(np.complex64)
            np.testing.assert_array_equal(got, alone[j][k], err_msg=f"{mode} step {step} job {j}")
    k, tuning, launches = b.info()
    assert not tuning
    assert k in ((1,) if mode == "serial" else (nstreams,) if nstreams else (1, 2, 4))
    assert launches >= 3 * len(out)
    b.close()
    for c in corrs:
        c.close()


def test_tile_tuner_keeps_results(batch_jobs):
    """gx_batch_tune_tiles times every launch-shape candidate per shape class
    and sets the fastest; the shapes change no bit of any job's results
    (every candidate of every job is checked here too)."""
    import torch
    from difx_b200 import gxcorr
    out, alone = batch_jobs
    corrs = [gxcorr.Correlator.from_desc(jd) for _, jd, _ in out]
    bufs = [torch.zeros((2 * c.result_length,), dtype=torch.float32, device="cuda") for c in corrs]
    for j, c in enumerate(corrs):
        for xv in (0, 1):
            for fi in (2, 4, 8):
                c.set_tiles(xv, fi)
                c.subint_device(out[j][2][0][0], bufs[j].data_ptr())
                c.synchronize()
                np.testing.assert_array_equal(bufs[j].cpu().numpy().view(np.complex64), alone[j][0],
                                              err_msg=f"job {j} tiles {xv}/{fi}")
        c.set_tiles(0, 0)
    b = gxcorr.Batch(corrs, [x.data_ptr() for x in bufs], mode="graph", nstreams=2)
    n = b.tune_tiles([subs[0][0] for _, _, subs in out], reps=1)
    assert 1 <= n <= len(out)
    b.run([subs[1][0] for _, _, subs in out])
    b.synchronize()
    for j in range(len(out)):
        np.testing.assert_array_equal(bufs[j].cpu().numpy().view(np.complex64), alone[j][1])
    b.close()
    for c in corrs:
        c.close()
