"""gx_subint_device_noalloc: the subint entry point for callers that cannot
allocate device memory (host frameworks that own all device memory and only
pass buffers in; threads that must not call cudaMalloc/cudaFree, which can
wait for every stream of the device).  It keeps its scratch in one
library-wide device array, so these checks run last: two calls in a row
through the C ABI must each give exactly what the allocating entry point
(gx_subint_device on a handle) gives -- the same kernels over the same pass
length, so bit for bit -- without changing the device's free memory, and a
job too large for the array must be refused with a clear message."""
import ctypes as C

import numpy as np
import pytest

from tests import jobs

pytestmark = pytest.mark.gpu

REC_TOL = 1e-5
W_TOL = 1e-6


def _device_inputs(torch, si):
    dev = [torch.from_numpy(d).cuda() for d in si.data]
    torch.cuda.synchronize()
    return dev


def test_noalloc_matches_allocating_entry_point():
    import torch
    from difx_b200 import capi, gxcorr
    from oracle import pyoracle

    spec = jobs.spec_c1(name="c1noalloc", seed=77)
    prep = jobs.prepare(spec, [100_000_000], invalid_frac=0.02)
    si = prep.subs[0]
    dev = _device_inputs(torch, si)
    sd = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in dev], [len(d) for d in si.data],
                         [x.ctypes.data for x in si.control], len(si.control[0]), prep.interps[0])

    c = gxcorr.Correlator.from_desc(prep.jd)
    ref_out = torch.zeros(2 * c.result_length, dtype=torch.float32, device="cuda")
    c.subint_device(sd, ref_out.data_ptr())
    c.synchronize()
    expected = ref_out.cpu().numpy().view(np.complex64)
    c.close()

    orc = pyoracle.Oracle()
    rl, bl, bw, ac, acw = orc.layout(prep.jd)
    offs = jobs.record_offsets(prep.jd, bl, ac, spec)
    wslots = []
    nbl = prep.jd.desc.nbaselines
    for f in range(prep.jd.desc.nfreqs):
        for j in range(nbl):
            if bw[f * nbl + j] >= 0:
                wslots += [2 * bw[f * nbl + j] + p for p in range(4)]
    for s in range(spec.nstations):
        wslots += [2 * acw[s] + k for k in range(2 * spec.nbands)]
    wslots = np.array(wslots)

    stream = torch.cuda.Stream()
    outs = [torch.full((2 * rl,), float("nan"), dtype=torch.float32, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for call in range(2):
        out = outs[call]
        # the array is placed on the device with the library's module (at the
        # latest by the first call), so free memory is compared around the second
        free0 = torch.cuda.mem_get_info()[0] if call == 1 else None
        gxcorr.subint_device_noalloc(prep.jd, sd, out.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
        got = out.cpu().numpy().view(np.complex64)
        assert np.all(np.isfinite(got.view(np.float32))), call
        m = jobs.record_metric(got, expected, offs, spec.nchan)
        assert m < REC_TOL, (call, m)
        gf, ef = got.view(np.float32), expected.view(np.float32)
        wrel = np.max(np.abs(gf[wslots] - ef[wslots]) / np.maximum(np.abs(ef[wslots]), 1e-30))
        assert wrel < W_TOL, (call, wrel)
        assert np.array_equal(gf, ef), (call, "not bit-identical to gx_subint_device")


def test_noalloc_rejects_jobs_over_the_scratch_limit():
    from difx_b200 import capi, gxcorr
    from difx_b200.jobfiles import JobSpec, Subband

    # 64 stations x 4096 channels: the accumulators alone exceed the scratch array
    spec = JobSpec(name="huge", nstations=64, subbands=[Subband(6000.0 + 64 * i, 64.0, "U", 4096) for i in range(4)],
                   nbits=8, sampling="COMPLEX", subint_ns=64_000_000, execute_seconds=2)
    import torch
    jd = capi.job_desc_from_spec(spec)
    host_only = gxcorr.Correlator.from_desc(jd, device=-1)
    rl = host_only.result_length
    host_only.close()
    # real device buffers of the right size, so nothing could be written out of
    # bounds even if the size check were wrong; all-zero control words mark
    # every block invalid
    data = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(2 * rl, dtype=torch.float32, device="cuda")
    ctrl = np.zeros(3 + spec.blocks_per_send // 30 + 1, np.int32)
    sd = capi.SubintDesc(0, 0, 0, 0.0, [data.data_ptr()] * 64, [64] * 64, [ctrl.ctypes.data] * 64, len(ctrl),
                         np.zeros((64, 3)))
    torch.cuda.synchronize()
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.subint_device_noalloc(jd, sd, out.data_ptr(), 0)
    torch.cuda.synchronize()
    assert ei.value.status == 2
    assert "no-allocation limit" in str(ei.value)
