"""The request loop on the GPU: requests of three different jobs (real 2-bit
with the FP32 X-step, complex 8-bit with the split-FP16 tensor-core X-step,
lower-sideband real) submitted together and run concurrently give the same
result arrays as each request run alone on its own handle -- bit for bit,
since every kernel is deterministic for a given handle configuration; with
device-resident inputs too."""
import numpy as np
import pytest

from difx_b200 import capi
from tests import jobs

pytestmark = pytest.mark.gpu


def _jobs():
    out = []
    for spec, xs in ((jobs.spec_c1(name="srv1", seed=41), capi.GX_XSTEP_FP32),
                     (jobs.spec_cplx8(name="srv2", seed=43), capi.GX_XSTEP_TC_FP16_HILO),
                     (jobs.spec_lsb(name="srv3", seed=47), capi.GX_XSTEP_FP32)):
        starts = [100_000_000 + k * spec.subint_ns for k in range(2)]
        out.append((spec, xs, jobs.prepare(spec, starts, invalid_frac=0.02)))
    return out


def _alone(gx, spec, xs, prep):
    c = gx.Correlator.from_desc(capi.job_desc_from_spec(spec, xstep=xs))
    res = [c.subint(sd).copy() for sd in prep.sds]
    c.close()
    return res


def test_results_same_alone_and_in_the_mix():
    from difx_b200 import gxcorr as gx
    J = _jobs()
    alone = [_alone(gx, *j) for j in J]
    corrs = [gx.Correlator.from_desc(capi.job_desc_from_spec(spec, xstep=xs)) for spec, xs, _ in J]
    budget = sum(c.device_bytes() for c in corrs) + (1 << 30)
    srv = gx.Server(slots=3, hbm_budget_bytes=budget)
    ids = [srv.attach(c) for c in corrs]
    outs, tickets = [], []
    for k in range(2):                      # interleave the jobs' requests
        for j, (spec, xs, prep) in enumerate(J):
            o = np.zeros(corrs[j].result_length, np.complex64)
            outs.append((j, k, o))
            tickets.append(srv.submit(ids[j], prep.sds[k], o.ctypes.data, keep=o))
    lat = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    for c in corrs:
        c.close()
    assert st.completed == 6 and all(x > 0 for x in lat)
    for j, k, o in outs:
        assert np.array_equal(o, alone[j][k]), (j, k)


def test_device_inputs_same_as_alone():
    import torch
    from difx_b200 import gxcorr as gx
    J = _jobs()
    alone = [_alone(gx, *j) for j in J]
    corrs = [gx.Correlator.from_desc(capi.job_desc_from_spec(spec, xstep=xs)) for spec, xs, _ in J]
    srv = gx.Server(slots=3, hbm_budget_bytes=sum(c.device_bytes() for c in corrs) + (8 << 30), device_inputs=True)
    ids = [srv.attach(c) for c in corrs]
    outs, tickets = [], []
    for k in range(2):
        for j, (spec, xs, prep) in enumerate(J):
            si, ip = prep.subs[k], prep.interps[k]
            dev = [torch.from_numpy(x).cuda() for x in si.data]
            sd = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in dev], [len(x) for x in si.data],
                                 [x.ctypes.data for x in si.control], len(si.control[0]), ip)
            o = np.zeros(corrs[j].result_length, np.complex64)
            outs.append((j, k, o))
            tickets.append(srv.submit(ids[j], sd, o.ctypes.data, keep=(o, dev)))
    for t in tickets:
        srv.wait(t)
    srv.close()
    for c in corrs:
        c.close()
    for j, k, o in outs:
        assert np.array_equal(o, alone[j][k]), (j, k)
