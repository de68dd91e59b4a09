"""Batch API argument checks on the CPU (no GPU needed): host-only handles,
duplicate handles, bad modes and branch counts are rejected with status codes."""
import ctypes as C

import pytest

from difx_b200 import capi, gxcorr
from tests import jobs


def _open(handles, ptrs, mode=2, nstreams=0):
    n = len(handles)
    hs = (C.c_void_p * max(1, n))(*[h for h in handles])
    rs = (C.c_void_p * max(1, n))(*ptrs)
    b = C.c_void_p()
    return gxcorr.lib().gx_batch_open(hs, rs, n, mode, nstreams, C.byref(b))


def test_batch_open_rejects_bad_arguments():
    c = gxcorr.Correlator.from_desc(capi.job_desc_from_spec(jobs.spec_c1()), device=-1)
    h = c.h.value
    assert _open([h], [4096]) == 8                      # GX_ERR_STATE: host-only handle
    assert _open([], []) == 1                           # no jobs
    assert _open([h], [4096], mode=3) == 1              # unknown mode
    assert _open([h], [4096], nstreams=17) == 1         # more branches than the runner has
    assert _open([h], [0]) == 1                         # no result buffer
    assert _open([h, h], [4096, 8192]) == 1             # the same handle twice
    c.close()


def test_batch_null_calls():
    L = gxcorr.lib()
    assert L.gx_batch_run(None, None) == 1
    assert L.gx_batch_synchronize(None, None) == 1
    assert L.gx_batch_info(None, None, None, None) == 1
    assert L.gx_batch_close(None) == 1
    assert L.gx_batch_last_error(None) == b"null batch"
