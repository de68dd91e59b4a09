"""Visibility output (mpifxcorr/src/visibility.cpp), CPU side.

* The host model's (u, v, w) (Model::interpolateUVW, model.cpp:177-217) is
  bit-identical to the reference's on the job files.
* The reference's own Visibility, run through the harness, writes SWIN
  records that the reader in difx_b200.swin parses: one record per product
  with positive weight, 74-byte headers with the sync word, baseline numbers
  256 (t1 + 1) + t2 + 1, polarisation pairs and the integration centre time.
"""
import os

import numpy as np
import pytest

from difx_b200 import swin
from oracle import pyoracle
from tests import jobs

pytestmark = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")


def _job(**kw):
    spec = jobs.spec_c1(name="vis", seed=13, int_time=0.016, **kw)
    return spec, jobs.prepare(spec, [100_000_000, 108_000_000], invalid_frac=0.02)


def test_uvw_matches_reference_bit_exactly():
    from difx_b200.gxcorr import Correlator
    spec, prep = _job()
    ref = jobs.reference_for(prep.paths["input"])
    c = Correlator.from_input(prep.paths["input"], device=-1)
    for off in (0.008, 0.1, 0.4567, 1.9):
        for a in range(spec.nstations):
            for b in range(spec.nstations):
                g = c.uvw(0, off, a, b)
                r = ref.uvw(0, off, a, b)
                assert np.array_equal(g, r), (off, a, b, g, r)
    c.close()


def test_reference_visibility_records(tmp_path, oracle_lib):
    spec, prep = _job()
    ref = jobs.reference_for(prep.paths["input"])
    res = [ref.process(si) for si in prep.subs]
    out = str(tmp_path / "ref.difx")
    ref.vis_write(res, 0, 0, 100_000_000, out)
    files = os.listdir(out)
    assert len(files) == 1 and files[0].startswith("DIFX_") and files[0].endswith(".s0000.b0000")
    recs = swin.read_records(os.path.join(out, files[0]), spec.nchan)
    nbl = spec.nstations * (spec.nstations - 1) // 2
    ncross = nbl * len(spec.subbands) * 4
    nauto = spec.nstations * spec.nbands * 2
    assert len(recs) == ncross + nauto
    for h, data in recs[:ncross]:
        assert int(h["version"]) == 1 and int(h["config"]) == 0 and int(h["bin"]) == 0
        t1, t2 = int(h["baseline"]) // 256 - 1, int(h["baseline"]) % 256 - 1
        assert 0 <= t1 < t2 < spec.nstations
        assert h["pol"] in (b"RR", b"LL", b"RL", b"LR")
        assert 0 < float(h["weight"]) <= 1.0
        # the integration centre: start + int_time / 2
        assert abs(float(h["seconds"]) - (spec.start_seconds + 0.1 + spec.int_time / 2)) < 1e-9
        np.testing.assert_array_equal(h["uvw"], ref.uvw(0, 0.1 + spec.int_time / 2, t1, t2))
        assert np.all(np.isfinite(data))
    for h, data in recs[ncross:]:
        assert int(h["baseline"]) % 257 == 0 and np.all(h["uvw"] == 0)
