"""Subint-parallel integration over ranks (difx_b200.dist) on the CPU: the
round-robin share of subints, and two gloo ranks whose partial integrations
are summed into rank 0's before it writes (fake correlator and writer with
integer-valued result arrays, so that the sum is exact)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from difx_b200 import dist as gxdist


def test_subints_of_rank_partition():
    for world in (1, 2, 3, 8):
        for nsub in (0, 1, 7, 16):
            got = sorted(i for r in range(world) for i in gxdist.subints_of_rank(nsub, r, world))
            assert got == list(range(nsub))
    with pytest.raises(ValueError):
        gxdist.subints_of_rank(4, 2, 2)


RL = 1000   # complex floats per result array


def _result(i):
    return (np.arange(2 * RL, dtype=np.float32) % 97 + 3 * i).astype(np.float32)


class FakeCorr:
    def __init__(self):
        self.done = []

    def subint_device(self, sub, ptr):
        self.done.append(sub)
        self.out[:] = torch.from_numpy(_result(sub))

    def synchronize(self):
        pass


class FakeVis:
    def __init__(self, corr):
        self.corr = corr
        self.buf = torch.zeros(2 * RL)
        self.nsub = 0
        self.written = None

    def add(self, ptr):
        self.buf += self.corr.out
        self.nsub += 1

    def buffer(self):
        return 0, 2 * RL, self.nsub

    def set_subints(self, n):
        self.nsub = n

    def clear(self):
        self.buf.zero_()
        self.nsub = 0

    def write(self, scan, sec, ns):
        self.written = (self.buf.clone(), self.nsub)
        self.clear()
        return 1


def _rank(rank, world, port, nsub, outdir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    corr = FakeCorr()
    res = torch.zeros(2 * RL)
    corr.out = res
    vis = FakeVis(corr)
    n = gxdist.correlate_integration(corr, vis, list(range(nsub)), res, 0, 0, 0, view=lambda v: v.buf)
    np.save(os.path.join(outdir, f"r{rank}.npy"),
            np.array([n, vis.nsub, len(corr.done)] + ([vis.written[1]] if vis.written else [-1])))
    if vis.written is not None:
        np.save(os.path.join(outdir, "sum.npy"), vis.written[0].numpy())
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("nsub", [5, 8])
def test_two_ranks_sum_into_rank0(tmp_path, nsub):
    mp.spawn(_rank, args=(2, _free_port(), nsub, str(tmp_path)), nprocs=2, join=True)
    r0 = np.load(tmp_path / "r0.npy")
    r1 = np.load(tmp_path / "r1.npy")
    assert r0[0] == 1 and r1[0] == 0            # rank 0 wrote, rank 1 did not
    assert r0[2] + r1[2] == nsub                  # every subint correlated once
    assert r0[2] == (nsub + 1) // 2
    assert r0[3] == nsub                          # the written sum holds every subint
    assert r1[1] == 0                             # rank 1's partial buffer was cleared
    want = sum(_result(i).astype(np.float64) for i in range(nsub))
    np.testing.assert_array_equal(np.load(tmp_path / "sum.npy"), want.astype(np.float32))
