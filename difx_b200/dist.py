"""Subint-parallel correlation over several GPUs, one process per GPU.

The reference's FxManager shares the subints of a job out over its Core
processes (fxmanager.cpp:331-336) and sums the result arrays they return into
its Visibility (Visibility::addData, visibility.cpp:192-205).  Here rank r of
N correlates subints r, r + N, r + 2N, ... of each integration on its own GPU
and adds them into its own device integration buffer (gx_vis_add).  At the end
of the integration one collective sums the partial buffers into rank 0's
(NCCL over NVLink between GPUs; gloo in the CPU tests) with the subint counts
beside them, and rank 0 normalises and writes the records (gx_vis_write) while
the other ranks clear theirs.  The data path has no other exchange: every
subint is correlated where its data is.
"""
from __future__ import annotations

from typing import Optional, Sequence

import torch
import torch.distributed as dist


def subints_of_rank(nsub: int, rank: int, world: int) -> list:
    """Subints of an integration correlated by `rank` (round robin, as the
    FxManager hands consecutive subints to successive Cores)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, nsub, world))


def rank_and_world(group=None):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def reduce_partial(buf: torch.Tensor, nsub: int, group=None, dst: int = 0) -> int:
    """Sums `buf` over the ranks into rank `dst`'s `buf` (in place) and returns
    the total number of subints the sum holds (on every rank)."""
    _, world = rank_and_world(group)
    if world == 1:
        return int(nsub)
    dist.reduce(buf, dst=dst, op=dist.ReduceOp.SUM, group=group)
    cnt = torch.tensor([int(nsub)], dtype=torch.int64, device=buf.device)
    dist.all_reduce(cnt, op=dist.ReduceOp.SUM, group=group)
    return int(cnt.item())


class DeviceFloats:
    """A device float32 array owned by the library, seen by torch through the
    CUDA array interface (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f4", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def integration_tensor(vis) -> torch.Tensor:
    """The Visibility's device integration buffer as a torch tensor (shared memory)."""
    ptr, n, _ = vis.buffer()
    return torch.as_tensor(DeviceFloats(ptr, n), device=torch.device("cuda", torch.cuda.current_device()))


def correlate_integration(corr, vis, subs: Sequence, dev_results: torch.Tensor, scan: int, sec: int, ns: int,
                          group=None, view=integration_tensor) -> int:
    """One integration of a job over the ranks of `group`.

    corr: this rank's Correlator; vis: its Visibility; subs[i]: the i-th subint
    of the integration (device data, every rank holds the descriptors; only
    this rank's subints are read); dev_results: a device array of
    2 x result_length floats.  Returns the records written (rank 0) or 0."""
    rank, world = rank_and_world(group)
    for i in subints_of_rank(len(subs), rank, world):
        corr.subint_device(subs[i], dev_results.data_ptr())
        vis.add(dev_results.data_ptr())
    corr.synchronize()                       # the handle's stream holds the adds
    if world > 1:
        _, _, mine = vis.buffer()
        buf = view(vis)
        total = reduce_partial(buf, mine, group)
        if buf.is_cuda:
            torch.cuda.synchronize()         # the sum is in place before the writer runs
        if rank != 0:
            vis.clear()
            return 0
        vis.set_subints(total)
    return vis.write(scan, sec, ns)
