"""Sharded Fock builds across processes, one GPU each (torch.distributed).

Every rank holds the whole molecule; the canonical shell-quartet lists are
split into cost-balanced bra-pair ranges (``partition``), each rank builds
its partial J/K and two-electron gradient, and the engine calls back into a
reducer after each build to sum the partial matrices over the ranks (an
NCCL all-reduce over NVLink for CUDA buffers).  Diagonalisation /
purification and DIIS are replicated: identical inputs give identical
densities on every rank.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N


def partition(costs, parts: int):
    """Contiguous ranges of items with balanced total cost: bounds[0..parts]."""
    c = np.ascontiguousarray(np.asarray(costs, dtype=np.float64))
    b = (ctypes.c_int * (parts + 1))()
    N.check(N.lib().pyfacc_partition(len(c), c.ctypes.data_as(N.P_double), parts, b), "pyfacc_partition")
    return list(b)


class _CudaView:
    """A float64 device buffer seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def allreduce_sum(t, group=None):
    """In-place sum over the ranks of a torch tensor (NCCL for CUDA, gloo for CPU)."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


class TorchReducer:
    """Engine callback summing a device buffer over the process group."""

    def __init__(self, group=None):
        self.group = group
        self.cb = N.REDUCE_FN(self._reduce)

    def _reduce(self, ctx, ptr, count):
        import torch
        try:
            t = torch.as_tensor(_CudaView(int(ptr), int(count)), device="cuda")
            allreduce_sum(t, self.group)
            torch.cuda.current_stream().synchronize()
            return 0
        except Exception:  # reported to the engine as a failed reduction
            return 1


def attach_reducer(system, reducer) -> None:
    N.check(N.lib().pyfacc_system_set_reducer(system.handle, reducer.cb, None), "pyfacc_system_set_reducer")
    system._reducer = reducer  # keep the callback alive with the system


def sharded_system(mol, group=None, **options):
    """A System holding this rank's shard of the Fock builds, reduced over
    the default (or given) process group."""
    import torch.distributed as dist
    from . import System
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    s = System(mol, shard_rank=rank, shard_count=world, **options)
    attach_reducer(s, TorchReducer(group))
    return s
