"""Multi-GPU use of the ERI path: one process per GPU, quartets sharded by cost.

Every screened unique quartet contributes independently to the dense and
derivative tensors, to J and K, and to the adjoint gradient, so each rank keeps a
cost-balanced contiguous range of every class's quartet list
(``qx_set_shard``) and the ranks' partial results are summed by one all-reduce
(NCCL over NVLink between GPUs; gloo for the host-side tests).  The reference
runs on one host and has no counterpart; the partials it would sum are the
per-quartet contributions of ``libint_interface.cc:2610-2690`` (gradient
tensor) and ``hartree_fock.py:26-28`` (J/K).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from . import _lib
from .engine import EriEngine


def partition_costs(cost, nranks: int) -> np.ndarray:
    """Bounds (nranks + 1) of the cost-balanced contiguous cut the library uses."""
    c = np.ascontiguousarray(np.asarray(cost, dtype=np.float64).reshape(-1))
    b = np.zeros(nranks + 1, dtype=np.int64)
    _lib.check(_lib.load().qx_partition_costs(C.c_void_p(c.ctypes.data), c.size, int(nranks),
                                              C.c_void_p(b.ctypes.data)), "qx_partition_costs")
    return b


def _rank_world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def shard(engine: EriEngine, group=None) -> EriEngine:
    """Restrict ``engine`` to this process's rank of ``group``."""
    rank, world = _rank_world(group)
    engine.set_shard(rank, world)
    return engine


def _sum(t: torch.Tensor, group) -> torch.Tensor:
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def grad_adjoint(engine: EriEngine, D: torch.Tensor, cj: float = 1.0, ck: float = -0.5, group=None) -> torch.Tensor:
    """Full adjoint gradient (3N) from a sharded engine: local part + all-reduce."""
    return _sum(engine.grad_adjoint(D, cj, ck), group)


def jk(engine: EriEngine, D: torch.Tensor, group=None):
    """Full J and K from a sharded engine, summed in one all-reduce."""
    J, K = engine.jk(D)
    n = J.shape[0]
    JK = _sum(torch.cat([J.reshape(-1), K.reshape(-1)]), group)
    return JK[: n * n].view(n, n), JK[n * n:].view(n, n)
