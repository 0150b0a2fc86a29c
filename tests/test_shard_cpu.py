"""Host side of the multi-GPU path, on CPU: the cost-balanced partition and the
all-reduce of per-rank partial results, with world_size-2 gloo process groups.

The partition is the library's own host function (no GPU needed); the partial
results come from a stand-in engine that returns each rank's share of known
full matrices, so the test checks the plumbing that ``quax_b200.integrals.sharded``
adds around the GPU kernels.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_covers_and_balances():
    from quax_b200.integrals.sharded import partition_costs

    rng = np.random.default_rng(3)
    # primitive-quartet costs of a class list, sorted largest first as the library sorts them
    cost = np.sort((rng.integers(1, 9, 5000) ** 2 * rng.integers(1, 9, 5000) ** 2).astype(float))[::-1]
    for nr in (1, 2, 3, 8):
        b = partition_costs(cost, nr)
        assert b[0] == 0 and b[-1] == cost.size and np.all(np.diff(b) >= 0)
        share = np.array([cost[b[r]:b[r + 1]].sum() for r in range(nr)])
        assert abs(share.sum() - cost.sum()) < 1e-6
        assert np.max(np.abs(share - cost.sum() / nr)) <= cost.max()  # within one item of even
    assert list(partition_costs([], 4)) == [0, 0, 0, 0, 0]
    b = partition_costs([5.0, 1.0], 4)  # more ranks than items: empty ranges allowed
    assert b[0] == 0 and b[-1] == 2 and np.all(np.diff(b) >= 0)
    with pytest.raises(ValueError):
        partition_costs([1.0, -1.0], 2)


class _PartialEngine:
    """Stand-in for a sharded EriEngine: rank r owns rows r::world of the full J/K
    and of the gradient, zero elsewhere, as the GPU shards own disjoint quartets."""

    def __init__(self, rank, world, J, K, g):
        mask = np.zeros(J.shape[0], dtype=bool)
        mask[rank::world] = True
        self.J = torch.from_numpy(np.where(mask[:, None], J, 0.0))
        self.K = torch.from_numpy(np.where(mask[:, None], K, 0.0))
        gm = np.zeros_like(g)
        gm[rank::world] = g[rank::world]
        self.g = torch.from_numpy(gm)

    def jk(self, D):
        return self.J.clone(), self.K.clone()

    def grad_adjoint(self, D, cj, ck):
        return self.g.clone()


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from quax_b200.integrals import sharded

        rng = np.random.default_rng(7)
        n = 9
        J = rng.normal(size=(n, n))
        K = rng.normal(size=(n, n))
        g = rng.normal(size=12)
        eng = _PartialEngine(rank, world, J, K, g)
        Jf, Kf = sharded.jk(eng, torch.zeros(n, n))
        gf = sharded.grad_adjoint(eng, torch.zeros(n, n))
        # every rank computes the same partition of a shared cost list
        cost = np.arange(1, 101, dtype=float)[::-1]
        b = torch.from_numpy(sharded.partition_costs(cost, world))
        allb = [torch.zeros_like(b) for _ in range(world)]
        dist.all_gather(allb, b)
        ok = (np.abs(Jf.numpy() - J).max() < 1e-14 and np.abs(Kf.numpy() - K).max() < 1e-14
              and np.abs(gf.numpy() - g).max() < 1e-14 and all(torch.equal(x, b) for x in allb))
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_partials_sum_to_full():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: True, 1: True}
