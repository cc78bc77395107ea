"""Batched fits over processes (gprx_b200.partition_by_cost and
sharded_batch_fit) on the CPU.

The ragged problem list is split by Σ n_i³ (longest processing time first);
each rank fits its shard and one all_gather_object at the end gives every rank
all results in the original order.  Two gloo ranks run here with a CPU stand-in
for the per-GPU GprBatch (the oracle's NLML and gradient at the starting θ, in
place of the device fit), so the partition, the shard hand-off and the gather
are checked without a GPU; the CUDA GprBatch itself is checked against the
oracle in test_batch_gpu.py.
"""

import math
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import gprx_b200 as gx
import oracle_lib as O

NODES = [[1, 2], [10, 0], [13, 0]]  # RbfKernel + PeriodicKernel


def test_partition_covers_every_problem_once_and_balances_cost():
    rs = np.random.RandomState(3)
    sizes = np.floor(np.exp(rs.uniform(math.log(32), math.log(1024), size=4096))).astype(int)
    cost = sizes.astype(float) ** 3
    for parts in (1, 2, 3, 8):
        shards = gx.partition_by_cost(sizes, parts)
        assert len(shards) == parts
        allidx = np.sort(np.concatenate(shards))
        assert np.array_equal(allidx, np.arange(sizes.size))
        loads = [cost[s].sum() for s in shards]
        # LPT bound: no shard exceeds another by more than the largest problem
        assert max(loads) - min(loads) <= cost.max()
        assert all(np.all(np.diff(s) > 0) for s in shards)
    # deterministic, and more shards than problems leaves some empty
    assert all(np.array_equal(a, b) for a, b in zip(gx.partition_by_cost(sizes, 8), gx.partition_by_cost(sizes, 8)))
    few = gx.partition_by_cost([10, 500, 20], 5)
    assert sorted(len(s) for s in few) == [0, 0, 1, 1, 1] and list(few[0]) == [1]
    with pytest.raises(gx.InvalidConfig):
        gx.partition_by_cost([1, 2], 0)


class OracleBatch:
    """CPU stand-in for one rank's GprBatch: 'fits' by evaluating the oracle
    at θ0 and returning θ0 (enough to check which problems a rank received
    and that the gathered results line up)."""

    def __init__(self, kernel, xs, ys, d, jitter, device):
        self.xs, self.ys, self.d = xs, ys, d

    def fit(self, params0, optimizer=None):
        k = len(self.xs)
        nl = np.zeros(k)
        gn = np.zeros(k)
        for i in range(k):
            n = np.asarray(self.ys[i]).size
            v, g, _, _ = O.exact_eval(NODES, params0[i], self.xs[i], n, self.d, self.ys[i])
            nl[i], gn[i] = v, np.linalg.norm(g)
        sizes = np.array([np.asarray(y).size for y in self.ys])
        return gx.BatchFit(params0.copy(), nl, sizes, sizes * 2, gn, np.ones(k, dtype=bool), np.zeros(k, np.int32))


def problems():
    rs = np.random.RandomState(11)
    sizes = [5, 40, 17, 90, 3, 64, 28, 51, 12, 75, 33]
    xs, ys = [], []
    for n in sizes:
        x = rs.uniform(0, 5, size=(n, 3))
        xs.append(x.T.reshape(-1).copy())
        ys.append(np.sin(x[:, 0]) + 0.1 * rs.standard_normal(n))
    p0 = np.tile([0.0, 0.0, math.log(15.0), math.log(0.1)], (len(sizes), 1))
    p0[:, 2] += 0.01 * np.arange(len(sizes))
    return sizes, xs, ys, p0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes, xs, ys, p0 = problems()
        spec = gx.RbfKernel(1.0) + gx.PeriodicKernel(1.0, 15.0)
        r = gx.sharded_batch_fit(spec, xs, ys, 3, p0, rank, world, dist.all_gather_object, batch_factory=OracleBatch)
        np.savez(out % rank, params=r.params, nlml=r.nlml, iters=r.iterations, status=r.status,
                 conv=r.converged)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_every_problem_in_order(tmp_path, world):
    out = str(tmp_path / "rank%d.npz")
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    sizes, xs, ys, p0 = problems()
    res = [np.load(out % k) for k in range(world)]
    for k in range(1, world):
        for key in ("params", "nlml", "iters", "status", "conv"):
            assert np.array_equal(res[0][key], res[k][key]), key
    r = res[0]
    assert np.array_equal(r["params"], p0)
    assert np.array_equal(r["iters"], np.array(sizes))
    assert np.all(r["status"] == 0) and np.all(r["conv"])
    for i, n in enumerate(sizes):
        v, _, _, _ = O.exact_eval(NODES, p0[i], xs[i], n, 3, ys[i])
        assert r["nlml"][i] == v
