"""The sharded VFE protocol (gprx_b200.sharded_value_and_gradient) across two
gloo ranks on the CPU: each rank holds part of the points, the two exchange
buffers are summed by torch.distributed.all_reduce between the phases, and
every rank must end with the unsharded NLML and gradient (the oracle's,
|a − e| / max(|e|, 1) ≤ 1e-10).  The per-shard compute here is the numpy
mirror in sgpr_shard_np.py; the CUDA shard phases are checked against the
unsharded CUDA evaluation in test_sgpr_shard_gpu.py.
"""

import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import gprx_b200 as gx
import oracle_lib as O
from sgpr_shard_np import NumpyShard

TOL = 1e-10


def data():
    rs = np.random.RandomState(7)
    n, m, d = 500, 24, 3
    x = rs.uniform(0, 1, size=(n, d))
    y = np.sin(4 * x[:, 0]) + np.cos(3 * x[:, 1]) + 0.1 * rs.standard_normal(n)
    z = x[rs.choice(n, m, replace=False)]
    params = np.array([math.log(0.4), math.log(0.6), math.log(0.5), math.log(0.05)])
    return x, y, z, params


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, cuts, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, y, z, params = data()
        lo, hi = cuts[rank], cuts[rank + 1]
        shard = NumpyShard(x[lo:hi], y[lo:hi], z)
        calls = []

        def all_reduce(t):
            calls.append(t.numel())
            dist.all_reduce(t)

        nl, g = gx.sharded_value_and_gradient(shard, params, all_reduce, device="cpu")
        np.save(out % rank, np.concatenate([[nl], g, calls]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("cuts", [[0, 250, 500], [0, 1, 500], [0, 333, 500]], ids=["half", "one-point", "uneven"])
def test_two_gloo_ranks_get_the_unsharded_result(tmp_path, cuts):
    world = 2
    out = str(tmp_path / "rank%d.npy")
    mp.start_processes(_rank, args=(world, _free_port(), cuts, out), nprocs=world, join=True, start_method="spawn")
    x, y, z, params = data()
    n, d = x.shape
    m = z.shape[0]
    orc = O.Sgpr([[11, d]], params, x.T.reshape(-1).copy(), n, d, y, z.T.reshape(-1).copy(), m)
    r = [np.load(out % k) for k in range(world)]
    p = params.size
    for k in range(world):
        nl, g, calls = r[k][0], r[k][1:1 + p], r[k][1 + p:]
        assert O.rel_err(nl, orc.nlml()) <= TOL, (nl, orc.nlml())
        assert np.all(O.rel_err(g, orc.grad()) <= TOL), (g, orc.grad())
        # two exchanges, of the sizes the shard states
        assert list(calls) == [m * m + m + 3, m * m + d + 1]
    assert r[0][0] == r[1][0] and np.array_equal(r[0][1:1 + p], r[1][1:1 + p])
