"""The CUDA shard phases of the VFE evaluation (gprx_sgpr_shard_*): shards
of the points, each its own handle on the one GPU, with the exchange
buffers summed over the shards between the phases (what the all-reduce does
across processes), must give the unsharded NLML and gradient — against the
unsharded CUDA evaluation and the oracle at 1e-10 (FP64), and against the
FP64 evaluation at 1e-8 / 1e-6 in the mixed form — and leave each handle
predicting with the global posterior.
"""

import math

import numpy as np
import pytest
import torch

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def data(n, m, d, seed):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 1, size=(n, d))
    y = np.sin(5 * x[:, 0]) + np.cos(3 * x[:, -1]) + 0.1 * rs.standard_normal(n)
    z = x[rs.choice(n, m, replace=False)]
    return x, y, z


def col(a):
    return np.ascontiguousarray(a.T).reshape(-1)


def model(x, y, z, ls, noise, prec=gx.Precision.Fp64):
    n, d = x.shape
    return gx.Sgpr(gx.RbfArdKernel(ls), gx.GaussianLikelihood(noise), precision=prec).with_optimizer(
        gx.Fixed()).factor(col(x), n, d, y, col(z), z.shape[0])


def shard_eval(shards, params):
    """The three phases over several handles, the exchanges summed."""
    n1, n2 = shards[0].shard_sizes()
    e1 = [torch.empty(n1, dtype=torch.float64, device="cuda") for _ in shards]
    e2 = [torch.empty(n2, dtype=torch.float64, device="cuda") for _ in shards]
    for s, e in zip(shards, e1):
        s.shard_assemble(params, e)
    tot1 = torch.stack(e1).sum(0)
    nls = [s.shard_nlml(tot1, e) for s, e in zip(shards, e2)]
    tot2 = torch.stack(e2).sum(0)
    gs = [s.shard_gradient(tot2) for s in shards]
    return nls, gs


def test_fp64_shards_match_the_unsharded_evaluation():
    n, m, d = 3000, 64, 3
    x, y, z = data(n, m, d, 1)
    ls = [0.3, 0.5, 0.4]
    params = np.array([math.log(v) for v in ls] + [math.log(0.05)])
    cuts = [0, 1000, 1001, 3000]  # one shard of a single point
    shards = [model(x[a:b], y[a:b], z, ls, 0.05) for a, b in zip(cuts[:-1], cuts[1:])]
    full = model(x, y, z, ls, 0.05)
    nl_f, g_f = full.value_and_gradient(params)
    orc = O.Sgpr([[11, d]], params, col(x), n, d, y, col(z), m)
    for rep in range(2):  # the handles keep no state between evaluations
        nls, gs = shard_eval(shards, params)
        for nl, g in zip(nls, gs):
            assert O.rel_err(nl, nl_f) <= TOL and np.all(O.rel_err(g, g_f) <= TOL), (nl, nl_f, g, g_f)
            assert O.rel_err(nl, orc.nlml()) <= TOL and np.all(O.rel_err(g, orc.grad()) <= TOL)
        assert all(v == nls[0] for v in nls) and all(np.array_equal(g, gs[0]) for g in gs)
    # each shard now predicts with the global posterior
    rs = np.random.RandomState(3)
    xs = rs.uniform(0, 1, size=(50, d))
    p_f = full.predict(col(xs), 50, d)
    for s in shards:
        p = s.predict(col(xs), 50, d)
        assert np.all(O.rel_err(p.mean, p_f.mean) <= TOL) and np.all(O.rel_err(p.variance, p_f.variance) <= TOL)


def test_one_shard_through_the_orchestrator_is_the_plain_evaluation():
    n, m, d = 900, 32, 2
    x, y, z = data(n, m, d, 2)
    ls = [0.5, 0.7]
    params = np.array([math.log(v) for v in ls] + [math.log(0.1)])
    s = model(x, y, z, ls, 0.1)
    nl, g = gx.sharded_value_and_gradient(s, params, lambda t: None, device="cuda")
    nl_f, g_f = model(x, y, z, ls, 0.1).value_and_gradient(params)
    assert O.rel_err(nl, nl_f) <= TOL and np.all(O.rel_err(g, g_f) <= TOL)
    nl2, g2 = gx.sharded_value_and_gradient(s, params, lambda t: None, device="cuda", gradient=False)
    assert nl2 == nl and g2 is None


def test_mixed_shards_match_fp64():
    # each shard above the size where the Gram products are emulated
    n, m, d = 40000, 256, 3
    x, y, z = data(n, m, d, 4)
    ls = [0.3, 0.5, 0.4]
    params = np.array([math.log(v) for v in ls] + [math.log(0.05)])
    shards = [model(x[a:b], y[a:b], z, ls, 0.05, gx.Precision.Mixed) for a, b in ((0, 20000), (20000, 40000))]
    nl_f, g_f = model(x, y, z, ls, 0.05).value_and_gradient(params)
    nls, gs = shard_eval(shards, params)
    for nl, g in zip(nls, gs):
        assert O.rel_err(nl, nl_f) <= 1e-8 and np.all(O.rel_err(g, g_f) <= 1e-6), (nl, nl_f, g, g_f)
