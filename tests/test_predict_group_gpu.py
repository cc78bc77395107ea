"""Grouped prediction (gprx_exact_predict_group): small requests against
several fitted exact models in one launch, as the serving loop batches them.

Each request's mean and variance are compared with the oracle at
|a − e| / max(|e|, 1) ≤ 1e-10 and with the model's own predict at 1e-12 (a
different summation order), and a request gives the same values bit for bit
alone and inside a larger group.
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

TOL = 1e-10
D = 3


def model(n, seed, ls, noise):
    rs = np.random.RandomState(seed)
    x = rs.standard_normal((n, D))
    y = np.sin(x.sum(1)) + 0.1 * rs.standard_normal(n)
    xc = x.T.reshape(-1).copy()
    spec = gx.RbfArdKernel(ls)
    m = gx.Gpr(spec, gx.GaussianLikelihood(noise)).with_optimizer(gx.Fixed()).factor(xc, n, D, y)
    params = np.array([math.log(v) for v in ls] + [math.log(noise)])
    return m, xc, y, params


def test_group_matches_oracle_single_and_alone():
    ms = [model(100, 1, [0.7, 1.1, 1.6], 0.05), model(640, 2, [1.3, 0.9, 2.0], 0.1), model(1024, 3, [1.0, 1.0, 1.0], 0.02)]
    rs = np.random.RandomState(4)
    # (model, q): two requests on the middle model, tile edges 1, 16, 17
    plan = [(0, 1), (1, 16), (2, 17), (1, 100), (0, 33)]
    reqs = [(ms[i][0], rs.standard_normal(q * D), q) for i, q in plan]
    for kind in (gx.VarianceKind.Latent, gx.VarianceKind.Observation):
        out = gx.predict_group([r[0] for r in reqs], [r[1] for r in reqs], [r[2] for r in reqs], kind)
        for (i, q), (m, xs, _), p in zip(plan, reqs, out):
            _, xc, y, params = ms[i]
            n = y.size
            mo, vo = O.exact_predict([[11, D]], params, xc, n, D, y, xs, q, int(kind))
            assert np.all(O.rel_err(p.mean, mo) <= TOL) and np.all(O.rel_err(p.variance, vo) <= TOL)
            single = m.predict_with(xs, q, D, gx.PredictOptions(kind))
            assert np.allclose(p.mean, single.mean, rtol=1e-12, atol=1e-14)
            assert np.allclose(p.variance, single.variance, rtol=1e-12, atol=1e-14)
        # each request alone gives the same bits as inside the group
        for (m, xs, q), p in zip(reqs, out):
            a = gx.predict_group([m], [xs], [q], kind)[0]
            assert np.array_equal(a.mean, p.mean) and np.array_equal(a.variance, p.variance)


def test_group_refuses_online_and_large_models():
    m, xc, y, params = model(200, 5, [1.0, 1.0, 1.0], 0.1)
    big = model(1100, 6, [1.0, 1.0, 1.0], 0.1)[0]
    xs = np.zeros(2 * D)
    with pytest.raises(gx.GprError):
        gx.predict_group([m, big], [xs, xs], [2, 2])
    on = m.into_online()
    with pytest.raises(gx.InvalidConfig):
        gx.predict_group([on], [xs], [2])
