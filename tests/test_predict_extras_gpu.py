"""Leave-one-out, query covariance and posterior draws from the resident
factor (gprx_exact_loo / gprx_exact_predict_covariance / gprx_exact_sample)
against the oracle, |a − e| / max(|e|, 1) ≤ 1e-10 (FP64), for a fitted model
and for an online model after inserts and deletes.
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

TOL = 1e-10
NODES = [[1, 2], [10, 0], [11, 2]]  # Rbf + RbfArd(2)


def spec(params):
    return gx.RbfKernel(math.exp(params[0])) + gx.RbfArdKernel([math.exp(params[1]), math.exp(params[2])])


def data(n, seed):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 4, size=(n, 2))
    y = np.sin(x[:, 0]) + 0.3 * np.cos(2 * x[:, 1]) + 0.1 * rs.standard_normal(n)
    return x, y


def col(a):
    return np.ascontiguousarray(a.T).reshape(-1)


PARAMS = np.array([math.log(0.9), math.log(1.3), math.log(0.7), math.log(0.08)])


def fitted(x, y):
    n = x.shape[0]
    return gx.Gpr(spec(PARAMS), gx.GaussianLikelihood(math.exp(PARAMS[-1]))).with_optimizer(gx.Fixed()).factor(
        col(x), n, 2, y)


@pytest.mark.parametrize("n", [1, 2, 65, 129, 300, 1100])
def test_loo_matches_oracle(n):
    x, y = data(n, n)
    m = fitted(x, y)
    for kind in (0, 1):
        p = m.loo_predict_with(gx.PredictOptions(kind))
        mo, vo = O.exact_loo(NODES, PARAMS, col(x), n, 2, y, kind)
        assert np.all(O.rel_err(p.mean, mo) <= TOL), n
        assert np.all(O.rel_err(p.variance, vo) <= TOL), n
    # after a gradient evaluation (which consumes the factor) the LOO is the same
    m.value_and_gradient(PARAMS)
    p2 = m.loo_predict()
    assert np.all(O.rel_err(p2.mean, O.exact_loo(NODES, PARAMS, col(x), n, 2, y, 1)[0]) <= TOL)


@pytest.mark.parametrize("n,q", [(50, 1), (300, 37), (1000, 130)])
def test_covariance_matches_oracle(n, q):
    x, y = data(n, 7 + n)
    xs = np.random.RandomState(q).uniform(0, 4, size=(q, 2))
    m = fitted(x, y)
    for kind in (0, 1):
        c = m.predict_covariance_with(col(xs), q, 2, gx.PredictOptions(kind))
        mo, co = O.exact_covariance(NODES, PARAMS, col(x), n, 2, y, col(xs), q, kind)
        assert np.all(O.rel_err(c.mean, mo) <= TOL)
        assert np.all(O.rel_err(c.covariance, co) <= TOL)
        # the diagonal is the plain prediction's variance
        p = m.predict_with(col(xs), q, 2, gx.PredictOptions(kind))
        assert np.all(O.rel_err(np.diag(c.covariance), p.variance) <= TOL)


def test_sample_matches_oracle():
    n, q, draws, seed = 400, 40, 6, 11
    x, y = data(n, 3)
    xs = np.random.RandomState(5).uniform(0, 4, size=(q, 2))
    m = fitted(x, y)
    out = m.sample(col(xs), q, 2, draws, seed)
    want = O.exact_sample(NODES, PARAMS, col(x), n, 2, y, col(xs), q, 1, draws, seed)
    assert out.shape == (q * draws,)
    assert np.all(O.rel_err(out, want) <= 1e-9)
    assert m.sample(col(xs), q, 2, 0, seed).size == 0
    # same seed, same draws
    assert np.array_equal(out, m.sample(col(xs), q, 2, draws, seed))


def test_online_model_loo_and_covariance():
    x, y = data(200, 9)
    extra_x, extra_y = data(5, 10)
    on = fitted(x, y).into_online()
    pts, ys = list(x), list(y)
    for i in range(5):
        on.insert(extra_x[i], extra_y[i])
        pts.append(extra_x[i])
        ys.append(extra_y[i])
    for slot in (3, 100):
        pid = on.point_ids()[slot]
        on.delete(pid)
        del pts[slot]
        del ys[slot]
    xa, ya = np.array(pts), np.array(ys)
    n = xa.shape[0]
    assert on.n() == n
    for kind in (0, 1):
        p = on.loo_predict_with(gx.PredictOptions(kind))
        mo, vo = O.exact_loo(NODES, PARAMS, col(xa), n, 2, ya, kind)
        assert np.all(O.rel_err(p.mean, mo) <= TOL) and np.all(O.rel_err(p.variance, vo) <= TOL)
    xs = np.random.RandomState(1).uniform(0, 4, size=(12, 2))
    c = on.predict_covariance(col(xs), 12, 2)
    mo, co = O.exact_covariance(NODES, PARAMS, col(xa), n, 2, ya, col(xs), 12, 1)
    assert np.all(O.rel_err(c.mean, mo) <= TOL) and np.all(O.rel_err(c.covariance, co) <= TOL)
