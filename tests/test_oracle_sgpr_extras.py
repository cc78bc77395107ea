"""CPU checks of the oracle's VFE query covariance and posterior draws (the
parity references of gprx_sgpr_predict_covariance / gprx_sgpr_sample): the diagonal
is the predictive variance, the matrix is symmetric, and with the inducing
inputs at the training points the VFE posterior is the exact one, so the
covariance and the seeded draws equal the exact model's (1e-8)."""

import math

import numpy as np

import oracle_lib as O

NODES = [[1, 2], [10, 0], [11, 2]]  # Rbf + RbfArd(2)
PARAMS = np.array([math.log(0.9), math.log(1.3), math.log(0.7), math.log(0.08)])


def col(a):
    return np.ascontiguousarray(np.asarray(a, dtype=float).T).reshape(-1)


def setup(n=9, seed=4):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 6, size=(n, 2))
    y = np.sin(x[:, 0]) + 0.3 * np.cos(2 * x[:, 1])
    xs = rs.uniform(0, 6, size=(5, 2))
    return x, y, xs


def test_sgpr_covariance_diagonal_and_symmetry():
    x, y, xs = setup()
    z = x[::2]
    s = O.Sgpr(NODES, PARAMS, col(x), len(y), 2, y, col(z), len(z))
    for kind in (0, 1):
        mean, cov = s.covariance(col(xs), 5, kind)
        pm, pv = s.predict(col(xs), 5, kind)
        assert np.array_equal(mean, pm) and np.array_equal(np.diag(cov), pv)
        off = cov - np.diag(np.diag(cov))
        assert np.max(np.abs(off - off.T)) <= 1e-14


def test_sgpr_with_inducing_at_the_points_is_exact():
    x, y, xs = setup()
    s = O.Sgpr(NODES, PARAMS, col(x), len(y), 2, y, col(x), len(y))
    for kind in (0, 1):
        mean, cov = s.covariance(col(xs), 5, kind)
        me, ce = O.exact_covariance(NODES, PARAMS, col(x), len(y), 2, y, col(xs), 5, kind)
        assert np.max(np.abs(mean - me)) <= 1e-8 and np.max(np.abs(cov - ce)) <= 1e-8
    draws = s.sample(col(xs), 5, 1, 4, 7)
    de = O.exact_sample(NODES, PARAMS, col(x), len(y), 2, y, col(xs), 5, 1, 4, 7)
    assert np.max(np.abs(draws - np.asarray(de).reshape(4, 5))) <= 1e-7
