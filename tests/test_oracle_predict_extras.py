"""CPU checks of the oracle's leave-one-out, query covariance and posterior
draws (the parity references of gprx_exact_loo / _predict_covariance / _sample),
pinned on identities the reference's own tests use (src/gpr/tests.rs:1727-1870:
LOO at n = 1 is the prior, LOO matches a refit without the point, the
observation variance is the latent one plus the noise) and on the draw
formula μ + L z with the seeded generator's normals (src/prediction.rs:206-243).
"""

import math

import numpy as np

import gprx_b200 as gx
import oracle_lib as O

NODES = [[1, 2], [10, 0], [11, 2]]  # Rbf + RbfArd(2)


def setup(n, seed=0):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 4, size=(n, 2))
    y = np.sin(x[:, 0]) + 0.3 * np.cos(2 * x[:, 1]) + 0.1 * rs.standard_normal(n)
    params = np.array([math.log(0.9), math.log(1.3), math.log(0.7), math.log(0.08)])
    return x, y, params


def col(a):
    return np.ascontiguousarray(a.T).reshape(-1)


def test_loo_at_one_point_is_the_prior():
    x, y, params = setup(1)
    m, v = O.exact_loo(NODES, params, col(x), 1, 2, y, 1)
    k = O.exact_covariance(NODES, params, col(x), 1, 2, y, col(x), 1, 0)[1][0, 0]  # posterior at the point
    assert abs(m[0]) <= 1e-12
    prior = 2.0 + math.exp(params[-1])  # two unit-variance RBF terms plus the noise
    assert abs(v[0] - prior) <= 1e-12 * prior
    assert k < prior


def test_loo_matches_a_refit_without_the_point():
    n = 9
    x, y, params = setup(n, 1)
    for kind in (0, 1):
        m, v = O.exact_loo(NODES, params, col(x), n, 2, y, kind)
        for i in range(n):
            keep = [j for j in range(n) if j != i]
            mo, vo = O.exact_predict(NODES, params, col(x[keep]), n - 1, 2, y[keep], col(x[i:i + 1]), 1, kind)
            assert O.rel_err(m[i], mo[0]) <= 1e-10 and O.rel_err(v[i], vo[0]) <= 1e-10, (i, kind)


def test_loo_observation_is_latent_plus_noise():
    n = 12
    x, y, params = setup(n, 2)
    _, lat = O.exact_loo(NODES, params, col(x), n, 2, y, 0)
    _, obs = O.exact_loo(NODES, params, col(x), n, 2, y, 1)
    noise = math.exp(params[-1])
    assert np.all(np.abs(obs - np.maximum(lat, 0) - noise) <= 1e-12 * obs + 1e-15 * (lat > 0))


def test_covariance_diagonal_and_mean_are_the_prediction():
    n, q = 30, 7
    x, y, params = setup(n, 3)
    xs = np.random.RandomState(4).uniform(0, 4, size=(q, 2))
    for kind in (0, 1):
        mean, cov = O.exact_covariance(NODES, params, col(x), n, 2, y, col(xs), q, kind)
        mo, vo = O.exact_predict(NODES, params, col(x), n, 2, y, col(xs), q, kind)
        assert np.all(O.rel_err(mean, mo) <= 1e-12)
        assert np.all(O.rel_err(np.diag(cov), vo) <= 1e-10)
        assert np.allclose(cov, cov.T, rtol=0, atol=1e-15)


def test_draws_are_mean_plus_cholesky_times_seeded_normals():
    n, q, draws, seed = 25, 6, 5, 17
    x, y, params = setup(n, 5)
    xs = np.random.RandomState(6).uniform(0, 4, size=(q, 2))
    out = O.exact_sample(NODES, params, col(x), n, 2, y, col(xs), q, 1, draws, seed)
    mean, cov = O.exact_covariance(NODES, params, col(x), n, 2, y, col(xs), q, 1)
    lc = np.linalg.cholesky(cov)
    z = gx.SeededRng(seed).normal(q * draws).reshape(draws, q)
    want = (mean[None, :] + z @ lc.T).reshape(-1)
    assert np.all(O.rel_err(out, want) <= 1e-12)
    assert O.exact_sample(NODES, params, col(x), n, 2, y, col(xs), q, 1, 0, seed).size == 0
