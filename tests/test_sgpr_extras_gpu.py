"""gprx_sgpr_predict_covariance / gprx_sgpr_sample against the oracle (whose
VFE covariance is pinned on the inducing-at-the-points identity with the
exact model): |a − e| / max(|e|, 1) ≤ 1e-10 for the mean and covariance,
1e-9 for the seeded draws; the diagonal equals gprx_sgpr_predict's variance
bit for bit."""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O
from test_sgpr_gpu import TREES, grid, model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,m,q", [(80, 12, 1), (300, 33, 17), (1000, 129, 150)])
@pytest.mark.parametrize("tree", range(len(TREES)))
def test_sgpr_covariance_and_draws_match_oracle(n, m, q, tree):
    d, nodes, theta, spacing = TREES[tree]
    rs = np.random.RandomState(n + 11 * tree)
    zp = grid(m, d, 1.6 * spacing, rs)
    hi = zp.max(axis=0) + 0.5 * spacing
    x = (rs.uniform(0, 1, size=(n, d)) * hi).T.reshape(-1)
    y = np.sin(6 * x[:n]) + 0.1 * rs.standard_normal(n)
    z = zp.T.reshape(-1)
    params = np.array(theta + [math.log(0.05)])
    orc = O.Sgpr(nodes, params, x, n, d, y, z, m)
    f = model(nodes, theta, 0.05, x, n, d, y, z, m)
    xs = (rs.uniform(0, 1, size=(q, d)) * hi).T.reshape(-1)
    for kind in (0, 1):
        c = f.predict_covariance_with(xs, q, d, gx.PredictOptions(kind))
        mo, co = orc.covariance(xs, q, kind)
        assert np.all(O.rel_err(c.mean, mo) <= 1e-10)
        assert np.all(O.rel_err(c.covariance, co) <= 1e-10)
        p = f.predict_with(xs, q, d, gx.PredictOptions(kind))
        assert np.array_equal(np.diag(c.covariance), p.variance)
    draws = f.sample_with(xs, q, d, gx.PredictOptions(1), 3, 11)
    do = orc.sample(xs, q, 1, 3, 11)
    assert np.all(O.rel_err(draws, do.reshape(-1)) <= 1e-9)


def test_sgpr_set_params_refit_and_accessors():
    d, nodes, theta, spacing = TREES[1]
    rs = np.random.RandomState(5)
    n, m = 300, 33
    zp = grid(m, d, 1.6 * spacing, rs)
    hi = zp.max(axis=0) + 0.5 * spacing
    x = (rs.uniform(0, 1, size=(n, d)) * hi).T.reshape(-1)
    y = np.sin(6 * x[:n]) + 0.1 * rs.standard_normal(n)
    z = zp.T.reshape(-1)
    f = model(nodes, theta, 0.05, x, n, d, y, z, m)
    moved = np.array(theta + [math.log(0.05)]) + 0.05
    f.set_params(moved)
    assert np.allclose(f.get_params(), moved, rtol=0, atol=1e-15)
    orc = O.Sgpr(nodes, moved, x, n, d, y, z, m)
    assert O.rel_err(f.neg_log_marginal_likelihood(), orc.nlml()) <= 1e-10
    assert abs(f.likelihood().noise_variance - math.exp(moved[-1])) <= 1e-15
    assert np.allclose(f.to_kernel().get_params(), moved[:-1], rtol=0, atol=0)
    v0 = f.neg_log_marginal_likelihood()
    f.refit()  # Fixed: reassembles at the current θ
    assert f.neg_log_marginal_likelihood() == v0
    f.with_optimizer(gx.Lbfgs().with_max_iterations(10)).refit()
    assert f.neg_log_marginal_likelihood() <= v0 + 1e-12
    bad = moved.copy()
    bad[0] = float("nan")
    before = f.get_params().copy()
    with pytest.raises(gx.InvalidHyperparameter):
        f.set_params(bad)
    assert np.array_equal(f.get_params(), before)


def test_sgpr_jitter_policy_reaches_the_device():
    # a K_mm with duplicated inducing inputs fails without jitter: the fixed
    # policy retries once with its j, as the oracle does with the same policy
    d, nodes, theta, spacing = TREES[0]
    rs = np.random.RandomState(9)
    n, m = 120, 9
    zp = grid(m - 1, d, 1.6 * spacing, rs)
    zp = np.vstack([zp, zp[:1]])
    hi = zp.max(axis=0) + 0.5 * spacing
    x = (rs.uniform(0, 1, size=(n, d)) * hi).T.reshape(-1)
    y = np.sin(6 * x[:n]) + 0.1 * rs.standard_normal(n)
    z = zp.T.reshape(-1)
    params = np.array(theta + [math.log(0.05)])
    pol = gx.JitterPolicy.fixed(1e-6)
    from test_sgpr_gpu import spec
    f = gx.Sgpr(spec(nodes, theta), gx.GaussianLikelihood(0.05)).with_jitter_policy(pol).with_optimizer(
        gx.Fixed()).factor(x, n, d, y, z, m)
    orc = O.Sgpr(nodes, params, x, n, d, y, z, m, jitter=(0, 1e-6, 1.0, 0, 1e-6))
    assert f.kmm_jitter() == orc.kmm_jitter == 1e-6
    assert O.rel_err(f.neg_log_marginal_likelihood(), orc.nlml()) <= 1e-10
