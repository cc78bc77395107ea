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
