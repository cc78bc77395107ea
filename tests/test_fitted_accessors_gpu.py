"""FittedGpr's data and model accessors and refit (src/gpr/fitted.rs:291-330,
836, 1084-1166): x / y give back the training data bit for bit (an online
model's current points in id order), likelihood / to_kernel the current θ,
refit re-runs the stored optimizer from the current θ (Fixed: refactors at
it), into_trainer returns a trainer at the fitted θ."""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu


def data(n=60, d=2, seed=3):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 4, size=(n, d))
    y = np.sin(x[:, 0]) + 0.3 * np.cos(2 * x[:, 1]) + 0.1 * rs.standard_normal(n)
    return np.ascontiguousarray(x.T).reshape(-1), y


def trainer():
    return gx.Gpr(gx.RbfKernel(0.8) + gx.RbfArdKernel([1.2, 0.6]), gx.GaussianLikelihood(0.05))


def test_data_and_model_accessors():
    x, y = data()
    m = trainer().with_optimizer(gx.Fixed()).factor(x, 60, 2, y)
    assert np.array_equal(m.x(), x) and np.array_equal(m.y(), y)
    assert abs(m.likelihood().noise_variance - 0.05) <= 1e-15
    assert np.allclose(m.to_kernel().get_params(), m.get_params()[:-1], rtol=0, atol=0)


def test_refit_fixed_refactors_and_lbfgs_continues():
    x, y = data()
    m = trainer().with_optimizer(gx.Fixed()).factor(x, 60, 2, y)
    v0 = m.neg_log_marginal_likelihood()
    m.refit()
    assert m.neg_log_marginal_likelihood() == v0
    f = trainer().with_optimizer(gx.Lbfgs().with_max_iterations(5)).fit(x, 60, 2, y)
    v5 = f.neg_log_marginal_likelihood()
    f.refit()
    v10 = f.neg_log_marginal_likelihood()
    assert v10 <= v5 + 1e-12 and f.report is not None
    f.with_optimizer(gx.TrustRegion().with_max_iterations(50)).refit()
    theta = f.get_params()
    v, g = f.value_and_gradient(theta)
    assert v <= v10 + 1e-12 and np.max(np.abs(g)) <= 1e-4


def test_into_trainer_keeps_the_fitted_theta():
    x, y = data()
    f = trainer().with_optimizer(gx.Lbfgs()).fit(x, 60, 2, y)
    theta = f.get_params().copy()
    t = f.into_trainer()
    g = t.with_optimizer(gx.Fixed()).factor(x, 60, 2, y)
    assert np.allclose(g.get_params(), theta, rtol=0, atol=1e-15)


def test_online_data_in_id_order():
    x, y = data(n=30)
    pts = x.reshape(2, 30).T
    on = trainer().with_optimizer(gx.Fixed()).factor(x, 30, 2, y).into_online()
    held = {int(i): k for i, k in zip(on.point_ids(), range(30))}
    rs = np.random.RandomState(0)
    extra = rs.uniform(0, 4, size=(3, 2))
    for k in range(3):
        held[on.insert(extra[k], 0.1 * k)] = 30 + k
    on.delete(on.point_ids()[4])
    allp = np.vstack([pts, extra])
    ally = np.concatenate([y, 0.1 * np.arange(3)])
    order = [held[int(i)] for i in on.point_ids()]
    assert np.array_equal(on.x(), np.ascontiguousarray(allp[order].T).reshape(-1))
    assert np.array_equal(on.y(), ally[order])
