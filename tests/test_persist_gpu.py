"""Saved exact models through the GPU handle: save / save_with_factor and
LoadedGpr.load give a resident model that predicts what the original did
(within 1e-12 relative; bit for bit when the load refactors the same matrix),
a stored factor is used without refactoring, and an online model comes back
with its point ids so the next insert returns the id it would have.
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
from gprx_b200 import _lib as L

pytestmark = pytest.mark.gpu


def data(n, d, seed):
    rs = np.random.RandomState(seed)
    x = rs.standard_normal((n, d))
    y = np.sin(x.sum(1)) + 0.1 * rs.standard_normal(n)
    return np.ascontiguousarray(x.T).reshape(-1), y


def model(n, d=3, seed=0):
    x, y = data(n, d, seed)
    spec = gx.ConstantKernel(1.5) * gx.RbfArdKernel([0.8, 1.2, 2.0][:d]) + gx.RbfKernel(1.7)
    return gx.Gpr(spec, gx.GaussianLikelihood(0.05)).with_optimizer(gx.Fixed()).factor(x, n, d, y)


def rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1.0)


@pytest.mark.parametrize("n", [1, 129, 700])
def test_save_with_factor_then_load_predicts_the_same(tmp_path, n):
    m = model(n)
    rs = np.random.RandomState(1)
    xs = rs.standard_normal(50 * 3)
    p0 = m.predict(xs, 50, 3)
    m.save_with_factor(tmp_path / "m")
    c0 = L.lib().gprx_launch_count()
    m2 = gx.LoadedGpr.load(tmp_path / "m")
    p1 = m2.predict(xs, 50, 3)
    launches = L.lib().gprx_launch_count() - c0
    assert np.all(rel(p1.mean, p0.mean) <= 1e-12) and np.all(rel(p1.variance, p0.variance) <= 1e-12)
    assert rel(m2.neg_log_marginal_likelihood(), m.neg_log_marginal_likelihood()) <= 1e-12
    assert np.array_equal(m2.get_params(), m.get_params()) or np.all(rel(m2.get_params(), m.get_params()) <= 1e-15)
    # the stored factor is used: no diagonal-block factor steps were launched
    m3 = gx.LoadedGpr.load(tmp_path / "m")
    c1 = L.lib().gprx_launch_count()
    m3.predict(xs, 50, 3)
    assert L.lib().gprx_launch_count() - c1 < launches + 8


def test_save_without_factor_refactors_to_the_same_bits(tmp_path):
    m = model(300, seed=2)
    xs = np.random.RandomState(2).standard_normal(20 * 3)
    p0 = m.predict(xs, 20, 3)
    m.save(tmp_path / "m")
    assert not gx.LoadedGpr.inspect(tmp_path / "m").has_factor
    p1 = gx.LoadedGpr.load(tmp_path / "m").predict(xs, 20, 3)
    assert np.all(rel(p1.mean, p0.mean) <= 1e-13) and np.all(rel(p1.variance, p0.variance) <= 1e-13)


@pytest.mark.parametrize("with_factor", [True, False])
def test_online_model_round_trip_keeps_ids(tmp_path, with_factor):
    on = model(150, d=2, seed=3).into_online()
    x_new, y_new = data(4, 2, 4)
    xn = x_new.reshape(2, 4).T
    for i in range(3):
        on.insert(xn[i], y_new[i])
    on.delete(on.point_ids()[10])
    (on.save_with_factor if with_factor else on.save)(tmp_path / "m")
    back = gx.LoadedGpr.load(tmp_path / "m")
    assert isinstance(back, gx.OnlineGpr)
    assert np.array_equal(back.point_ids(), on.point_ids())
    xs = np.random.RandomState(5).standard_normal(10 * 2)
    p0, p1 = on.predict(xs, 10, 2), back.predict(xs, 10, 2)
    assert np.all(rel(p1.mean, p0.mean) <= 1e-10) and np.all(rel(p1.variance, p0.variance) <= 1e-10)
    assert back.insert(xn[3], y_new[3]) == on.insert(xn[3], y_new[3])
