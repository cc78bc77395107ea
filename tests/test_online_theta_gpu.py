"""θ writes, NLML + gradient evaluations and Hessians on an online model
(OnlineGpr::set_params / value_and_gradient_into / hessian_into,
src/gpr/online.rs:659-697): they run through a plain LLT of the current
points and leave the model online at the new θ (with_llt_view,
src/gpr/online.rs:1151-1185).  Checked against the oracle on the points the
model holds after inserts and deletes (1e-10; Hessian 1e-9 of max|H|); a
failed write leaves the model's factor, α and θ as they were (bit for bit)."""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

NODES = [[1, 2], [10, 0], [11, 2]]  # Rbf + RbfArd(2)
D = 2


def col(a):
    return np.ascontiguousarray(np.asarray(a, dtype=float).T).reshape(-1)


def online_model(seed=0, start=40):
    rs = np.random.RandomState(seed)
    pts = rs.uniform(0, 4, size=(start + 30, D))
    ys = np.sin(pts[:, 0]) + 0.3 * np.cos(2 * pts[:, 1]) + 0.05 * rs.standard_normal(len(pts))
    params = np.array([math.log(0.9), math.log(1.3), math.log(0.7), math.log(0.05)])
    spec = gx.KernelSpec.from_nodes(NODES, params[:-1])
    m = gx.Gpr(spec, gx.GaussianLikelihood(math.exp(params[-1]))).with_optimizer(gx.Fixed()).factor(
        col(pts[:start]), start, D, ys[:start])
    on = m.into_online()
    held = {int(i): k for i, k in zip(on.point_ids(), range(start))}
    for k in range(start, start + 12):
        held[on.insert(pts[k], ys[k])] = k
    for pid in list(on.point_ids()[[3, 17, 30]]):
        on.delete(pid)
        del held[int(pid)]
    return on, pts, ys, held, params, rs


def current(on, pts, ys, held):
    order = [held[int(i)] for i in on.point_ids()]
    return pts[order], ys[order]


def test_online_eval_and_hessian_match_oracle():
    on, pts, ys, held, params, _ = online_model()
    x, y = current(on, pts, ys, held)
    n = len(y)
    moved = params + np.array([0.1, -0.05, 0.08, 0.2])
    v, g = on.value_and_gradient(moved)
    vo, go, _, _ = O.exact_eval(NODES, moved, col(x), n, D, y)
    assert O.rel_err(v, vo) <= 1e-10 and np.all(O.rel_err(g, go) <= 1e-10)
    h = on.hessian(moved)
    ho = O.exact_hessian(NODES, moved, col(x), n, D, y)
    assert np.max(np.abs(h - ho)) <= 1e-9 * max(np.max(np.abs(ho)), 1.0)
    # still online, now at `moved`: its NLML and the next insert follow the new θ
    assert O.rel_err(on.neg_log_marginal_likelihood(), vo) <= 1e-10
    k = max(held.values()) + 1
    held[on.insert(pts[k], ys[k])] = k
    x2, y2 = current(on, pts, ys, held)
    vo2 = O.exact_eval(NODES, moved, col(x2), len(y2), D, y2, grad=False)[0]
    assert O.rel_err(on.neg_log_marginal_likelihood(), vo2) <= 1e-10
    xs = np.array([[0.5, 1.5], [2.5, 3.1]])
    p = on.predict(col(xs), 2, D)
    mo, vvo = O.exact_predict(NODES, moved, col(x2), len(y2), D, y2, col(xs), 2, 0)
    assert np.all(O.rel_err(p.mean, mo) <= 1e-10)


def test_online_set_params_then_insert():
    on, pts, ys, held, params, _ = online_model(seed=1)
    moved = params - 0.1
    on.set_params(moved)
    assert np.allclose(on.get_params(), moved, rtol=0, atol=1e-15)
    x, y = current(on, pts, ys, held)
    vo = O.exact_eval(NODES, moved, col(x), len(y), D, y, grad=False)[0]
    assert O.rel_err(on.neg_log_marginal_likelihood(), vo) <= 1e-10
    pid = on.point_ids()[5]
    on.delete(pid)
    del held[int(pid)]
    x, y = current(on, pts, ys, held)
    vo = O.exact_eval(NODES, moved, col(x), len(y), D, y, grad=False)[0]
    assert O.rel_err(on.neg_log_marginal_likelihood(), vo) <= 1e-10


def test_online_failed_write_leaves_the_model():
    on, pts, ys, held, params, _ = online_model(seed=2)
    xs = np.array([[1.0, 2.0], [3.0, 0.5]])
    before = (on.neg_log_marginal_likelihood(), on.predict(col(xs), 2, D).mean.copy(), on.get_params().copy())
    bad = params.copy()
    bad[1] = float("nan")
    with pytest.raises(gx.InvalidHyperparameter):
        on.set_params(bad)
    with pytest.raises(gx.InvalidHyperparameter):
        on.value_and_gradient(bad)
    after = (on.neg_log_marginal_likelihood(), on.predict(col(xs), 2, D).mean, on.get_params())
    assert after[0] == before[0] and np.array_equal(after[1], before[1]) and np.array_equal(after[2], before[2])
    k = max(held.values()) + 1
    held[on.insert(pts[k], ys[k])] = k
    x, y = current(on, pts, ys, held)
    vo = O.exact_eval(NODES, params, col(x), len(y), D, y, grad=False)[0]
    assert O.rel_err(on.neg_log_marginal_likelihood(), vo) <= 1e-10
