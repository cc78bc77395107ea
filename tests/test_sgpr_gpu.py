"""GPU parity of the VFE sparse GPR path through the C ABI.

Goldens: GPyTorch SGPR (tests/sparse_gpytorch.rs, tests/online_sgpr_gpytorch.rs)
at 1e-8; everything else against the CPU oracle at 1e-10 (NLML, gradient,
moments), measured as |a − e| / max(|e|, 1), from n = 80 to n = 10⁵ with
m = 1024.
"""

import itertools
import json
import math
import os

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_GOLD = 1e-8
TOL = 1e-10


def load(name):
    with open(os.path.join(GOLD, name)) as fh:
        return json.load(fh)


def spec(nodes, theta):
    it = iter(nodes)
    th = list(theta)

    def build():
        kind, arg = next(it)
        if kind in (1, 2):
            kids = [build() for _ in range(arg)]
            k = kids[0]
            for c in kids[1:]:
                k = (k + c) if kind == 1 else (k * c)
            return k
        if kind == 10:
            return gx.RbfKernel(math.exp(th.pop(0)))
        if kind == 12:
            return gx.ConstantKernel(math.exp(th.pop(0)))
        if kind == 13:
            a, b = th.pop(0), th.pop(0)
            return gx.PeriodicKernel(math.exp(a), math.exp(b))
        return gx.RbfArdKernel([math.exp(th.pop(0)) for _ in range(arg)])

    return build()


def model(nodes, theta, noise, x, n, d, y, z, m):
    return gx.Sgpr(spec(nodes, theta), gx.GaussianLikelihood(noise)).with_optimizer(gx.Fixed()).factor(
        x, n, d, y, z, m)


@pytest.mark.parametrize("case", load("sgpr_goldens.json"), ids=lambda c: c["name"])
def test_sgpr_golden_through_abi(case):
    n, d, q, m = case["n"], case["d"], case["q"], case["m"]
    f = model(case["nodes"], case["theta"], case["noise_variance"], case["x"], n, d, case["y"], case["z"], m)
    assert O.rel_err(f.neg_log_marginal_likelihood(), case["nlml"]) <= TOL_GOLD
    for kind, key in ((0, "latent_variance"), (1, "observation_variance")):
        p = f.predict_with(case["xs"], q, d, gx.PredictOptions(kind))
        assert np.all(O.rel_err(p.mean, case["mean"]) <= TOL_GOLD)
        assert np.all(O.rel_err(p.variance, case[key]) <= TOL_GOLD)


# (d, nodes, θ, domain length per point-spacing): the domain grows with m so
# that K_mm stays well conditioned (a parity check between two FP64 codes is
# only as tight as κ(K_mm)·ε allows)
TREES = [
    (2, [[11, 2]], [math.log(0.4), math.log(0.7)], 0.5),
    (3, [[2, 2], [12, 0], [11, 3]], [math.log(1.5), math.log(0.6), math.log(0.9), math.log(1.3)], 0.6),
    (1, [[1, 2], [10, 0], [13, 0]], [math.log(0.2), math.log(0.5), math.log(0.45)], 0.3),
    (4, [[10, 0]], [math.log(0.8)], 0.8),
]


def grid(m, d, sp, rs):
    """m inducing points on a jittered grid of spacing sp (κ(K_mm) stays small)."""
    k = int(math.ceil(m ** (1.0 / d)))
    pts = np.array(list(itertools.product(range(k), repeat=d)), dtype=float)[:m] * sp
    return pts + 0.05 * sp * rs.uniform(-1, 1, size=pts.shape)


@pytest.mark.parametrize("n,m", [(80, 12), (300, 33), (1000, 129), (2000, 256)])
@pytest.mark.parametrize("tree", range(len(TREES)))
def test_sgpr_eval_matches_oracle(n, m, tree):
    d, nodes, theta, spacing = TREES[tree]
    rs = np.random.RandomState(n + 7 * tree)
    zp = grid(m, d, 1.6 * spacing, rs)
    hi = zp.max(axis=0) + 0.5 * spacing
    x = (rs.uniform(0, 1, size=(n, d)) * hi).T.reshape(-1)
    y = np.sin(6 * x[:n]) + 0.1 * rs.standard_normal(n)
    z = zp.T.reshape(-1)
    params = np.array(theta + [math.log(0.05)])
    orc = O.Sgpr(nodes, params, x, n, d, y, z, m)
    f = model(nodes, theta, 0.05, x, n, d, y, z, m)
    assert f.kmm_jitter() == orc.kmm_jitter
    nl, g = f.value_and_gradient(params)
    assert O.rel_err(nl, orc.nlml()) <= TOL, (nl, orc.nlml())
    assert np.all(O.rel_err(g, orc.grad()) <= TOL), (g, orc.grad())
    q = 23
    xs = (rs.uniform(0, 1, size=(q, d)) * hi).T.reshape(-1)
    for kind in (0, 1):
        mo, vo = orc.predict(xs, q, kind)
        p = f.predict_with(xs, q, d, gx.PredictOptions(kind))
        assert np.all(O.rel_err(p.mean, mo) <= TOL)
        assert np.all(O.rel_err(p.variance, vo) <= TOL)


@pytest.mark.parametrize("n,tree", [(20000, 1), (20000, 3), (40000, 1), (40000, 3), (100000, 1)])
def test_sgpr_eval_large_n_matches_oracle(n, tree):
    # m = 1024 inducing inputs and n up to 10⁵: the sums over n (the trace
    # term's Nyström residuals, ‖y‖², A y, the cross contraction) keep 1e-10
    m = 1024
    d, nodes, theta, spacing = TREES[tree]
    rs = np.random.RandomState(n + 7 * tree)
    zp = grid(m, d, 1.6 * spacing, rs)
    hi = zp.max(axis=0) + 0.5 * spacing
    x = (rs.uniform(0, 1, size=(n, d)) * hi).T.reshape(-1)
    y = np.sin(6 * x[:n]) + 0.1 * rs.standard_normal(n)
    z = zp.T.reshape(-1)
    params = np.array(theta + [math.log(0.05)])
    orc = O.Sgpr(nodes, params, x, n, d, y, z, m)
    f = model(nodes, theta, 0.05, x, n, d, y, z, m)
    assert f.kmm_jitter() == orc.kmm_jitter
    nl, g = f.value_and_gradient(params)
    assert O.rel_err(nl, orc.nlml()) <= TOL, (nl, orc.nlml())
    assert np.all(O.rel_err(g, orc.grad()) <= TOL), (g, orc.grad())
    q = 23
    xs = (rs.uniform(0, 1, size=(q, d)) * hi).T.reshape(-1)
    mo, vo = orc.predict(xs, q, 1)
    p = f.predict(xs, q, d)
    assert np.all(O.rel_err(p.mean, mo) <= TOL) and np.all(O.rel_err(p.variance, vo) <= TOL)


@pytest.mark.parametrize("case", load("online_sgpr_goldens.json"), ids=lambda c: c["name"])
def test_online_sgpr_golden_through_abi(case):
    n, d, q = case["n"], case["d"], case["q"]
    x = np.asarray(case["x"]).reshape(d, n)
    y = np.asarray(case["y"])
    zall = np.asarray(case["z"]).reshape(d, case["m"])
    s0, m0 = case["start_n"], case["start_m"]
    z = [zall[:, i] for i in range(m0)]
    f = model(case["nodes"], case["theta"], case["noise_variance"], x[:, :s0].reshape(-1), s0, d, y[:s0],
              np.array(z).T.reshape(-1), m0)
    on = f.into_online()
    for k, step in enumerate(case["steps"]):
        if k > 0:
            op = case["ops"][k - 1]
            if op["kind"] == "insert":
                on.insert(x[:, op["pop_index"]], y[op["pop_index"]])
            elif op["kind"] == "delete":
                on.delete(on.point_ids()[op["slot"]])
            elif op["kind"] == "insert_inducing":
                z.append(zall[:, op["pop_index"]])
                assert on.insert_inducing(zall[:, op["pop_index"]]) == max(on.inducing_ids())
            else:
                z.pop(op["slot"])
                on.delete_inducing(on.inducing_ids()[op["slot"]])
            assert on.m() == len(z)
        assert on.n() == step["n"]
        assert O.rel_err(on.neg_log_marginal_likelihood(), step["neg_log_marginal_likelihood"]) <= TOL_GOLD, k
        for kind, key in ((0, "latent_variance"), (1, "observation_variance")):
            p = on.predict_with(case["xs"], q, d, gx.PredictOptions(kind))
            assert np.all(O.rel_err(p.mean, step["mean"]) <= TOL_GOLD), k
            assert np.all(O.rel_err(p.variance, step[key]) <= TOL_GOLD), k


def test_online_sgpr_sequence_matches_oracle():
    # X insert / delete in place (rank-1 up/downdate of L_B), the pivot-gate
    # decision bit-exact with the oracle's, ids never reused
    rs = np.random.RandomState(9)
    d, n0, m = 2, 150, 20
    nodes, theta = [[11, 2]], [math.log(0.5), math.log(0.8)]
    pts = rs.uniform(0, 1, size=(n0 + 100, d))
    ys = np.sin(5 * pts.sum(1))
    z = pts[:m].T.reshape(-1)
    params = theta + [math.log(0.05)]
    f = model(nodes, theta, 0.05, pts[:n0].T.reshape(-1), n0, d, ys[:n0], z, m)
    on = f.into_online()
    orc = O.Sgpr(nodes, params, pts[:n0].T.reshape(-1), n0, d, ys[:n0], z, m)
    ids = list(range(n0))
    nxt = n0
    xs = rs.uniform(0, 1, size=(7, d)).T.reshape(-1)
    for step in range(40):
        if rs.rand() < 0.5:
            a = on.insert(pts[nxt], ys[nxt])
            b = orc.insert(pts[nxt], ys[nxt])
            assert a == b
            ids.append(a)
            nxt += 1
        else:
            slot = rs.randint(len(ids))
            pid = ids.pop(slot)
            assert on.point_ids()[slot] == pid
            on.delete(pid)
            orc.delete(pid)
        assert on.last_step_in_place() == bool(orc.last_in_place)
        assert np.array_equal(on.point_ids(), np.array(ids, dtype=np.uint64))
        assert O.rel_err(on.neg_log_marginal_likelihood(), orc.nlml()) <= TOL
        pm = on.predict(xs, 7, d)
        mo, vo = orc.predict(xs, 7, 1)
        assert np.all(O.rel_err(pm.mean, mo) <= TOL)
        assert np.all(O.rel_err(pm.variance, vo) <= TOL)


def test_sgpr_fit_decreases_nlml_and_matches_oracle_at_optimum():
    rs = np.random.RandomState(4)
    n, d, m = 600, 2, 36
    x = rs.uniform(0, 2, size=n * d)
    y = np.sin(3 * x[:n]) * np.cos(2 * x[n:]) + 0.1 * rs.standard_normal(n)
    z = grid(m, d, 0.35, rs).T.reshape(-1)
    s = gx.Sgpr(gx.RbfArdKernel([0.5, 0.5]), gx.GaussianLikelihood(0.5))
    start = s.with_optimizer(gx.Fixed()).factor(x, n, d, y, z, m).neg_log_marginal_likelihood()
    f = s.fit(x, n, d, y, z, m)
    p = f.get_params()
    nl = f.neg_log_marginal_likelihood()
    assert nl < start
    orc = O.Sgpr([[11, 2]], p, x, n, d, y, z, m)
    assert O.rel_err(nl, orc.nlml()) <= TOL
    g0 = O.Sgpr([[11, 2]], s.kernel.get_params() + [math.log(0.5)], x, n, d, y, z, m).grad()
    assert np.linalg.norm(orc.grad()) < 1e-2 * np.linalg.norm(g0)


def test_inducing_ids_changes_and_errors():
    # ids are never reused; each change equals a fresh factor at the new Z
    # (the oracle's set_inducing), and a failed change keeps the old set
    rs = np.random.RandomState(21)
    d, n, m = 2, 300, 12
    nodes, theta = [[11, 2]], [math.log(0.4), math.log(0.6)]
    params = theta + [math.log(0.05)]
    x = rs.uniform(0, 1, size=(n, d))
    y = np.sin(4 * x.sum(1)) + 0.05 * rs.standard_normal(n)
    z = [x[i] for i in range(m)]
    on = model(nodes, theta, 0.05, x.T.reshape(-1), n, d, y, np.array(z).T.reshape(-1), m).into_online()
    assert list(on.inducing_ids()) == list(range(m))
    orc = O.Sgpr(nodes, params, x.T.reshape(-1), n, d, y, np.array(z).T.reshape(-1), m)
    xs = rs.uniform(0, 1, size=(15, d)).T.reshape(-1)
    new = rs.uniform(0, 1, size=(3, d))
    for k in range(3):
        assert on.insert_inducing(new[k]) == m + k
        z.append(new[k])
    for iid in (3, 0, 13):
        slot = list(on.inducing_ids()).index(iid)
        on.delete_inducing(iid)
        z.pop(slot)
    assert list(on.inducing_ids()) == [1, 2, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14]
    orc.set_inducing(np.array(z).T.reshape(-1), len(z))
    assert O.rel_err(on.neg_log_marginal_likelihood(), orc.nlml()) <= TOL
    p = on.predict(xs, 15, d)
    mo, vo = orc.predict(xs, 15, 1)
    assert np.all(O.rel_err(p.mean, mo) <= TOL) and np.all(O.rel_err(p.variance, vo) <= TOL)
    with pytest.raises(gx.IndexOutOfRange):
        on.delete_inducing(3)
    with pytest.raises(gx.NonFiniteInput):
        on.insert_inducing([float("nan"), 0.0])
    assert on.m() == len(z)
    one = model(nodes, theta, 0.05, x.T.reshape(-1), n, d, y, x[:1].T.reshape(-1), 1).into_online()
    with pytest.raises(gx.InsufficientData):
        one.delete_inducing(0)


def test_inducing_insert_bordered_matches_oracle_and_gate():
    # inducing inserts take the bordered update (O(n m)) when the factor and
    # the bordered pivots hold, else the assembly: the decision is the
    # oracle's bit for bit, and NLML, gradient and predictions agree at 1e-10
    rs = np.random.RandomState(12)
    d, n, m = 2, 500, 9
    nodes, theta = [[11, 2]], [math.log(0.3), math.log(0.45)]
    params = np.array(theta + [math.log(0.05)])
    x = rs.uniform(0, 1, size=(n, d))
    y = np.sin(4 * x.sum(1)) + 0.05 * rs.standard_normal(n)
    z = [x[i] for i in range(m)]
    zc = np.array(z).T.reshape(-1)
    on = model(nodes, theta, 0.05, x.T.reshape(-1), n, d, y, zc, m).into_online()
    orc = O.Sgpr(nodes, params, x.T.reshape(-1), n, d, y, zc, m)
    xs = rs.uniform(0, 1, size=(11, d)).T.reshape(-1)
    kinds = []
    for k in range(8):
        zn = rs.uniform(0, 1, size=d) if k != 5 else z[2] + 1e-9  # a near duplicate sends it to the assembly
        on.insert_inducing(zn)
        orc.insert_inducing(zn)
        z.append(zn)
        assert on.last_step_in_place() == bool(orc.last_in_place), k
        kinds.append(bool(orc.last_in_place))
        assert O.rel_err(on.neg_log_marginal_likelihood(), orc.nlml()) <= TOL, k
        nl, g = on.value_and_gradient(params)
        assert O.rel_err(nl, orc.nlml()) <= TOL and np.all(O.rel_err(g, orc.grad()) <= TOL), k
        p = on.predict(xs, 11, d)
        mo, vo = orc.predict(xs, 11, 1)
        assert np.all(O.rel_err(p.mean, mo) <= TOL) and np.all(O.rel_err(p.variance, vo) <= TOL), k
    assert kinds[0] and not kinds[5]
    assert on.m() == m + 8 and list(on.inducing_ids()) == list(range(m + 8))
