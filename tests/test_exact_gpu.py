"""GPU parity of the exact-GPR path through the C ABI.

Every case is checked against the CPU oracle (oracle/gprx_oracle.cpp) on the
same inputs, and the golden cases against the reference's committed goldens.
Tolerance: |a − e| / max(|e|, 1) ≤ 1e-10 against the oracle (FP64 end to end)
and ≤ 1e-8 against the reference goldens (tests/goldens.rs:15).
"""

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
TOL_ORACLE = 1e-10


def load(name):
    with open(os.path.join(GOLD, name)) as fh:
        return json.load(fh)


def spec_from_nodes(nodes, theta, d):
    """KernelSpec from a prefix node list and log θ (fixture format)."""
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
        if kind == 11:
            ls = [math.exp(th.pop(0)) for _ in range(arg)]
            return gx.RbfArdKernel(ls)
        raise KeyError(kind)

    return build()


def fixed_model(nodes, theta, noise, x, n, d, y):
    spec = spec_from_nodes(nodes, theta, d)
    return gx.Gpr(spec, gx.GaussianLikelihood(noise)).with_optimizer(gx.Fixed()).factor(x, n, d, y)


def rel(a, e):
    return O.rel_err(a, e)


@pytest.mark.parametrize("case", load("exact_goldens.json") + load("sklearn_goldens.json"), ids=lambda c: c["name"])
def test_exact_golden_through_abi(case):
    n, d, q = case["n"], case["d"], case["q"]
    m = fixed_model(case["nodes"], case["theta"], case["noise_variance"], case["x"], n, d, case["y"])
    assert rel(m.neg_log_marginal_likelihood(), case["nlml"]) <= TOL_GOLD
    params = np.array(case["theta"] + [math.log(case["noise_variance"])])
    v, g = m.value_and_gradient(params)
    assert rel(v, case["nlml"]) <= TOL_GOLD
    if case["grad_kernel"] is not None:
        assert np.all(rel(g[:-1], case["grad_kernel"]) <= TOL_GOLD), (g, case["grad_kernel"])
    if case["grad_noise"] is not None:
        assert rel(g[-1], case["grad_noise"]) <= TOL_GOLD
    lat = m.predict_with(case["xs"], q, d, gx.PredictOptions(gx.VarianceKind.Latent))
    obs = m.predict(case["xs"], q, d)
    assert np.all(rel(lat.mean, case["mean"]) <= TOL_GOLD)
    assert np.all(rel(obs.mean, case["mean"]) <= TOL_GOLD)
    assert np.all(rel(lat.variance, case["latent_variance"]) <= TOL_GOLD)
    assert np.all(rel(obs.variance, case["observation_variance"]) <= TOL_GOLD)


TREES = {
    "rbf": ([[10, 0]], [math.log(0.9)]),
    "const_ard": (None, None),  # built per d
    "rbf_plus_periodic": ([[1, 2], [10, 0], [13, 0]], [math.log(1.1), math.log(0.8), math.log(1.7)]),
    "sum_of_products": ([[1, 2], [2, 2], [12, 0], [10, 0], [10, 0]], [math.log(1.3), math.log(0.7), math.log(2.0)]),
}


def tree(name, d):
    if name == "const_ard":
        rs = np.random.RandomState(d)
        ls = np.exp(rs.uniform(math.log(0.5), math.log(3.0), size=d))
        return [[2, 2], [12, 0], [11, d]], [math.log(2.0)] + list(np.log(ls))
    return TREES[name]


def make_data(n, d, seed, periodic=False):
    rs = np.random.RandomState(seed)
    x = rs.standard_normal((n, d)) if not periodic else rs.uniform(0, 3, size=(n, d))
    y = np.sin(x.sum(1)) + 0.1 * rs.standard_normal(n)
    return x.T.reshape(-1).copy(), y


# block edges of the 128-wide panel and of the 64-wide fill tiles
SIZES = [1, 2, 7, 63, 64, 65, 127, 128, 129, 257, 300]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("name", ["rbf", "const_ard", "rbf_plus_periodic", "sum_of_products"])
def test_exact_eval_matches_oracle(n, name):
    d = 1 if name == "rbf_plus_periodic" else 3
    nodes, theta = tree(name, d)
    noise = 0.3 if name == "rbf_plus_periodic" else 0.05
    x, y = make_data(n, d, seed=n * 7 + len(name), periodic=(name == "rbf_plus_periodic"))
    params = np.array(theta + [math.log(noise)])
    nl_o, g_o, a_o, _ = O.exact_eval(nodes, params, x, n, d, y)
    m = fixed_model(nodes, theta, noise, x, n, d, y)
    nl, g = m.value_and_gradient(params)
    assert rel(nl, nl_o) <= TOL_ORACLE, (nl, nl_o)
    assert np.all(rel(g, g_o) <= TOL_ORACLE), (g, g_o)
    # value-only path (keeps L) and the factor's NLML
    assert rel(m.value(params), nl_o) <= TOL_ORACLE
    assert rel(m.neg_log_marginal_likelihood(), nl_o) <= TOL_ORACLE
    assert np.all(rel(m.alpha(), a_o) <= 1e-9)
    q = 37
    rs = np.random.RandomState(n)
    xs = rs.standard_normal(q * d)
    for kind in (0, 1):
        mo, vo = O.exact_predict(nodes, params, x, n, d, y, xs, q, kind)
        p = m.predict_with(xs, q, d, gx.PredictOptions(kind))
        assert np.all(rel(p.mean, mo) <= TOL_ORACLE)
        assert np.all(rel(p.variance, vo) <= TOL_ORACLE)


def test_exact_eval_mid_size_ard8_matches_oracle():
    # the C2 tree (Constant · RbfArd, d = 8) at n = 1536, three θ
    n, d = 1536, 8
    nodes, theta = tree("const_ard", d)
    x, y = make_data(n, d, seed=11)
    m = fixed_model(nodes, theta, 0.0025, x, n, d, y)
    rs = np.random.RandomState(1)
    for k in range(3):
        params = np.array(theta + [math.log(0.0025)]) + 0.1 * rs.standard_normal(len(theta) + 1)
        nl_o, g_o, _, _ = O.exact_eval(nodes, params, x, n, d, y)
        nl, g = m.value_and_gradient(params)
        assert rel(nl, nl_o) <= TOL_ORACLE
        assert np.all(rel(g, g_o) <= TOL_ORACLE), (g, g_o)


def test_exact_eval_c2_size_fp64_matches_oracle():
    # the C2 size and tree (n = 8192, Constant · RbfArd d = 8, x ~ N(0, I₈),
    # σn² = 0.05²) in the plain FP64 form, one evaluation against the oracle
    n, d = 8192, 8
    nodes, theta = tree("const_ard", d)
    x, y = make_data(n, d, seed=12)
    m = fixed_model(nodes, theta, 0.0025, x, n, d, y)
    params = np.array(theta + [math.log(0.0025)])
    nl_o, g_o, a_o, _ = O.exact_eval(nodes, params, x, n, d, y)
    nl, g = m.value_and_gradient(params)
    assert rel(nl, nl_o) <= TOL_ORACLE, (nl, nl_o)
    assert np.all(rel(g, g_o) <= TOL_ORACLE), (g, g_o)
    q = 64
    xs = np.random.RandomState(13).standard_normal(q * d)
    mo, vo = O.exact_predict(nodes, params, x, n, d, y, xs, q, 1)
    p = m.predict(xs, q, d)
    assert np.all(rel(p.mean, mo) <= TOL_ORACLE) and np.all(rel(p.variance, vo) <= TOL_ORACLE)


def test_eval_is_deterministic():
    n, d = 700, 3
    nodes, theta = tree("const_ard", d)
    x, y = make_data(n, d, seed=5)
    m = fixed_model(nodes, theta, 0.01, x, n, d, y)
    params = np.array(theta + [math.log(0.01)])
    a = m.value_and_gradient(params)
    b = m.value_and_gradient(params)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])


def test_cholesky_failure_restores_previous_theta():
    # a periodic leaf on a 3-D Euclidean distance is indefinite: with a tiny
    # noise the factor fails (CholeskyFailed, stage Fit) and the model keeps
    # the previous θ and its factor (src/gpr/exact_fit.rs:196-206).
    n, d = 60, 3
    nodes, theta = [[13, 0]], [math.log(1.0), math.log(1.0)]
    x, y = make_data(n, d, seed=2, periodic=True)
    good = np.array(theta + [math.log(5.0)])
    m = fixed_model(nodes, theta, 5.0, x, n, d, y)
    before = m.neg_log_marginal_likelihood()
    bad = np.array(theta + [math.log(1e-4)])
    with pytest.raises(gx.CholeskyFailed) as ei:
        m.value_and_gradient(bad)
    assert ei.value.stage == gx.CholeskyStage.Fit and ei.value.matrix_size == n
    assert np.allclose(m.get_params(), good)
    assert m.neg_log_marginal_likelihood() == pytest.approx(before, rel=1e-14)
    with pytest.raises(O.OracleError):
        O.exact_eval(nodes, bad, x, n, d, y)


def test_jitter_retry_matches_oracle():
    n, d = 60, 3
    nodes, theta = [[13, 0]], [math.log(1.0), math.log(1.0)]
    x, y = make_data(n, d, seed=2, periodic=True)
    noise = 1e-4
    params = np.array(theta + [math.log(noise)])
    jit = (1, 1e-3, 10.0, 6, 10.0)
    with pytest.raises(O.OracleError):
        O.exact_eval(nodes, params, x, n, d, y)
    nl_o, g_o, _, j_o = O.exact_eval(nodes, params, x, n, d, y, jitter=jit)
    spec = spec_from_nodes(nodes, theta, d)
    g = gx.Gpr(spec, gx.GaussianLikelihood(noise)).with_optimizer(gx.Fixed())
    g = g.with_jitter_adaptive(*jit[1:])
    m = g.factor(x, n, d, y)
    assert m.factor_jitter() == j_o and j_o > 0
    nl, gr = m.value_and_gradient(params)
    assert rel(nl, nl_o) <= TOL_ORACLE
    assert np.all(rel(gr, g_o) <= TOL_ORACLE)


@pytest.mark.parametrize("case", load("online_goldens.json"), ids=lambda c: c["name"])
def test_online_insert_golden_through_abi(case):
    n, d, q, s = case["n"], case["d"], case["q"], case["start_n"]
    x = np.asarray(case["x"]).reshape(d, n)
    y = np.asarray(case["y"])
    m = fixed_model(case["nodes"], case["theta"], case["noise_variance"], x[:, :s].reshape(-1), s, d, y[:s])
    on = m.into_online()
    for k, step in enumerate(case["steps"]):
        if k > 0:
            on.insert(x[:, s + k - 1], y[s + k - 1])
        assert on.n() == step["n"]
        p = on.predict(case["xs"], q, d)
        assert np.all(rel(p.mean, step["mean"]) <= TOL_GOLD)
        assert np.all(rel(p.variance, step["observation_variance"]) <= TOL_GOLD)
        assert rel(on.neg_log_marginal_likelihood(), step["neg_log_marginal_likelihood"]) <= TOL_GOLD


@pytest.mark.parametrize("start", [5, 40, 150])
def test_online_insert_delete_sequence_matches_oracle(start):
    # tests/online_ops.rs:110-197: random insert / delete sequences; ids are
    # never reused and compaction keeps buffer order (bit-exact id logic)
    rs = np.random.RandomState(start)
    d = 2
    nodes, theta = [[11, 2]], [math.log(0.9), math.log(1.4)]
    noise = 0.05
    pts = rs.uniform(0, 4, size=(start + 200, d))
    ys = np.sin(pts.sum(1))
    live = list(range(start))
    x0 = pts[live].T.reshape(-1)
    m = fixed_model(nodes, theta, noise, x0, start, d, ys[live])
    on = m.into_online()
    orc = O.Online(nodes, theta + [math.log(noise)], x0, start, d, ys[live])
    nxt = start
    xs = rs.uniform(0, 4, size=(6, d)).T.reshape(-1)
    for step in range(40):
        if rs.rand() < 0.55 and nxt < len(pts):
            a = on.insert(pts[nxt], ys[nxt])
            b = orc.insert(pts[nxt], ys[nxt])
            assert a == b
            nxt += 1
        elif on.n() > 1:
            slot = rs.randint(on.n())
            pid = on.point_ids()[slot]
            assert pid == orc.ids()[slot]
            on.delete(pid)
            orc.delete(pid)
        assert np.array_equal(on.point_ids(), orc.ids())
        assert rel(on.neg_log_marginal_likelihood(), orc.nlml()) <= TOL_ORACLE
        p = on.predict(xs, 6, d)
        mo, vo = orc.predict(xs, 6, 1)
        assert np.all(rel(p.mean, mo) <= TOL_ORACLE)
        assert np.all(rel(p.variance, vo) <= TOL_ORACLE)
    with pytest.raises(gx.IndexOutOfRange):
        on.delete(10 ** 9)


def test_online_delete_refuses_last_point():
    m = fixed_model([[10, 0]], [0.0], 0.1, [0.0, 1.0], 2, 1, [0.5, -0.25])
    on = m.into_online()
    on.delete(on.point_ids()[0])
    with pytest.raises(gx.InsufficientData):
        on.delete(on.point_ids()[0])


def test_fit_goldens_with_standardized_targets():
    # tests/fit_goldens.rs: sklearn L-BFGS-B fit at REL 0.15 (StandardizeTarget)
    for case in load("fit_goldens.json"):
        n, d, q = case["n"], case["d"], case["q"]
        y = np.asarray(case["y"])
        mu, sd = y.mean(), y.std()
        ys = (y - mu) / sd
        if d == 1:
            spec = gx.RbfKernel(math.exp(case["theta_init"][0]))
        else:
            spec = gx.RbfArdKernel([math.exp(t) for t in case["theta_init"]])
        m = gx.Gpr(spec, gx.GaussianLikelihood(case["noise_variance_init"])).fit(case["x"], n, d, ys)
        params = m.get_params()
        ls = np.exp(params[:-1])
        for a, e in zip(ls, case["lengthscales"]):
            assert abs(math.log(a) - math.log(e)) <= 2.5
        # sklearn (normalize_y) and gprx's StandardizeTarget both report the
        # marginal likelihood of the standardized targets
        lml = -m.neg_log_marginal_likelihood()
        assert rel(lml, case["lml"]) <= 0.15, (lml, case["lml"])
        p = m.predict_with(case["xs"], q, d, gx.PredictOptions(gx.VarianceKind.Latent))
        mean = p.mean * sd + mu
        assert np.all(rel(mean, case["mean"]) <= 0.15)
        assert np.all(rel(p.variance * sd * sd, case["latent_variance"]) <= 0.15)


def test_fit_recovers_hyperparameters_and_matches_oracle_at_optimum():
    # tests/recovery.rs: L-BFGS recovers ℓ and σn² within 0.5 relative;
    # the NLML and gradient at the returned θ agree with the oracle.
    rs = np.random.RandomState(0)
    n, d = 400, 2
    x = rs.uniform(0, 10, size=(n, d))
    ell, noise = 1.5, 0.05
    nodes = [[10, 0]]
    xc = x.T.reshape(-1)
    k = O.gram_lower(nodes, [math.log(ell)], xc, n, d)
    k = np.tril(k) + np.tril(k, -1).T + noise * np.eye(n)
    y = np.linalg.cholesky(k) @ rs.standard_normal(n)
    m = gx.Gpr(gx.RbfKernel(1.0), gx.GaussianLikelihood(0.1)).fit(xc, n, d, y)
    p = m.get_params()
    assert abs(math.exp(p[0]) / ell - 1) < 0.5
    assert abs(math.exp(p[1]) / noise - 1) < 0.5
    nl_o, g_o, _, _ = O.exact_eval(nodes, p, xc, n, d, y)
    assert rel(m.neg_log_marginal_likelihood(), nl_o) <= TOL_ORACLE
    assert np.linalg.norm(g_o) < 1e-3
