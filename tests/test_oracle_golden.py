"""Pins the CPU oracle against the reference's own goldens (CPU only).

The oracle (oracle/gprx_oracle.cpp) is the parity reference for the CUDA
backend; these tests are what make it trustworthy.  Tolerances are the
reference's: 1e-8 for the sklearn / libgp / GPyTorch goldens
(tests/goldens.rs:15, tests/online_libgp.rs, tests/sparse_gpytorch.rs),
measured as |a − e| / max(|e|, 1) (tests/common/check.rs:8-10).
"""

import json
import os

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-8


def load(name):
    with open(os.path.join(GOLD, name)) as fh:
        return json.load(fh)


def test_rng_sequence_is_pinned():
    pins = load("rng_pins.json")["seeds"]
    for seed, vals in pins.items():
        assert O.rng_seq(int(seed), 4) == [int(v) for v in vals]


def _exact_cases():
    return load("exact_goldens.json") + load("sklearn_goldens.json")


@pytest.mark.parametrize("case", _exact_cases(), ids=lambda c: c["name"])
def test_exact_golden(case):
    n, d, q = case["n"], case["d"], case["q"]
    params = case["theta"] + [np.log(case["noise_variance"])]
    nlml, grad, _, _ = O.exact_eval(case["nodes"], params, case["x"], n, d, case["y"])
    assert O.rel_err(nlml, case["nlml"]) <= TOL
    if case["grad_kernel"] is not None:
        assert np.all(O.rel_err(grad[:-1], case["grad_kernel"]) <= TOL), (grad, case["grad_kernel"])
    if case["grad_noise"] is not None:
        assert O.rel_err(grad[-1], case["grad_noise"]) <= TOL
    for kind, key in ((0, "latent_variance"), (1, "observation_variance")):
        mean, var = O.exact_predict(case["nodes"], params, case["x"], n, d, case["y"], case["xs"], q, kind)
        assert np.all(O.rel_err(mean, case["mean"]) <= TOL)
        assert np.all(O.rel_err(var, case[key]) <= TOL), (var, case[key])


def test_exact_gradient_matches_finite_difference():
    # value_and_gradient_matches_nlml_and_finite_difference (src/gpr/tests.rs:1351)
    rs = np.random.RandomState(3)
    n, d = 30, 3
    x = rs.uniform(0, 3, size=n * d)
    y = rs.standard_normal(n)
    # (a periodic leaf on a Euclidean distance is not positive definite for
    # d > 1 in general, so that tree gets a large noise)
    trees = [
        ([[2, 2], [12, 0], [11, 3]], [0.3, -0.2, 0.1, 0.4], 0.3),
        ([[1, 2], [10, 0], [13, 0]], [0.1, 0.5, 0.7], 2.0),
        ([[1, 2], [2, 2], [12, 0], [10, 0], [10, 0]], [0.2, -0.1, 0.6], 0.3),
    ]
    for nodes, theta, noise in trees:
        params = np.array(theta + [np.log(noise)])
        _, g, _, _ = O.exact_eval(nodes, params, x, n, d, y)
        h = 1e-5
        for i in range(len(params)):
            pp, pm = params.copy(), params.copy()
            pp[i] += h
            pm[i] -= h
            fp = O.exact_eval(nodes, pp, x, n, d, y, grad=False)[0]
            fm = O.exact_eval(nodes, pm, x, n, d, y, grad=False)[0]
            assert abs((fp - fm) / (2 * h) - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


@pytest.mark.parametrize("case", load("online_goldens.json"), ids=lambda c: c["name"])
def test_online_insert_golden(case):
    n, d, q, s = case["n"], case["d"], case["q"], case["start_n"]
    x = np.asarray(case["x"]).reshape(d, n)
    y = np.asarray(case["y"])
    params = case["theta"] + [np.log(case["noise_variance"])]
    on = O.Online(case["nodes"], params, x[:, :s].reshape(-1), s, d, y[:s])
    for k, step in enumerate(case["steps"]):
        if k > 0:
            on.insert(x[:, s + k - 1], y[s + k - 1])
        assert on.n == step["n"]
        mean, var = on.predict(case["xs"], q, 1)
        assert np.all(O.rel_err(mean, step["mean"]) <= TOL)
        assert np.all(O.rel_err(var, step["observation_variance"]) <= TOL)
        assert O.rel_err(on.nlml(), step["neg_log_marginal_likelihood"]) <= TOL


def test_online_delete_matches_fresh_factor():
    # tests/online_ops.rs:110-197: random insert/delete sequences against a fresh factor at 1e-12
    rs = np.random.RandomState(11)
    d = 2
    nodes = [[11, 2]]
    params = [np.log(0.9), np.log(1.4), np.log(0.05)]
    pts = rs.uniform(0, 4, size=(60, d))
    ys = np.sin(pts.sum(1))
    live = list(range(12))
    on = O.Online(nodes, params, pts[live].T.reshape(-1), len(live), d, ys[live])
    nxt = 12
    xs = rs.uniform(0, 4, size=(5, d))
    for step in range(30):
        if rs.rand() < 0.5 and nxt < 60:
            on.insert(pts[nxt], ys[nxt])
            live.append(nxt)
            nxt += 1
        else:
            slot = rs.randint(len(live))
            on.delete(on.ids()[slot])
            live.pop(slot)
        fresh = O.Online(nodes, params, pts[live].T.reshape(-1), len(live), d, ys[live])
        assert O.rel_err(on.nlml(), fresh.nlml()) <= 1e-12
        m1, v1 = on.predict(xs.T.reshape(-1), 5, 1)
        m2, v2 = fresh.predict(xs.T.reshape(-1), 5, 1)
        assert np.all(O.rel_err(m1, m2) <= 1e-11)
        assert np.all(O.rel_err(v1, v2) <= 1e-11)


@pytest.mark.parametrize("case", load("sgpr_goldens.json"), ids=lambda c: c["name"])
def test_sgpr_golden(case):
    n, d, q, m = case["n"], case["d"], case["q"], case["m"]
    params = case["theta"] + [np.log(case["noise_variance"])]
    s = O.Sgpr(case["nodes"], params, case["x"], n, d, case["y"], case["z"], m)
    assert O.rel_err(s.nlml(), case["nlml"]) <= TOL
    for kind, key in ((0, "latent_variance"), (1, "observation_variance")):
        mean, var = s.predict(case["xs"], q, kind)
        assert np.all(O.rel_err(mean, case["mean"]) <= TOL)
        assert np.all(O.rel_err(var, case[key]) <= TOL)


def test_sgpr_gradient_matches_finite_difference():
    rs = np.random.RandomState(5)
    n, m = 80, 12
    # (the periodic tree runs in 1-D, where a periodic leaf is positive definite)
    for d, nodes, theta in ((2, [[11, 2]], [np.log(0.4), np.log(0.7)]),
                            (2, [[2, 2], [12, 0], [10, 0]], [np.log(1.5), np.log(0.3)]),
                            (1, [[1, 2], [10, 0], [13, 0]], [np.log(0.2), np.log(0.5), np.log(0.45)])):
        x = rs.uniform(0, 1, size=n * d)
        y = np.sin(6 * x[:n]) + 0.1 * rs.standard_normal(n)
        z = x.reshape(d, n)[:, :m].reshape(-1)
        params = np.array(theta + [np.log(0.05)])
        g = O.Sgpr(nodes, params, x, n, d, y, z, m).grad()
        h = 1e-5
        for i in range(len(params)):
            pp, pm = params.copy(), params.copy()
            pp[i] += h
            pm[i] -= h
            fp = O.Sgpr(nodes, pp, x, n, d, y, z, m).nlml()
            fm = O.Sgpr(nodes, pm, x, n, d, y, z, m).nlml()
            assert abs((fp - fm) / (2 * h) - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, g[i], (fp - fm) / (2 * h))


@pytest.mark.parametrize("case", load("online_sgpr_goldens.json"), ids=lambda c: c["name"])
def test_online_sgpr_golden(case):
    n, d, q = case["n"], case["d"], case["q"]
    x = np.asarray(case["x"]).reshape(d, n)
    y = np.asarray(case["y"])
    zall = np.asarray(case["z"]).reshape(d, case["m"])
    s0, m0 = case["start_n"], case["start_m"]
    params = case["theta"] + [np.log(case["noise_variance"])]
    z = [zall[:, i] for i in range(m0)]
    sg = O.Sgpr(case["nodes"], params, x[:, :s0].reshape(-1), s0, d, y[:s0],
                np.array(z).T.reshape(-1), m0)
    ids = list(range(s0))
    for k, step in enumerate(case["steps"]):
        if k > 0:
            op = case["ops"][k - 1]
            if op["kind"] == "insert":
                ids.append(sg.insert(x[:, op["pop_index"]], y[op["pop_index"]]))
            elif op["kind"] == "delete":
                sg.delete(ids.pop(op["slot"]))
            elif op["kind"] == "insert_inducing":
                z.append(zall[:, op["pop_index"]])
                sg.set_inducing(np.array(z).T.reshape(-1), len(z))
            else:
                z.pop(op["slot"])
                sg.set_inducing(np.array(z).T.reshape(-1), len(z))
        assert sg.n == step["n"] and len(z) == step["m"]
        assert O.rel_err(sg.nlml(), step["neg_log_marginal_likelihood"]) <= TOL, k
        for kind, key in ((0, "latent_variance"), (1, "observation_variance")):
            mean, var = sg.predict(case["xs"], q, kind)
            assert np.all(O.rel_err(mean, step["mean"]) <= TOL), k
            assert np.all(O.rel_err(var, step[key]) <= TOL), k
