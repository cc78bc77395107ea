"""GPU parity of the batched exact-GPR path (gprx_batch_*) through the C ABI.

Every problem of a batch is checked against the CPU oracle's single-model
evaluation on the same inputs: |a − e| / max(|e|, 1) ≤ 1e-10 for NLML and
gradient (FP64 end to end).  A problem's result does not depend on the batch
it runs in (one CTA computes it in a fixed order), so the same problem alone
and in a mixed batch must agree bit for bit.
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

TOL = 1e-10

# (d, nodes, kernel spec builder from log θ)
RBF_PER = (3, [[1, 2], [10, 0], [13, 0]],
           lambda t: gx.RbfKernel(math.exp(t[0])) + gx.PeriodicKernel(math.exp(t[1]), math.exp(t[2])))
CONST_ARD = (3, [[2, 2], [12, 0], [11, 3]],
             lambda t: gx.ConstantKernel(math.exp(t[0])) * gx.RbfArdKernel([math.exp(v) for v in t[1:4]]))
RBF2 = (2, [[10, 0]], lambda t: gx.RbfKernel(math.exp(t[0])))
RBF_PER1 = (1, [[1, 2], [10, 0], [13, 0]],
            lambda t: gx.RbfKernel(math.exp(t[0])) + gx.PeriodicKernel(math.exp(t[1]), math.exp(t[2])))


def problems(sizes, d, seed, box=5.0):
    rs = np.random.RandomState(seed)
    xs, ys = [], []
    for n in sizes:
        x = rs.uniform(0, box, size=(n, d))
        y = np.sin(x[:, 0]) + 0.5 * np.cos(x[:, -1]) + 0.1 * rs.standard_normal(n)
        xs.append(x.T.reshape(-1))
        ys.append(y)
    return xs, ys


def random_params(count, kind, rs):
    d, nodes, _ = kind
    out = []
    for _ in range(count):
        if kind is RBF_PER:
            # the periodic kernel of a Euclidean distance is indefinite in 3-d
            # unless the period is long against the domain
            t = [math.log(rs.uniform(0.5, 2.0)), math.log(rs.uniform(0.7, 2.0)), math.log(rs.uniform(10.0, 20.0))]
        elif kind is RBF_PER1:
            t = [math.log(rs.uniform(0.5, 2.0)), math.log(rs.uniform(0.7, 2.0)), math.log(rs.uniform(0.5, 2.0))]
        elif kind is CONST_ARD:
            t = [math.log(rs.uniform(0.5, 2.0))] + [math.log(rs.uniform(0.5, 3.0)) for _ in range(3)]
        else:
            t = [math.log(rs.uniform(0.3, 2.0))]
        out.append(t + [math.log(rs.uniform(0.05, 0.3))])
    return np.array(out)


SIZES = [1, 2, 7, 31, 32, 33, 64, 100, 127, 128, 129, 200, 255, 256, 257, 300, 383, 385, 511, 640, 1024]


@pytest.mark.parametrize("kind", [RBF_PER, RBF_PER1, CONST_ARD, RBF2],
                         ids=["rbf+periodic", "rbf+periodic-1d", "const*ard", "rbf"])
def test_batch_eval_matches_oracle(kind):
    d, nodes, spec = kind
    rs = np.random.RandomState(3)
    sizes = list(SIZES)
    rs.shuffle(sizes)
    xs, ys = problems(sizes, d, 11)
    params = random_params(len(sizes), kind, rs)
    b = gx.GprBatch(spec(params[0][:-1]), xs, ys, d)
    nl, g, st = b.value_and_gradient(params)
    ok = 0
    for i, n in enumerate(sizes):
        try:
            nl_o, g_o, _, _ = O.exact_eval(nodes, params[i], xs[i], n, d, ys[i])
        except O.OracleError as e:
            assert st[i] == e.status, (n, st[i], e.status)
            continue
        assert st[i] == 0, (n, st[i])
        ok += 1
        assert O.rel_err(nl[i], nl_o) <= TOL, (n, nl[i], nl_o)
        assert np.all(O.rel_err(g[i], g_o) <= TOL), (n, g[i], g_o)
    assert ok == len(sizes)


def test_batch_problem_result_independent_of_batch():
    d, nodes, spec = RBF_PER
    rs = np.random.RandomState(5)
    sizes = [int(v) for v in np.exp(rs.uniform(math.log(32), math.log(700), size=40))]
    xs, ys = problems(sizes, d, 12)
    params = random_params(len(sizes), RBF_PER, rs)
    b = gx.GprBatch(spec(params[0][:-1]), xs, ys, d)
    nl, g, st = b.value_and_gradient(params)
    assert np.all(st == 0)
    for i in (0, 7, 23):
        solo = gx.GprBatch(spec(params[i][:-1]), [xs[i]], [ys[i]], d)
        nl1, g1, st1 = solo.value_and_gradient(params[i:i + 1])
        assert st1[0] == 0
        assert nl1[0] == nl[i] and np.array_equal(g1[0], g[i])
    # a second evaluation of the same batch is bit-identical
    nl2, g2, _ = b.value_and_gradient(params)
    assert np.array_equal(nl, nl2) and np.array_equal(g, g2)


def test_batch_failed_problems_do_not_disturb_the_others():
    d, nodes, spec = RBF_PER
    rs = np.random.RandomState(6)
    sizes = [50, 120, 80, 300, 64]
    xs, ys = problems(sizes, d, 13)
    params = random_params(len(sizes), RBF_PER, rs)
    # problem 1: a length scale outside (1e-5, 1e5); problem 4: a non-finite θ
    params[1][0] = math.log(1e6)
    params[4][2] = float("nan")
    b = gx.GprBatch(spec(params[0][:-1]), xs, ys, d)
    nl, g, st = b.value_and_gradient(params)
    assert st[1] == gx.api.L.INVALID_HYPERPARAMETER
    assert st[4] == gx.api.L.INVALID_HYPERPARAMETER
    for i in (0, 2, 3):
        assert st[i] == 0
        nl_o, g_o, _, _ = O.exact_eval(nodes, params[i], xs[i], sizes[i], d, ys[i])
        assert O.rel_err(nl[i], nl_o) <= TOL
        assert np.all(O.rel_err(g[i], g_o) <= TOL)


def test_batch_cholesky_failure_is_reported_per_problem():
    # a short-period periodic kernel in 3-d is not positive definite and the
    # noise sits at the interval's floor: problems whose factor fails report
    # CHOLESKY_FAILED exactly when the oracle's does
    d, nodes, spec = RBF_PER
    rs = np.random.RandomState(8)
    sizes = [40, 60, 90, 150]
    xs, ys = [], []
    for n in sizes:
        x = rs.uniform(0, 5, size=(n, d))
        xs.append(x.T.reshape(-1))
        ys.append(rs.standard_normal(n))
    params = np.array([[math.log(2.0), math.log(0.05), math.log(0.3), math.log(1.1e-5)]] * len(sizes))
    b = gx.GprBatch(spec(params[0][:-1]), xs, ys, d)
    nl, g, st = b.value_and_gradient(params)
    for i, n in enumerate(sizes):
        try:
            nl_o, g_o, _, _ = O.exact_eval(nodes, params[i], xs[i], n, d, ys[i])
        except O.OracleError as e:
            assert e.status == gx.api.L.CHOLESKY_FAILED
            assert st[i] == gx.api.L.CHOLESKY_FAILED
            continue
        assert st[i] == 0 and np.isfinite(nl[i])


def gp_draws(sizes, d, seed, theta):
    """y from the GP prior at θ (oracle Gram matrix) plus noise."""
    rs = np.random.RandomState(seed)
    _, nodes, _ = RBF_PER
    xs, ys = [], []
    for n in sizes:
        x = rs.uniform(0, 5, size=(n, d)).T.reshape(-1)
        K = O.gram_lower(nodes, theta[:-1], x, n, d)
        K = np.tril(K) + np.tril(K, -1).T + (math.exp(theta[-1]) + 1e-10) * np.eye(n)
        y = np.linalg.cholesky(K) @ rs.standard_normal(n)
        xs.append(x)
        ys.append(y)
    return xs, ys


def test_batch_fit_reaches_oracle_stationary_points():
    d, nodes, spec = RBF_PER
    theta_true = np.array([math.log(1.0), math.log(1.0), math.log(15.0), math.log(0.1)])
    rs = np.random.RandomState(21)
    sizes = [int(v) for v in np.exp(rs.uniform(math.log(32), math.log(400), size=24))]
    xs, ys = gp_draws(sizes, d, 22, theta_true)
    start = np.tile([math.log(1.0), math.log(1.0), math.log(12.0), math.log(0.1)], (len(sizes), 1))
    b = gx.GprBatch(spec(start[0][:-1]), xs, ys, d)
    nl0, _, st0 = b.value_and_gradient(start)
    assert np.all(st0 == 0)
    res = b.fit(start)
    assert np.all(res.status == 0), res.status
    assert np.all(res.nlml <= nl0 + 1e-12)
    lo, hi = math.log(1e-5), math.log(1e5)
    for i, n in enumerate(sizes):
        # the reported value is an evaluation at the returned θ
        nl_o, g_o, _, _ = O.exact_eval(nodes, res.params[i], xs[i], n, d, ys[i])
        assert O.rel_err(res.nlml[i], nl_o) <= TOL
        if res.converged[i]:
            # ∇ in z space of the logit map, as the optimizer sees it
            u = (res.params[i] - lo) / (hi - lo)
            jac = (hi - lo) * u * (1 - u) / ((hi - lo) / 4)
            assert np.linalg.norm(g_o * jac) < 1e-5, (i, g_o * jac)


def test_batch_fit_matches_single_model_fit():
    # a unimodal problem family: the batched optimizer and the single-model
    # optimizer (same algorithm, same starting point) reach the same optimum
    d, nodes, spec = RBF2
    rs = np.random.RandomState(31)
    sizes = [40, 90, 160, 250]
    xs, ys = problems(sizes, d, 32)
    start = np.tile([math.log(1.0), math.log(0.5)], (len(sizes), 1))
    b = gx.GprBatch(spec(start[0][:-1]), xs, ys, d)
    res = b.fit(start)
    assert np.all(res.status == 0)
    for i, n in enumerate(sizes):
        m = gx.Gpr(gx.RbfKernel(1.0), gx.GaussianLikelihood(0.5)).fit(xs[i], n, d, ys[i])
        nl = m.neg_log_marginal_likelihood()
        assert O.rel_err(res.nlml[i], nl) <= 1e-8, (i, res.nlml[i], nl)
        assert np.all(np.abs(res.params[i] - np.array(m.get_params())) <= 1e-4), (res.params[i], m.get_params())


@pytest.mark.parametrize("kind", [RBF_PER, CONST_ARD], ids=["rbf+periodic", "const*ard"])
def test_batch_every_tile_shape_gives_the_same_bits(kind):
    # the in-CTA GEMMs sum every output's k terms in the same order whatever
    # the tile shape, so the schedule changes only the time
    d, nodes, spec = kind
    rs = np.random.RandomState(21)
    sizes = list(SIZES)
    rs.shuffle(sizes)
    xs, ys = problems(sizes, d, 13)
    params = random_params(len(sizes), kind, rs)
    b = gx.GprBatch(spec(params[0][:-1]), xs, ys, d)
    out = []
    for k in range(len(gx.GprBatch.TILE_SHAPES)):
        b.set_schedule([k] * gx.GprBatch.SIZE_CLASSES)
        out.append(b.value_and_gradient(params))
    for nl, g, st in out[1:]:
        assert np.array_equal(st, out[0][2])
        assert np.array_equal(nl, out[0][0]) and np.array_equal(g, out[0][1])
    nl, g, st = out[-1]
    for i in (0, 5, 11):
        nl_o, g_o, _, _ = O.exact_eval(nodes, params[i], xs[i], sizes[i], d, ys[i])
        assert O.rel_err(nl[i], nl_o) <= TOL and np.all(O.rel_err(g[i], g_o) <= TOL)


def test_batch_autotune_picks_the_fastest_shape_per_class():
    d, nodes, spec = RBF_PER
    rs = np.random.RandomState(22)
    sizes = [int(v) for v in np.exp(rs.uniform(math.log(20), math.log(1000), size=300))]
    xs, ys = problems(sizes, d, 14)
    params = random_params(len(sizes), RBF_PER, rs)
    b = gx.GprBatch(spec(params[0][:-1]), xs, ys, d)
    _, _, tuned = b.schedule()
    assert not tuned
    t, ms, tuned = b.autotune(params)
    assert tuned
    present = {min(max(0, int(math.ceil(math.log2(max(n, 1) / 64.0)))), 7) for n in sizes}
    for c in range(gx.GprBatch.SIZE_CLASSES):
        if c in present:
            assert np.all(ms[c] > 0) and t[c] == int(np.argmin(ms[c])), (c, t[c], ms[c])
        else:
            assert np.all(ms[c] == 0)
    nl, g, st = b.value_and_gradient(params)
    assert np.all(st == 0)
    b.set_schedule([0] * gx.GprBatch.SIZE_CLASSES)
    nl0, g0, _ = b.value_and_gradient(params)
    assert np.array_equal(nl, nl0) and np.array_equal(g, g0)
    # a fit under the tuned schedule ends where the fixed one does
    b2 = gx.GprBatch(spec(params[0][:-1]), xs[:40], ys[:40], d)
    f1 = b2.fit(params[:40], gx.Lbfgs(max_iterations=15))
    b2.set_schedule([3] * gx.GprBatch.SIZE_CLASSES)
    f2 = b2.fit(params[:40], gx.Lbfgs(max_iterations=15))
    assert np.array_equal(f1.params, f2.params)
