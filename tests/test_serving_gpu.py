"""The serving loop (gprx_server_*): results are the same alone and in a mix,
small fits of several models share a batched launch, small predicts of one
or several models share a grouped launch, and the HBM budget evicts idle
models.

Each model's requests run in submission order on the model's own stream, so
a model's fit, predictions and online steps must give the same values
whether the server runs nothing else or a stream of other fits, predicts and
online steps at the same time (checked bit for bit; the tolerance stated by
the serving form is 1e-12 relative and the results meet it exactly).
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu


def data(n, d, seed):
    rs = np.random.RandomState(seed)
    x = rs.standard_normal((n, d))
    y = np.sin(x.sum(1)) + 0.05 * rs.standard_normal(n)
    return x.T.reshape(-1).copy(), y


def spec(d):
    return gx.RbfArdKernel([1.0] * d)


LB = gx.Lbfgs(max_iterations=25)


def script(srv, model, d, seed):
    """Predict, add 3 points, predict, remove 2 of the original points,
    predict; returns the outputs."""
    rs = np.random.RandomState(seed)
    q = 40
    xs = rs.standard_normal(q * d)
    out = []
    rid, m1, v1 = srv.submit_predict(model, xs, q)
    assert srv.wait(rid)[0] == 0
    out += [m1.copy(), v1.copy()]
    xa = rs.standard_normal(3 * d)
    ya = rs.standard_normal(3)
    rid, ids = srv.submit_add(model, xa, ya, 3)
    assert srv.wait(rid)[0] == 0
    out.append(ids.copy())
    rid, m2, v2 = srv.submit_predict(model, xs, q)
    assert srv.wait(rid)[0] == 0
    out += [m2.copy(), v2.copy()]
    rid = srv.submit_remove(model, [5, 11])
    assert srv.wait(rid)[0] == 0
    rid, m3, v3 = srv.submit_predict(model, xs, q)
    assert srv.wait(rid)[0] == 0
    out += [m3.copy(), v3.copy()]
    return out


def test_results_same_alone_and_in_the_mix():
    d = 4
    x, y = data(600, d, 1)
    # alone
    srv = gx.Server(workers=4)
    mid = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.05), x, 600, d, y, optimizer=LB)
    assert srv.wait(mid)[0] == 0
    alone = script(srv, mid, d, seed=7)
    srv.close()
    # in a mix: other fits, predictions and online steps in flight
    srv = gx.Server(workers=6)
    others = []
    for k, n in enumerate((300, 900, 1500, 450)):
        xo, yo = data(n, d, 20 + k)
        others.append((srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), xo, n, d, yo, optimizer=LB), n))
    mid = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.05), x, 600, d, y, optimizer=LB)
    rs = np.random.RandomState(3)
    pending = []
    for om, n in others:
        for _ in range(3):
            q = int(rs.randint(1, 500))
            pending.append(srv.submit_predict(om, rs.standard_normal(q * d), q)[0])
        pending.append(srv.submit_add(om, rs.standard_normal(2 * d), rs.standard_normal(2), 2)[0])
    assert srv.wait(mid)[0] == 0
    mixed = script(srv, mid, d, seed=7)
    for rid in pending:
        assert srv.wait(rid)[0] == 0
    for om, _ in others:
        assert srv.wait(om)[0] == 0
    srv.close()
    assert len(alone) == len(mixed)
    for a, b in zip(alone, mixed):
        assert np.array_equal(a, b)
    # and the direct API's fit (the server's small predicts run the grouped
    # kernel, which sums in another order than gprx_exact_predict)
    f = gx.Gpr(spec(d), gx.GaussianLikelihood(0.05), optimizer=LB).fit(x, 600, d, y)
    rs = np.random.RandomState(7)
    xs = rs.standard_normal(40 * d)
    p = f.predict(xs, 40, d)
    assert np.all(O.rel_err(p.mean, alone[0]) <= 1e-10) and np.all(O.rel_err(p.variance, alone[1]) <= 1e-10)


def test_consecutive_predicts_share_a_launch():
    d = 3
    x, y = data(800, d, 5)
    srv = gx.Server(workers=2)
    mid = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), x, 800, d, y, optimizer=LB)
    rs = np.random.RandomState(1)
    reqs = []
    for q in (5, 17, 1, 64):
        xs = rs.standard_normal(q * d)
        reqs.append((srv.submit_predict(mid, xs, q), xs, q))
    infos = [srv.wait(r[0][0])[1] for r in reqs]
    assert srv.wait(mid)[0] == 0
    assert all(i["merged"] == 4 for i in infos)
    # each output equals its own single prediction
    for (rid, mean, var), xs, q in reqs:
        r2, m2, v2 = srv.submit_predict(mid, xs, q)
        st, info = srv.wait(r2)
        assert st == 0 and info["merged"] == 1
        assert np.array_equal(mean, m2) and np.array_equal(var, v2)
    srv.close()


def test_hbm_budget_evicts_the_least_recently_used_model():
    d = 2
    srv = gx.Server(workers=1, hbm_budget_bytes=60 << 20)  # room for two models of n = 1200 (26 MB each)
    ids = []
    for k in range(3):
        x, y = data(1200, d, 40 + k)
        mid = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), x, 1200, d, y, optimizer=gx.Fixed())
        assert srv.wait(mid)[0] == 0
        ids.append(mid)
    st = srv.stats()
    assert st["resident_models"] == 2 and st["used_bytes"] <= 60 << 20
    rid, _, _ = srv.submit_predict(ids[0], np.zeros(d), 1)
    assert srv.wait(rid)[0] == gx.api.L.INVALID_CONFIG  # evicted
    rid, _, _ = srv.submit_predict(ids[2], np.zeros(d), 1)
    assert srv.wait(rid)[0] == 0
    srv.close()


def test_small_fits_share_one_batched_launch_and_match_alone():
    # fits of n ≤ 512 always run on the batched evaluator; fits waiting at the
    # heads of several models' queues share one launch, and each model's
    # results are bit for bit those of the same fit alone
    d = 4
    lb = gx.Lbfgs(max_iterations=25)
    sizes = (120, 300, 64, 500)
    sets = [data(n, d, 60 + k) for k, n in enumerate(sizes)]
    xs = np.random.RandomState(9).standard_normal(30 * d)
    alone = []
    for (x, y), n in zip(sets, sizes):
        srv = gx.Server(workers=2)
        mid = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), x, n, d, y, optimizer=lb)
        st, info = srv.wait(mid)
        assert st == 0 and info["merged"] == 1
        rid, m, v = srv.submit_predict(mid, xs, 30)
        assert srv.wait(rid)[0] == 0
        alone.append((m.copy(), v.copy()))
        assert srv.stats()["merged_fit_launches"] == 0
        srv.close()
    # together: one worker busy with a large fit while the small ones queue
    srv = gx.Server(workers=1)
    xb, yb = data(1500, d, 99)
    big = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), xb, 1500, d, yb, optimizer=lb)
    mids = [srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), x, n, d, y, optimizer=lb)
            for (x, y), n in zip(sets, sizes)]
    assert srv.wait(big)[0] == 0
    for k, mid in enumerate(mids):
        st, info = srv.wait(mid)
        assert st == 0 and info["merged"] == len(sizes)
        rid, m, v = srv.submit_predict(mid, xs, 30)
        assert srv.wait(rid)[0] == 0
        assert np.array_equal(m, alone[k][0]) and np.array_equal(v, alone[k][1])
    assert srv.stats()["merged_fit_launches"] == 1
    srv.close()
    # the plumbing: each model predicts from the batched fit's θ (the oracle's
    # prediction at the θ GprBatch.fit reaches for the same problem)
    for k, ((x, y), n) in enumerate(zip(sets, sizes)):
        theta0 = np.array(spec(d).get_params() + [math.log(0.1)])
        r = gx.GprBatch(spec(d), [x], [y], d).fit(theta0[None, :], lb)
        mo, vo = O.exact_predict([[11, d]], r.params[0], x, n, d, y, xs, 30, 1)
        assert np.all(O.rel_err(alone[k][0], mo) <= 1e-10) and np.all(O.rel_err(alone[k][1], vo) <= 1e-10)


def test_small_predicts_of_several_models_share_a_launch():
    d = 3
    srv = gx.Server(workers=1)
    mids = []
    for k, n in enumerate((700, 300, 900)):
        x, y = data(n, d, 70 + k)
        mids.append(srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), x, n, d, y, optimizer=gx.Fixed()))
    for mid in mids:
        assert srv.wait(mid)[0] == 0
    # a large fit keeps the one worker busy while predicts of the three models queue
    xb, yb = data(1500, d, 99)
    big = srv.submit_fit(spec(d), gx.GaussianLikelihood(0.1), xb, 1500, d, yb, optimizer=gx.Fixed())
    rs = np.random.RandomState(2)
    reqs = []
    for mid in mids + mids:
        q = int(rs.randint(1, 60))
        xs = rs.standard_normal(q * d)
        reqs.append((mid, srv.submit_predict(mid, xs, q), xs, q))
    assert srv.wait(big)[0] == 0
    for mid, (rid, mean, var), xs, q in reqs:
        st, info = srv.wait(rid)
        assert st == 0 and info["merged"] == len(reqs)
    assert srv.stats()["merged_launches"] >= 1
    # each equals the same request alone
    for mid, (rid, mean, var), xs, q in reqs:
        r2, m2, v2 = srv.submit_predict(mid, xs, q)
        st, info = srv.wait(r2)
        assert st == 0 and info["merged"] == 1
        assert np.array_equal(mean, m2) and np.array_equal(var, v2)
    srv.close()
