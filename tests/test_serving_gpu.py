"""The serving loop (gprx_server_*): results are the same alone and in a mix,
consecutive predicts share a launch, and the HBM budget evicts idle models.

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
    # and the same as the direct API
    f = gx.Gpr(spec(d), gx.GaussianLikelihood(0.05), optimizer=LB).fit(x, 600, d, y)
    rs = np.random.RandomState(7)
    xs = rs.standard_normal(40 * d)
    p = f.predict(xs, 40, d)
    assert np.array_equal(p.mean, alone[0]) and np.array_equal(p.variance, alone[1])


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
        assert np.allclose(mean, m2, rtol=1e-12, atol=1e-14) and np.allclose(var, v2, rtol=1e-12, atol=1e-14)
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
