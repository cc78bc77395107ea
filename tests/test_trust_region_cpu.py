"""The trust-region method (gprx_b200/csrc/trust_region.h, compiled for the
host, no device) on the reference's own optimizer tests
(src/optimizer/trust_region.rs:307-531): a quadratic bowl, √(1 + x²) from
starts where the plain Newton step diverges (points beyond |x| = 50 cannot be
evaluated), −cos x from a point of negative curvature, a shifted bowl; a
start that cannot be evaluated is an error; and the Hessian chained through
the logit map against finite differences."""

import json
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-6


def run_driver():
    exe = os.path.join(tempfile.mkdtemp(), "trust_region_driver")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-o", exe,
                           os.path.join(ROOT, "tests", "cpp", "trust_region_driver.cpp")])
    out = subprocess.check_output([exe], text=True)
    return {d["case"]: d for d in (json.loads(l) for l in out.splitlines() if l.strip())}


RES = None


def res():
    global RES
    if RES is None:
        RES = run_driver()
    return RES


def test_minimizes_quadratic_bowl():
    r = res()["bowl"]
    assert r["ok"] == 1 and abs(r["x"][0]) <= TOL and abs(r["x"][1]) <= TOL and r["f"] < 1e-12


def test_converges_where_the_plain_newton_step_diverges():
    for start in ("1.5", "2", "4", "-3"):
        r = res()["sqrt1p_" + start]
        assert r["ok"] == 1 and abs(r["x"][0]) <= 1e-6, r


def test_descends_when_the_hessian_is_not_positive_definite():
    r = res()["negative_curvature"]
    assert r["ok"] == 1 and r["f"] < -0.999


def test_shifted_bowl():
    r = res()["shifted_bowl"]
    assert abs(r["x"][0] - 0.3) <= TOL and abs(r["x"][1] + 0.2) <= TOL


def test_unevaluable_start_is_an_error():
    r = res()["bad_start"]
    assert r["ok"] == 0 and r["evals"] == 1


def test_logit_hessian_chain_rule():
    assert res()["logit_hessian"]["err"] < 1e-6


def test_rejects_bad_radii():
    # src/optimizer/trust_region.rs:459-464
    import gprx_b200 as gx
    import pytest

    for a in [(0.0, 1.0), (2.0, 1.0), (1.0, float("inf"))]:
        with pytest.raises(gx.InvalidConfig):
            gx.TrustRegion().with_radii(*a)
    o = gx.TrustRegion()._c()
    assert (o.max_iterations, o.initial_radius, o.max_radius) == (100, 1.0, 100.0)
    assert o.tolerance == 2.220446049250313e-16 ** 0.5


def test_sgpr_refuses_trust_region():
    import gprx_b200 as gx
    import pytest

    s = gx.Sgpr(gx.RbfKernel(1.0), gx.GaussianLikelihood(0.1)).with_optimizer(gx.TrustRegion())
    with pytest.raises(gx.InvalidConfig):
        s.fit([0.0, 1.0], 2, 1, [0.0, 1.0], [0.5], 1)
