"""The L-BFGS / Moré–Thuente / logit map (gprx_b200/csrc/lbfgs.h) on analytic
objectives, compiled for the host and run on the CPU (no device involved)."""

import json
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_driver():
    exe = os.path.join(tempfile.mkdtemp(), "lbfgs_driver")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-o", exe,
                           os.path.join(ROOT, "tests", "cpp", "lbfgs_driver.cpp")])
    out = subprocess.check_output([exe], text=True)
    return {d["case"]: d for d in (json.loads(l) for l in out.splitlines() if l.strip())}


def test_lbfgs_minimizes_rosenbrock_and_respects_the_barrier():
    res = run_driver()
    r = res["rosenbrock"]
    assert r["converged"] == 1 and abs(r["x"][0] - 1) < 1e-6 and abs(r["x"][1] - 1) < 1e-6
    b = res["barrier_quadratic"]
    # the minimum (2.5, −1) lies next to a region that cannot be evaluated
    assert abs(b["x"][0] - 2.5) < 1e-6 and abs(b["x"][1] + 1) < 1e-6 and b["f"] < 1e-10
    lg = res["logit"]
    assert lg["ok"] == 1 and lg["roundtrip"] < 1e-12 and lg["jac"] < 1e-6
