"""gprx_exact_hessian against the oracle's analytic Hessian (itself pinned on
finite differences of the golden-pinned gradient): the reference's own cases
(src/gpr/tests.rs:1394-1493), a periodic product and seeded ARD cases up to
n = 1100, with up to 15 kernel parameters.  FP64: |a − e| ≤ 1e-9 · max(max|e|, 1) per entry; the mixed form
(emulated products from n = 1024): 1e-6 on the same scale.  A second call
gives the same bits (src/gpr/tests.rs:1440-1442), and the model is left at
the evaluated θ like a gradient evaluation.
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O
from hessian_cases import ard_case, col, periodic_case, reference_cases

pytestmark = pytest.mark.gpu

# ard*_d12 has 15 kernel parameters: the per-row second-order launches and the
# pairwise trace products (the others take the single-launch forms)
CASES = reference_cases() + [periodic_case(), ard_case(65), ard_case(300), ard_case(97, d=12)]


def fitted(nodes, params, x, y, precision=gx.Precision.Fp64):
    n, d = x.shape
    spec = gx.KernelSpec.from_nodes(nodes, params[:-1])
    gpr = gx.Gpr(spec, gx.GaussianLikelihood(math.exp(params[-1])), precision=precision)
    return gpr.with_optimizer(gx.Fixed()).factor(col(x), n, d, y)


def check(h, e, tol):
    scale = max(np.max(np.abs(e)), 1.0)
    err = np.max(np.abs(h - e)) / scale
    assert err <= tol, (err, h, e)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_hessian_matches_oracle(case):
    _, nodes, params, x, y = case
    n, d = x.shape
    m = fitted(nodes, params, x, y)
    h = m.hessian(params)
    e = O.exact_hessian(nodes, params, col(x), n, d, y)
    check(h, e, 1e-9)
    assert np.array_equal(h, h.T)
    assert np.array_equal(h, m.hessian(params))


def test_hessian_at_other_params_then_state():
    _, nodes, params, x, y = ard_case(129)
    n, d = x.shape
    m = fitted(nodes, params, x, y)
    moved = np.array(params) + 0.1
    check(m.hessian(moved), O.exact_hessian(nodes, moved, col(x), n, d, y), 1e-9)
    # the model now sits at `moved`: value and prediction follow it
    v, g = m.value_and_gradient(moved)
    vo, go, _, _ = O.exact_eval(nodes, moved, col(x), n, d, y)
    assert O.rel_err(v, vo) <= 1e-10
    xs = x[:5] + 0.05
    mean = m.predict(col(xs), 5, d).mean
    mo, _ = O.exact_predict(nodes, moved, col(x), n, d, y, col(xs), 5, 0)
    assert np.all(O.rel_err(mean, mo) <= 1e-10)


def test_hessian_mixed_matches_oracle():
    _, nodes, params, x, y = ard_case(1100)
    n, d = x.shape
    m = fitted(nodes, params, x, y, gx.Precision.Mixed)
    check(m.hessian(params), O.exact_hessian(nodes, params, col(x), n, d, y), 1e-6)


def test_hessian_wrong_count():
    _, nodes, params, x, y = reference_cases()[0]
    m = fitted(nodes, params, x, y)
    with pytest.raises(gx.ShapeMismatch):
        m.hessian(params[:-1])
