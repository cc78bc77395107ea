"""CPU checks of the oracle's analytic NLML Hessian (the parity reference of
gprx_exact_hessian), pinned the way the reference pins its own
(src/gpr/tests.rs:1394-1493): every entry against central differences
(h = 1e-5) of the oracle's gradient, which the committed goldens pin, within
2e-4 · max(|fd|, 1); plus symmetry and repeatability.
"""

import numpy as np
import pytest

import oracle_lib as O
from hessian_cases import ard_case, col, periodic_case, reference_cases

CASES = reference_cases() + [periodic_case(), ard_case(12), ard_case(20, d=5)]


def fd_hessian(nodes, params, x, y, h=1e-5):
    n, d = x.shape
    p = len(params)
    out = np.zeros((p, p))
    for j in range(p):
        plus = np.array(params, dtype=float)
        minus = plus.copy()
        plus[j] += h
        minus[j] -= h
        gp = O.exact_eval(nodes, plus, col(x), n, d, y)[1]
        gm = O.exact_eval(nodes, minus, col(x), n, d, y)[1]
        out[:, j] = (gp - gm) / (2 * h)
    return out


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_hessian_matches_finite_differences(case):
    _, nodes, params, x, y = case
    n, d = x.shape
    hess = O.exact_hessian(nodes, params, col(x), n, d, y)
    fd = fd_hessian(nodes, params, x, y)
    scale = np.maximum(np.abs(fd), 1.0)
    assert np.all(np.abs(hess - fd) <= 2e-4 * scale), (hess, fd)
    assert np.array_equal(hess, hess.T)
    again = O.exact_hessian(nodes, params, col(x), n, d, y)
    assert np.array_equal(hess, again)
