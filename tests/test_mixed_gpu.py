"""The mixed-precision exact evaluation (Precision.Mixed) against the FP64
oracle and against the plain FP64 GPU path.

In the mixed form the factor and the inverse are computed together by
recursive halving: the coupling products (L21 = A21 X11ᵀ, A22 −= L21 L21ᵀ,
X21 = −X22 L21 X11) and K⁻¹ = XᵀX run on the int8 tensor cores as sliced FP64
emulations (7 int8 digits of 7 bits per row-scaled entry, exact int32 sums);
blocks of up to 4096 rows use the FP64 blocked factor; the fill, the log-det
and the gradient contraction stay FP64.
Targets: NLML within 1e-8 and gradient within 1e-6 relative to FP64,
|a − e| / max(|e|, 1).  Sizes from n = 1024 (the smallest n that uses the
emulated products) up, ragged ones included.
"""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O

pytestmark = pytest.mark.gpu

TOL_NLML = 1e-8
TOL_GRAD = 1e-6


def make_data(n, d, seed):
    rs = np.random.RandomState(seed)
    x = rs.standard_normal(n * d)
    y = np.sin(x[:n]) + 0.5 * np.cos(x[n:2 * n] if d > 1 else x[:n]) + 0.05 * rs.standard_normal(n)
    return x, y


def model(spec, noise, x, n, d, y, precision):
    return gx.Gpr(spec, gx.GaussianLikelihood(noise), precision=precision).with_optimizer(gx.Fixed()).factor(
        x, n, d, y)


@pytest.mark.parametrize("n", [1024, 1100, 1536, 2100, 4500, 8300])
def test_mixed_eval_matches_oracle_ard8(n):
    d = 8
    rs = np.random.RandomState(n)
    ls = np.exp(rs.uniform(math.log(0.3), math.log(3.0), size=d))
    spec = gx.ConstantKernel(2.0) * gx.RbfArdKernel(list(ls))
    nodes = [[2, 2], [12, 0], [11, d]]
    x, y = make_data(n, d, seed=n + 1)
    m = model(spec, 0.0025, x, n, d, y, gx.Precision.Mixed)
    f = model(spec, 0.0025, x, n, d, y, gx.Precision.Fp64)
    theta = np.array([math.log(2.0)] + list(np.log(ls)) + [math.log(0.0025)])
    for k in range(2):
        params = theta + 0.1 * rs.standard_normal(theta.size)
        nl_o, g_o, _, _ = O.exact_eval(nodes, params, x, n, d, y)
        nl, g = m.value_and_gradient(params)
        nl_f, g_f = f.value_and_gradient(params)
        assert O.rel_err(nl, nl_o) <= TOL_NLML, (nl, nl_o)
        assert np.all(O.rel_err(g, g_o) <= TOL_GRAD), (g, g_o)
        assert O.rel_err(nl, nl_f) <= TOL_NLML
        assert np.all(O.rel_err(g, g_f) <= TOL_GRAD)


def test_mixed_eval_matches_oracle_rbf_plus_periodic():
    n, d = 1300, 1
    spec = gx.RbfKernel(0.8) + gx.PeriodicKernel(1.1, 2.0)
    nodes = [[1, 2], [10, 0], [13, 0]]
    x, y = make_data(n, d, seed=3)
    m = model(spec, 0.01, x, n, d, y, gx.Precision.Mixed)
    params = np.array([math.log(0.8), math.log(1.1), math.log(2.0), math.log(0.01)])
    nl_o, g_o, _, _ = O.exact_eval(nodes, params, x, n, d, y)
    nl, g = m.value_and_gradient(params)
    assert O.rel_err(nl, nl_o) <= TOL_NLML
    assert np.all(O.rel_err(g, g_o) <= TOL_GRAD)


def test_mixed_small_n_is_the_fp64_path():
    # below n = 1024 the mixed form runs the FP64 products: same bits
    n, d = 700, 3
    spec = gx.ConstantKernel(1.5) * gx.RbfArdKernel([0.7, 1.2, 2.0])
    x, y = make_data(n, d, seed=9)
    params = np.array([math.log(1.5), math.log(0.7), math.log(1.2), math.log(2.0), math.log(0.05)])
    a = model(spec, 0.05, x, n, d, y, gx.Precision.Mixed).value_and_gradient(params)
    b = model(spec, 0.05, x, n, d, y, gx.Precision.Fp64).value_and_gradient(params)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])


def test_mixed_sgpr_matches_oracle():
    # n ≥ 16384 takes the emulated Gram products B = AAᵀ and H = GAᵀ (K
    # split into parts of 32768); the m×n solves stay FP64
    n, m, d = 70000, 256, 3
    rs = np.random.RandomState(12)
    x = rs.uniform(0, 1, size=n * d)
    y = np.sin(6 * x[:n]) + np.cos(4 * x[n:2 * n]) + 0.1 * rs.standard_normal(n)
    idx = rs.choice(n, m, replace=False)
    z = x.reshape(d, n)[:, idx].reshape(-1).copy()
    ls = [0.3, 0.5, 0.4]
    params = np.array([math.log(v) for v in ls] + [math.log(0.05)])
    orc = O.Sgpr([[11, d]], params, x, n, d, y, z, m)
    spec = gx.RbfArdKernel(ls)
    out = {}
    for prec in (gx.Precision.Mixed, gx.Precision.Fp64):
        f = gx.Sgpr(spec, gx.GaussianLikelihood(0.05), precision=prec).with_optimizer(gx.Fixed()).factor(
            x, n, d, y, z, m)
        out[prec] = f.value_and_gradient(params)
    nl, g = out[gx.Precision.Mixed]
    nl_f, g_f = out[gx.Precision.Fp64]
    assert O.rel_err(nl, orc.nlml()) <= TOL_NLML, (nl, orc.nlml())
    assert np.all(O.rel_err(g, orc.grad()) <= TOL_GRAD), (g, orc.grad())
    assert O.rel_err(nl, nl_f) <= TOL_NLML
    assert np.all(O.rel_err(g, g_f) <= TOL_GRAD)


def test_mixed_sgpr_matches_fp64_m1024():
    # m = 1024 inducing points: the Gram parts cover a 1024² output (more
    # elements than one grid-stride pass of the reduction), n over one
    # split-K part of 32768
    n, m, d = 40000, 1024, 4
    rs = np.random.RandomState(5)
    x = rs.uniform(0, 1, size=n * d)
    y = np.sin(5 * x[:n]) + np.cos(3 * x[n:2 * n]) + 0.1 * rs.standard_normal(n)
    z = x.reshape(d, n)[:, rs.choice(n, m, replace=False)].reshape(-1).copy()
    ls = [0.6, 0.9, 1.3, 0.8]
    params = np.array([math.log(v) for v in ls] + [math.log(0.1)])
    out = {}
    for prec in (gx.Precision.Mixed, gx.Precision.Fp64):
        f = gx.Sgpr(gx.RbfArdKernel(ls), gx.GaussianLikelihood(0.1), precision=prec).with_optimizer(
            gx.Fixed()).factor(x, n, d, y, z, m)
        out[prec] = f.value_and_gradient(params)
    nl, g = out[gx.Precision.Mixed]
    nl_f, g_f = out[gx.Precision.Fp64]
    assert O.rel_err(nl, nl_f) <= TOL_NLML, (nl, nl_f)
    assert np.all(O.rel_err(g, g_f) <= TOL_GRAD), (g, g_f)
