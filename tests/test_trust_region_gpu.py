"""Gpr::fit with the TrustRegion optimizer over gprx_exact_value_gradient_hessian:
the reference's own check (src/optimizer/trust_region.rs:329-365: 30
iterations lower the NLML of an RBF model below its start), a seeded ARD
problem where the trust region reaches the L-BFGS optimum (NLML within 1e-6,
gradient ≤ 1e-5), and the joint entry point against the separate ones.  The
NLML at the fitted θ is checked against the oracle (1e-10)."""

import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O
from hessian_cases import ard_case, col, reference_cases

pytestmark = pytest.mark.gpu


def test_trust_region_lowers_gpr_nlml():
    x = [0.0, 0.8, 1.7]
    y = [0.4, -0.2, 0.9]
    start_model = gx.Gpr(gx.RbfKernel(1.25), gx.GaussianLikelihood(0.16)).with_optimizer(gx.Fixed()).factor(
        x, 3, 1, y)
    start = start_model.neg_log_marginal_likelihood()
    fitted = gx.Gpr(gx.RbfKernel(1.25), gx.GaussianLikelihood(0.16)).with_optimizer(
        gx.TrustRegion().with_max_iterations(30)).fit(x, 3, 1, y)
    assert fitted.neg_log_marginal_likelihood() < start


def test_trust_region_reaches_the_lbfgs_optimum():
    _, nodes, params, x, y = ard_case(150)
    n, d = x.shape
    spec = gx.KernelSpec.from_nodes(nodes, params[:-1])
    lik = gx.GaussianLikelihood(math.exp(params[-1]))
    tr = gx.Gpr(spec, lik).with_optimizer(gx.TrustRegion().with_max_iterations(200)).fit(col(x), n, d, y)
    lb = gx.Gpr(spec, lik).with_optimizer(gx.Lbfgs().with_max_iterations(500)).fit(col(x), n, d, y)
    v_tr, v_lb = tr.neg_log_marginal_likelihood(), lb.neg_log_marginal_likelihood()
    assert v_tr <= v_lb + 1e-6, (v_tr, v_lb)
    theta = np.zeros(tr.num_params())
    theta[:] = tr.get_params()
    v, g = tr.value_and_gradient(theta)
    assert np.max(np.abs(g)) <= 1e-5 * max(1.0, abs(v)), g
    vo = O.exact_eval(nodes, theta, col(x), n, d, y)[0]
    assert O.rel_err(v, vo) <= 1e-10
    assert tr.report.evaluations >= tr.report.iterations


def test_joint_entry_matches_separate_calls():
    _, nodes, params, x, y = reference_cases()[3]
    n, d = x.shape
    spec = gx.KernelSpec.from_nodes(nodes, params[:-1])
    m = gx.Gpr(spec, gx.GaussianLikelihood(math.exp(params[-1]))).with_optimizer(gx.Fixed()).factor(col(x), n, d, y)
    v, g, h = m.value_gradient_hessian(params)
    v2, g2 = m.value_and_gradient(params)
    h2 = m.hessian(params)
    assert v == v2 and np.array_equal(g, g2) and np.array_equal(h, h2)
