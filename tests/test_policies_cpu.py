"""The trainer policies of the Python mirror (src/policy.rs:30-397,
src/gpr/trainer.rs): JitterPolicy's domain checks, the defaults (fixed(0) for
Gpr, adaptive(1e-8, 10, 5, 1e-3) for Sgpr, Cached distances, Retain, Accurate
exp), prefer_memory / prefer_speed, and the refusal of the FastApprox exp,
which the device does not build.  Host only."""

import math

import pytest

import gprx_b200 as gx


def test_jitter_policy_domain():
    assert gx.JitterPolicy.fixed(0.0) == gx.JitterPolicy.fixed(0.0)
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(gx.InvalidConfig):
            gx.JitterPolicy.fixed(bad)
    gx.JitterPolicy.adaptive(1e-8, 10.0, 5, 1e-3)
    for args in [(0.0, 10.0, 5, 1e-3), (1e-8, 1.0, 5, 1e-3), (1e-8, 10.0, 0, 1e-3), (1e-8, 10.0, 5, 1e-9),
                 (float("inf"), 10.0, 5, 1e-3), (1e-8, 10.0, 5, float("nan"))]:
        with pytest.raises(gx.InvalidConfig):
            gx.JitterPolicy.adaptive(*args)


def test_trainer_defaults_and_setters():
    g = gx.Gpr(gx.RbfKernel(1.25), gx.GaussianLikelihood(0.16))
    assert g.jitter_policy() == gx.JitterPolicy.fixed(0.0)
    assert g.math() == gx.KernelExp.Accurate
    assert (g.distance_cache_policy(), g.cholesky_buffer()) == (gx.DistanceCachePolicy.Cached, gx.CholeskyBuffer.Retain)
    g.with_prefer_memory()
    assert (g.distance_cache_policy(), g.cholesky_buffer()) == (gx.DistanceCachePolicy.Uncached, gx.CholeskyBuffer.Reuse)
    g.with_prefer_speed()
    assert (g.distance_cache_policy(), g.cholesky_buffer()) == (gx.DistanceCachePolicy.Cached, gx.CholeskyBuffer.Retain)
    pol = gx.JitterPolicy.adaptive(1e-6, 10.0, 3, 1e-2)
    assert g.with_jitter_policy(pol).jitter_policy() == pol
    assert g.with_optimizer(gx.Fixed()).jitter_policy() == pol
    with pytest.raises(gx.InvalidConfig):
        g.with_math(gx.KernelExp.FastApprox)
    assert g.num_params() == 2
    g.set_params([math.log(0.5), math.log(0.2)])
    assert abs(g.get_params()[0] - math.log(0.5)) < 1e-15 and abs(g.likelihood.noise_variance - 0.2) < 1e-15
    s = gx.Sgpr(gx.RbfKernel(1.0), gx.GaussianLikelihood(0.1))
    assert s.jitter_policy() == gx.JitterPolicy.adaptive(1e-8, 10.0, 5, 1e-3)
    assert s.with_jitter_policy(gx.JitterPolicy.fixed(1e-6)).with_optimizer(gx.Fixed()).jitter_policy() == \
        gx.JitterPolicy.fixed(1e-6)
