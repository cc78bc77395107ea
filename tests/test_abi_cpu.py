"""CPU-only checks of the C ABI: the library loads, exports every declared
symbol, validates arguments before touching a device, and its seeded RNG
reproduces the reference's pinned Xoshiro256++ sequence (src/rng.rs)."""

import ctypes as C
import json
import os

import numpy as np
import pytest

import gprx_b200 as gx
from gprx_b200 import _lib as L

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    declared = L.declared_symbols()
    assert len(declared) > 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert missing == []
    assert lib.gprx_abi_version() == 1


def test_rng_matches_pinned_sequence():
    pins = json.load(open(os.path.join(GOLD, "rng_pins.json")))["seeds"]
    for seed, vals in pins.items():
        r = gx.SeededRng(int(seed))
        assert [r.next_u64() for _ in range(4)] == [int(v) for v in vals]


def test_rng_ranges_and_subset():
    r = gx.SeededRng(7)
    for mx in (0, 1, 2, 9, 1000):
        for _ in range(200):
            assert r.up_to(mx) <= mx
    u = r.unit(1000)
    assert np.all((u >= 0.0) & (u < 1.0))
    s = gx.SeededRng(2).subset(1000, 100)
    assert len(set(s.tolist())) == 100 and s.max() < 1000
    # the same seed gives the same subset
    assert np.array_equal(s, gx.SeededRng(2).subset(1000, 100))


def _create(x, n, d, y, nodes, theta):
    arr = (L.KernelNode * len(nodes))()
    for i, (k, a) in enumerate(nodes):
        arr[i].kind, arr[i].arg = k, a
    th = L.f64(theta)
    h = C.c_void_p()
    st = L.lib().gprx_exact_create(L.ptr(L.f64(x)), n, d, L.ptr(L.f64(y)), arr, len(nodes), L.ptr(th), th.size,
                                   None, C.byref(h))
    return st, h


def test_create_rejects_bad_arguments_before_any_device_work():
    x = np.zeros(6)
    y = np.zeros(3)
    bad = x.copy()
    bad[1] = np.nan
    assert _create(bad, 3, 2, y, [(10, 0)], [0.0, -1.0])[0] == L.NONFINITE_INPUT
    assert _create(x, 0, 2, y, [(10, 0)], [0.0, -1.0])[0] == L.EMPTY_INPUT
    assert _create(x, 3, 2, y, [(10, 0)], [0.0])[0] == L.SHAPE_MISMATCH          # θ misses log σn²
    assert _create(x, 3, 2, y, [(99, 0)], [0.0, -1.0])[0] == L.INVALID_CONFIG    # unknown leaf
    assert _create(x, 3, 2, y, [(1, 2), (10, 0)], [0.0, -1.0])[0] == L.INVALID_CONFIG  # truncated sum
    assert _create(x, 3, 2, y, [(10, 0)], [30.0, -1.0])[0] == L.INVALID_HYPERPARAMETER  # ℓ > 1e5
    assert _create(x, 3, 2, y, [(11, 3)], [0.0, 0.0, 0.0, -1.0])[0] == L.SHAPE_MISMATCH  # ARD dims ≠ d


def test_kernel_spec_flattens_and_orders_parameters():
    k = gx.ConstantKernel(2.0) * gx.RbfArdKernel([1.0, 2.0]) + gx.PeriodicKernel(1.5, 3.0)
    assert k.nodes() == [(1, 2), (2, 2), (12, 0), (11, 2), (13, 0)]
    assert np.allclose(k.get_params(), np.log([2.0, 1.0, 2.0, 1.5, 3.0]))
    k2 = gx.RbfKernel(1.0) + gx.RbfKernel(2.0) + gx.RbfKernel(3.0)
    assert k2.nodes() == [(1, 3), (10, 0), (10, 0), (10, 0)]
    with pytest.raises(gx.InvalidHyperparameter):
        gx.RbfKernel(0.0)
