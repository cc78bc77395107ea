"""The allocation-free entry point, gprx_exact_eval_noalloc, through the C ABI.

Some callers cannot allocate device memory at the moment they need an
evaluation (work recorded while a CUDA graph is captured, code inside a
framework or a server that owns all of the device's memory, loops that cannot
afford cudaMalloc's device-wide synchronisation).  This entry point takes the
caller's device buffers and uses one fixed scratch array per GPU instead of
allocating.  The tests compare it with the existing batched entry point and
with the CPU oracle on the same problem, on calls in a row that share the
scratch (the array keeps the previous call's contents: other sizes, a failed
factor), at the tolerance the other parity tests use, and check the refusals
(a problem larger than the scratch, non-finite inputs, a device that is not
the stream's).  Device buffers for the inputs and outputs come from torch: the
test allocates them, the entry point does not.
"""

import ctypes as C
import math

import numpy as np
import pytest

import gprx_b200 as gx
import oracle_lib as O
from gprx_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-10
NODES = [[1, 2], [10, 0], [13, 0]]  # RbfKernel + PeriodicKernel, the oracle's prefix form


def _fn():
    f = L.lib().gprx_exact_eval_noalloc
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(L.KernelNode), C.c_int32, L.D,
                  C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def _problem(n, d, seed):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 5, size=(n, d))
    y = np.sin(x[:, 0]) + 0.5 * np.cos(x[:, -1]) + 0.1 * rs.standard_normal(n)
    return x.T.reshape(-1).copy(), y


def _stream(torch):
    return torch.cuda.current_stream(torch.device("cuda", 0)).cuda_stream


def _setup(torch):
    # the set-up-only call (n = 0): address lookup and kernel attribute, no work
    return _fn()(None, None, 0, 0, None, 0, None, 0, None, None, None, None, _stream(torch))


def _noalloc(torch, spec, x, y, n, d, params, options=None):
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    yd = torch.from_numpy(y).to(dev)
    p = params.size
    nl = torch.full((1,), -7.0, dtype=torch.float64, device=dev)
    g = torch.full((p,), -7.0, dtype=torch.float64, device=dev)
    st = torch.full((1,), -1, dtype=torch.int32, device=dev)
    nodes, nn = spec.node_array()
    pa = np.ascontiguousarray(params, dtype=np.float64)
    opt = C.byref(options) if options is not None else None
    rc = _fn()(xd.data_ptr(), yd.data_ptr(), n, d, nodes, nn, L.ptr(pa), p, opt, nl.data_ptr(), g.data_ptr(),
               st.data_ptr(), _stream(torch))
    torch.cuda.synchronize(dev)
    return rc, nl.item(), g.cpu().numpy(), int(st.item())


def _spec():
    return gx.RbfKernel(1.2) + gx.PeriodicKernel(0.9, 14.0)


def _theta(ell, ell_p, period, noise):
    return np.array([math.log(ell), math.log(ell_p), math.log(period), math.log(noise)])


def _rel(a, e):
    return np.abs(np.asarray(a) - np.asarray(e)) / np.maximum(np.abs(np.asarray(e)), 1.0)


def test_noalloc_setup_call_enqueues_nothing():
    torch = pytest.importorskip("torch")
    assert _setup(torch) == L.OK
    assert _setup(torch) == L.OK


@pytest.mark.parametrize("n", [1, 37, 200, 512])
def test_noalloc_matches_batched_entry_point_twice(n):
    torch = pytest.importorskip("torch")
    d = 3
    spec = _spec()
    x, y = _problem(n, d, 40 + n)
    batch = gx.GprBatch(spec, [x], [y], d)
    for params in (_theta(1.2, 0.9, 14.0, 0.1), _theta(0.7, 1.5, 11.0, 0.2)):  # two calls share the scratch
        rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, params)
        assert rc == L.OK and st == L.OK
        nl_b, g_b, st_b = batch.value_and_gradient(params[None, :])
        assert st_b[0] == L.OK
        assert _rel(nl, nl_b[0]) <= TOL
        assert np.all(_rel(g, g_b[0]) <= TOL)


def test_noalloc_sequence_of_sizes_and_a_failed_factor():
    # the scratch keeps whatever the previous call left (another n, so
    # another leading dimension; a factor that failed half way): each call
    # must still equal the batched entry point and the CPU oracle
    torch = pytest.importorskip("torch")
    d = 3
    spec = _spec()
    good = _theta(1.1, 1.0, 13.0, 0.1)
    for k, n in enumerate([37, 512, 1, 200, 512, 37]):
        x, y = _problem(n, d, 900 + k)
        rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, good)
        assert rc == L.OK and st == L.OK, (n, st)
        nl_b, g_b, st_b = gx.GprBatch(spec, [x], [y], d).value_and_gradient(good[None, :])
        assert st_b[0] == L.OK and _rel(nl, nl_b[0]) <= TOL and np.all(_rel(g, g_b[0]) <= TOL), n
        nl_o, g_o, _, _ = O.exact_eval(NODES, good, x, n, d, y)
        assert _rel(nl, nl_o) <= TOL and np.all(_rel(g, g_o) <= TOL), (n, nl, nl_o)
    # a periodic leaf on a 3-d Euclidean distance is indefinite; with the RBF
    # term at a tiny lengthscale (close to the identity) and little noise
    # (inside the default parameter intervals) the factor fails (the oracle
    # agrees), then a good call follows
    n = 120
    x, y = _problem(n, d, 77)
    bad = _theta(1e-3, 1.0, 1.0, 1e-4)
    with pytest.raises(O.OracleError):
        O.exact_eval(NODES, bad, x, n, d, y)
    rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, bad)
    assert rc == L.OK and st == L.CHOLESKY_FAILED and nl == 0.0 and np.all(g == 0.0)
    rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, good)
    assert rc == L.OK and st == L.OK
    nl_o, g_o, _, _ = O.exact_eval(NODES, good, x, n, d, y)
    assert _rel(nl, nl_o) <= TOL and np.all(_rel(g, g_o) <= TOL)


def test_noalloc_refuses_nonfinite_inputs():
    torch = pytest.importorskip("torch")
    n, d = 50, 3
    spec = _spec()
    params = _theta(1.2, 0.9, 14.0, 0.1)
    for where in ("x", "y"):
        x, y = _problem(n, d, 5)
        if where == "x":
            x[17] = float("nan")
        else:
            y[3] = float("inf")
        rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, params)
        assert rc == L.OK and st == L.NONFINITE_INPUT and nl == 0.0 and np.all(g == 0.0), where
    x, y = _problem(n, d, 5)  # the next call is clean again
    rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, params)
    nl_o, g_o, _, _ = O.exact_eval(NODES, params, x, n, d, y)
    assert rc == L.OK and st == L.OK and _rel(nl, nl_o) <= TOL and np.all(_rel(g, g_o) <= TOL)


def test_noalloc_rejects_problems_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    n, d = 513, 2
    spec = gx.RbfKernel(1.0)
    x, y = _problem(n, d, 3)
    rc, _, _, st = _noalloc(torch, spec, x, y, n, d, np.array([0.0, math.log(0.1)]))
    assert rc == L.CAPACITY and st == -1
    assert b"512" in L.last_error().message


def test_noalloc_rejects_a_device_other_than_the_streams():
    torch = pytest.importorskip("torch")
    n, d = 20, 2
    spec = gx.RbfKernel(1.0)
    x, y = _problem(n, d, 4)
    opt = L.Options()
    L.lib().gprx_options_default(C.byref(opt))
    opt.device = torch.cuda.device_count()  # a device the stream does not belong to
    rc, _, _, st = _noalloc(torch, spec, x, y, n, d, np.array([0.0, math.log(0.1)]), options=opt)
    assert rc == L.INVALID_CONFIG and st == -1
