"""The allocation-free entry point, gprx_exact_eval_noalloc, through the C ABI.

Some callers cannot allocate device memory at the moment they need an
evaluation (work recorded while a CUDA graph is captured, code inside a
framework or a server that owns all of the device's memory, loops that cannot
afford cudaMalloc's device-wide synchronisation).  This entry point takes the
caller's device buffers and uses one fixed scratch array per GPU instead of
allocating.  The test compares it with the existing batched entry point on the
same problem, on two calls in a row (the scratch keeps the previous call's
contents), at the tolerance the other parity tests use, and checks that a
problem larger than the scratch is refused.  Device buffers for the inputs and
outputs come from torch: the test allocates them, the entry point does not.
"""

import ctypes as C
import math

import numpy as np
import pytest

import gprx_b200 as gx
from gprx_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-10


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


def _noalloc(torch, spec, x, y, n, d, params):
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    yd = torch.from_numpy(y).to(dev)
    p = params.size
    nl = torch.zeros(1, dtype=torch.float64, device=dev)
    g = torch.zeros(p, dtype=torch.float64, device=dev)
    st = torch.full((1,), -1, dtype=torch.int32, device=dev)
    nodes, nn = spec.node_array()
    pa = np.ascontiguousarray(params, dtype=np.float64)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = _fn()(xd.data_ptr(), yd.data_ptr(), n, d, nodes, nn, L.ptr(pa), p, None, nl.data_ptr(), g.data_ptr(),
               st.data_ptr(), stream)
    torch.cuda.synchronize(dev)
    return rc, nl.item(), g.cpu().numpy(), int(st.item())


@pytest.mark.parametrize("n", [1, 37, 200, 512])
def test_noalloc_matches_batched_entry_point_twice(n):
    torch = pytest.importorskip("torch")
    d = 3
    spec = gx.RbfKernel(1.2) + gx.PeriodicKernel(0.9, 14.0)
    x, y = _problem(n, d, 40 + n)
    batch = gx.GprBatch(spec, [x], [y], d)
    thetas = [np.array([math.log(1.2), math.log(0.9), math.log(14.0), math.log(0.1)]),
              np.array([math.log(0.7), math.log(1.5), math.log(11.0), math.log(0.2)])]
    for params in thetas:  # two calls in a row share the scratch
        rc, nl, g, st = _noalloc(torch, spec, x, y, n, d, params)
        assert rc == L.OK and st == L.OK
        nl_b, g_b, st_b = batch.value_and_gradient(params[None, :])
        assert st_b[0] == L.OK
        assert abs(nl - nl_b[0]) / max(abs(nl_b[0]), 1.0) <= TOL
        assert np.all(np.abs(g - g_b[0]) / np.maximum(np.abs(g_b[0]), 1.0) <= TOL)


def test_noalloc_rejects_problems_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    n, d = 513, 2
    spec = gx.RbfKernel(1.0)
    x, y = _problem(n, d, 3)
    rc, _, _, _ = _noalloc(torch, spec, x, y, n, d, np.array([0.0, math.log(0.1)]))
    assert rc == L.CAPACITY
    assert b"512" in L.last_error().message
