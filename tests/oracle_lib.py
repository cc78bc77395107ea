"""ctypes wrapper of the CPU oracle (oracle/gprx_oracle.cpp).

Test infrastructure: the reference results the CUDA backend is compared against.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
"""

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "libgprx_oracle.so")

_lib = None

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)
U64 = C.POINTER(C.c_uint64)


def _ptr(a, t=D):
    return a.ctypes.data_as(t) if a is not None else None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(ORACLE_DIR, "gprx_oracle.cpp")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    L = C.CDLL(ORACLE_SO)
    L.orc_exact_eval.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, C.c_int, C.c_double,
                                 C.c_double, C.c_int, C.c_double, D, D, D, D]
    L.orc_exact_hessian.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, C.c_int, C.c_double,
                                    C.c_double, C.c_int, C.c_double, D]
    L.orc_exact_predict.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, C.c_int, C.c_double,
                                    C.c_double, C.c_int, C.c_double, D, C.c_int64, C.c_int, D, D]
    L.orc_exact_loo.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, C.c_int, C.c_double,
                                C.c_double, C.c_int, C.c_double, C.c_int, D, D]
    L.orc_exact_covariance.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, C.c_int, C.c_double,
                                       C.c_double, C.c_int, C.c_double, D, C.c_int64, C.c_int, D, D]
    L.orc_exact_sample.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, C.c_int, C.c_double,
                                   C.c_double, C.c_int, C.c_double, D, C.c_int64, C.c_int, C.c_int64, C.c_uint64, D]
    L.orc_gram_lower.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D]
    L.orc_cross.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, D, C.c_int64, C.c_int, D]
    L.orc_potrf.argtypes = [D, C.c_int64]
    L.orc_llt_inverse.argtypes = [D, C.c_int64, D]
    L.orc_num_params.argtypes = [I32, C.c_int]
    L.orc_online_create.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D]
    L.orc_online_create.restype = C.c_void_p
    L.orc_online_destroy.argtypes = [C.c_void_p]
    L.orc_online_n.argtypes = [C.c_void_p]
    L.orc_online_n.restype = C.c_int64
    L.orc_online_insert.argtypes = [C.c_void_p, D, C.c_double, U64]
    L.orc_online_delete.argtypes = [C.c_void_p, C.c_uint64]
    L.orc_online_ids.argtypes = [C.c_void_p, U64]
    L.orc_online_nlml.argtypes = [C.c_void_p]
    L.orc_online_nlml.restype = C.c_double
    L.orc_online_predict.argtypes = [C.c_void_p, D, C.c_int64, C.c_int, D, D]
    L.orc_online_ld.argtypes = [C.c_void_p, D]
    L.orc_sgpr_create.argtypes = [I32, C.c_int, D, C.c_int, D, C.c_int64, C.c_int, D, D, C.c_int64, C.c_int,
                                  C.c_double, C.c_double, C.c_int, C.c_double, C.POINTER(C.c_int)]
    L.orc_sgpr_create.restype = C.c_void_p
    L.orc_sgpr_destroy.argtypes = [C.c_void_p]
    L.orc_sgpr_nlml.argtypes = [C.c_void_p]
    L.orc_sgpr_nlml.restype = C.c_double
    L.orc_sgpr_grad.argtypes = [C.c_void_p, D]
    L.orc_sgpr_predict.argtypes = [C.c_void_p, D, C.c_int64, C.c_int, D, D]
    L.orc_sgpr_covariance.argtypes = [C.c_void_p, D, C.c_int64, C.c_int, D, D]
    L.orc_sgpr_sample.argtypes = [C.c_void_p, D, C.c_int64, C.c_int, C.c_int64, C.c_uint64, D]
    L.orc_sgpr_insert.argtypes = [C.c_void_p, D, C.c_double, U64]
    L.orc_sgpr_delete.argtypes = [C.c_void_p, C.c_uint64]
    L.orc_sgpr_set_inducing.argtypes = [C.c_void_p, D, C.c_int64]
    L.orc_sgpr_insert_inducing.argtypes = [C.c_void_p, D]
    L.orc_sgpr_n.argtypes = [C.c_void_p]
    L.orc_sgpr_n.restype = C.c_int64
    L.orc_sgpr_kmm_jitter.argtypes = [C.c_void_p]
    L.orc_sgpr_kmm_jitter.restype = C.c_double
    L.orc_sgpr_last_in_place.argtypes = [C.c_void_p]
    L.orc_rng_seed.argtypes = [U64, C.c_uint64]
    L.orc_rng_next.argtypes = [U64]
    L.orc_rng_next.restype = C.c_uint64
    L.orc_set_threads.argtypes = [C.c_int]
    _lib = L
    return L


def _nodes(nodes):
    return np.ascontiguousarray(np.asarray(nodes, dtype=np.int32).reshape(-1))


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


FIXED = (0, 0.0, 1.0, 0, 0.0)              # JitterPolicy::fixed(0.0)
SPARSE = (1, 1e-8, 10.0, 5, 1e-3)          # JitterPolicy::adaptive(1e-8, 10, 5, 1e-3)


class OracleError(RuntimeError):
    def __init__(self, status):
        super().__init__("oracle status %d" % status)
        self.status = status


def exact_eval(nodes, params, x, n, d, y, grad=True, jitter=FIXED):
    L = lib()
    nd = _nodes(nodes)
    p = _f(params)
    x = _f(x)
    y = _f(y)
    nl = np.zeros(1)
    g = np.zeros(len(p)) if grad else None
    a = np.zeros(n)
    ju = np.zeros(1)
    st = L.orc_exact_eval(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(x), n, d, _ptr(y), *jitter,
                          _ptr(nl), _ptr(g), _ptr(a), _ptr(ju))
    if st != 0:
        raise OracleError(st)
    return nl[0], g, a, ju[0]


def exact_hessian(nodes, params, x, n, d, y, jitter=FIXED):
    """Analytic NLML Hessian, p × p."""
    L = lib()
    nd = _nodes(nodes)
    p = _f(params)
    h = np.zeros(len(p) * len(p))
    st = L.orc_exact_hessian(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)), *jitter,
                             _ptr(h))
    if st != 0:
        raise OracleError(st)
    return h.reshape(len(p), len(p))


def exact_loo(nodes, params, x, n, d, y, kind, jitter=FIXED):
    L = lib()
    nd = _nodes(nodes)
    p = _f(params)
    mean = np.zeros(n)
    var = np.zeros(n)
    st = L.orc_exact_loo(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)), *jitter,
                         kind, _ptr(mean), _ptr(var))
    if st != 0:
        raise OracleError(st)
    return mean, var


def exact_covariance(nodes, params, x, n, d, y, xs, q, kind, jitter=FIXED):
    L = lib()
    nd = _nodes(nodes)
    p = _f(params)
    mean = np.zeros(q)
    cov = np.zeros(q * q)
    st = L.orc_exact_covariance(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)),
                                *jitter, _ptr(_f(xs)), q, kind, _ptr(mean), _ptr(cov))
    if st != 0:
        raise OracleError(st)
    return mean, cov.reshape(q, q, order="F")


def exact_sample(nodes, params, x, n, d, y, xs, q, kind, n_draws, seed, jitter=FIXED):
    L = lib()
    nd = _nodes(nodes)
    p = _f(params)
    out = np.zeros(q * n_draws)
    st = L.orc_exact_sample(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)),
                            *jitter, _ptr(_f(xs)), q, kind, n_draws, seed, _ptr(out))
    if st != 0:
        raise OracleError(st)
    return out


def exact_predict(nodes, params, x, n, d, y, xs, q, kind, jitter=FIXED):
    L = lib()
    nd = _nodes(nodes)
    p = _f(params)
    mean = np.zeros(q)
    var = np.zeros(q)
    st = L.orc_exact_predict(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)),
                             *jitter, _ptr(_f(xs)), q, kind, _ptr(mean), _ptr(var))
    if st != 0:
        raise OracleError(st)
    return mean, var


def gram_lower(nodes, theta, x, n, d):
    L = lib()
    nd = _nodes(nodes)
    th = _f(theta)
    k = np.zeros(n * n)
    st = L.orc_gram_lower(_ptr(nd, I32), len(nd) // 2, _ptr(th), len(th), _ptr(_f(x)), n, d, _ptr(k))
    if st != 0:
        raise OracleError(st)
    return k.reshape(n, n).T  # column-major → [i, j]


def cross(nodes, theta, x1, n1, x2, n2, d):
    L = lib()
    nd = _nodes(nodes)
    th = _f(theta)
    out = np.zeros(n1 * n2)
    L.orc_cross(_ptr(nd, I32), len(nd) // 2, _ptr(th), len(th), _ptr(_f(x1)), n1, _ptr(_f(x2)), n2, d, _ptr(out))
    return out.reshape(n2, n1).T


class Online:
    def __init__(self, nodes, params, x, n, d, y):
        L = lib()
        nd = _nodes(nodes)
        p = _f(params)
        self.d = d
        self.h = L.orc_online_create(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)))
        if not self.h:
            raise OracleError(1)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_online_destroy(self.h)
            self.h = None

    @property
    def n(self):
        return lib().orc_online_n(self.h)

    def insert(self, x, y):
        pid = C.c_uint64(0)
        st = lib().orc_online_insert(self.h, _ptr(_f(x)), float(y), C.byref(pid))
        if st != 0:
            raise OracleError(st)
        return pid.value

    def delete(self, pid):
        st = lib().orc_online_delete(self.h, int(pid))
        if st != 0:
            raise OracleError(st)

    def ids(self):
        out = np.zeros(self.n, dtype=np.uint64)
        lib().orc_online_ids(self.h, _ptr(out, U64))
        return out

    def nlml(self):
        return lib().orc_online_nlml(self.h)

    def predict(self, xs, q, kind):
        mean = np.zeros(q)
        var = np.zeros(q)
        lib().orc_online_predict(self.h, _ptr(_f(xs)), q, kind, _ptr(mean), _ptr(var))
        return mean, var

    def ld(self):
        n = self.n
        out = np.zeros(n * n)
        lib().orc_online_ld(self.h, _ptr(out))
        return out.reshape(n, n).T


class Sgpr:
    def __init__(self, nodes, params, x, n, d, y, z, m, jitter=SPARSE):
        L = lib()
        nd = _nodes(nodes)
        p = _f(params)
        self.p = len(p)
        st = C.c_int(0)
        self.h = L.orc_sgpr_create(_ptr(nd, I32), len(nd) // 2, _ptr(p), len(p), _ptr(_f(x)), n, d, _ptr(_f(y)),
                                   _ptr(_f(z)), m, *jitter, C.byref(st))
        if not self.h:
            raise OracleError(st.value)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sgpr_destroy(self.h)
            self.h = None

    def nlml(self):
        return lib().orc_sgpr_nlml(self.h)

    def grad(self):
        g = np.zeros(self.p)
        lib().orc_sgpr_grad(self.h, _ptr(g))
        return g

    def predict(self, xs, q, kind):
        mean = np.zeros(q)
        var = np.zeros(q)
        lib().orc_sgpr_predict(self.h, _ptr(_f(xs)), q, kind, _ptr(mean), _ptr(var))
        return mean, var

    def covariance(self, xs, q, kind):
        mean = np.zeros(q)
        cov = np.zeros(q * q)
        lib().orc_sgpr_covariance(self.h, _ptr(_f(xs)), q, kind, _ptr(mean), _ptr(cov))
        return mean, cov.reshape(q, q).T

    def sample(self, xs, q, kind, n_draws, seed):
        out = np.zeros(q * n_draws)
        st = lib().orc_sgpr_sample(self.h, _ptr(_f(xs)), q, kind, n_draws, seed, _ptr(out))
        if st != 0:
            raise OracleError(st)
        return out.reshape(n_draws, q)

    def insert(self, x, y):
        pid = C.c_uint64(0)
        st = lib().orc_sgpr_insert(self.h, _ptr(_f(x)), float(y), C.byref(pid))
        if st != 0:
            raise OracleError(st)
        return pid.value

    def delete(self, pid):
        st = lib().orc_sgpr_delete(self.h, int(pid))
        if st != 0:
            raise OracleError(st)

    def set_inducing(self, z, m):
        st = lib().orc_sgpr_set_inducing(self.h, _ptr(_f(z)), m)
        if st != 0:
            raise OracleError(st)

    def insert_inducing(self, z_new):
        """Bordered insert when the gates hold, else the assembly of the new
        set; last_in_place tells which (inducing_append, updates.rs:296-390)."""
        st = lib().orc_sgpr_insert_inducing(self.h, _ptr(_f(z_new)))
        if st != 0:
            raise OracleError(st)

    @property
    def n(self):
        return lib().orc_sgpr_n(self.h)

    @property
    def kmm_jitter(self):
        return lib().orc_sgpr_kmm_jitter(self.h)

    @property
    def last_in_place(self):
        return lib().orc_sgpr_last_in_place(self.h)


def rng_seq(seed, count):
    L = lib()
    st = np.zeros(4, dtype=np.uint64)
    L.orc_rng_seed(_ptr(st, U64), seed)
    return [L.orc_rng_next(_ptr(st, U64)) for _ in range(count)]


def rel_err(a, e):
    """|a − e| / max(|e|, 1): the reference's tolerance metric (tests/common/check.rs:8-10)."""
    a = np.asarray(a, dtype=np.float64)
    e = np.asarray(e, dtype=np.float64)
    return np.abs(a - e) / np.maximum(np.abs(e), 1.0)
