"""ctypes binding of libgprx_cuda.so (include/gprx_cuda.h).

The library is built in-tree (gprx_b200/lib/libgprx_cuda.so) by
`python -m gprx_b200.build`.  There is no CPU fallback: when the library is
missing or fails to load, `lib()` raises.
"""

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libgprx_cuda.so")

D = C.POINTER(C.c_double)
U64 = C.POINTER(C.c_uint64)
I32 = C.POINTER(C.c_int32)

# status codes (gprx_status)
OK = 0
CHOLESKY_FAILED = 1
NONFINITE_KERNEL = 2
SHAPE_MISMATCH = 3
INVALID_POINT_ID = 4
INSUFFICIENT_DATA = 5
CUDA_ERROR = 6
TIMEOUT = 7
INVALID_HYPERPARAMETER = 8
NONFINITE_INPUT = 9
EMPTY_INPUT = 10
OUT_OF_MEMORY = 11
INVALID_CONFIG = 12
NOT_CONVERGED = 13
INVALID_ARGUMENT = 14
CAPACITY = 16
NOT_POSITIVE_DEFINITE = 17
PERSIST_FAILED = 18
UNSUPPORTED_PERSIST_VERSION = 19

# kernel node kinds
NODE_SUM, NODE_PRODUCT = 1, 2
LEAF_RBF, LEAF_RBF_ARD, LEAF_CONSTANT, LEAF_PERIODIC = 10, 11, 12, 13

PRECISION_FP64, PRECISION_MIXED = 0, 1
VARIANCE_LATENT, VARIANCE_OBSERVATION = 0, 1


class KernelNode(C.Structure):
    _fields_ = [("kind", C.c_int32), ("arg", C.c_int32)]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("jitter_kind", C.c_int32), ("jitter_initial", C.c_double),
                ("jitter_multiplier", C.c_double), ("jitter_max_retries", C.c_int32), ("jitter_max", C.c_double),
                ("device", C.c_int32), ("block_size", C.c_int32)]


class PersistInfo(C.Structure):
    _fields_ = [("n", C.c_uint64), ("d", C.c_uint64), ("n_nodes", C.c_int32), ("n_theta", C.c_int32),
                ("has_factor", C.c_int32), ("factor_kind", C.c_int32), ("factor_jitter", C.c_double),
                ("jitter", Options), ("next_point_id", C.c_uint64)]


class LbfgsOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_uint64), ("tolerance", C.c_double), ("history_size", C.c_int32),
                ("restarts", C.c_int32), ("seed", C.c_uint64), ("interval_lo", C.c_double),
                ("interval_hi", C.c_double)]


class TrustRegionOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_uint64), ("tolerance", C.c_double), ("initial_radius", C.c_double),
                ("max_radius", C.c_double), ("restarts", C.c_int32), ("seed", C.c_uint64),
                ("interval_lo", C.c_double), ("interval_hi", C.c_double)]


class FitReport(C.Structure):
    _fields_ = [("nlml", C.c_double), ("iterations", C.c_uint64), ("evaluations", C.c_uint64),
                ("grad_norm", C.c_double), ("converged", C.c_int32)]


class ErrorInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("jitter", C.c_double), ("matrix_size", C.c_uint64), ("stage", C.c_int32),
                ("cuda_error", C.c_int32), ("iterations", C.c_uint64), ("message", C.c_char * 256)]


class ServerOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("workers", C.c_int32), ("hbm_budget_bytes", C.c_uint64)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("model", C.c_uint64), ("kind", C.c_int32), ("submit_ns", C.c_int64),
                ("start_ns", C.c_int64), ("end_ns", C.c_int64), ("merged", C.c_int32), ("message", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("merged_launches", C.c_uint64), ("used_bytes", C.c_uint64),
                ("resident_models", C.c_uint64), ("merged_fit_launches", C.c_uint64)]


class Rng(C.Structure):
    _fields_ = [("s", C.c_uint64 * 4)]


_lib = None

# name → (restype, argtypes)
_SIGS = {
    "gprx_abi_version": (C.c_int32, []),
    "gprx_options_default": (None, [C.POINTER(Options)]),
    "gprx_options_default_sparse": (None, [C.POINTER(Options)]),
    "gprx_lbfgs_options_default": (None, [C.POINTER(LbfgsOptions)]),
    "gprx_trust_region_options_default": (None, [C.POINTER(TrustRegionOptions)]),
    "gprx_last_error": (C.c_int32, [C.POINTER(ErrorInfo)]),
    "gprx_launch_count": (C.c_uint64, []),
    "gprx_exact_create": (C.c_int32, [D, C.c_uint64, C.c_uint64, D, C.POINTER(KernelNode), C.c_int32, D, C.c_int32,
                                      C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "gprx_exact_destroy": (C.c_int32, [C.c_void_p]),
    "gprx_exact_set_data": (C.c_int32, [C.c_void_p, D, D]),
    "gprx_exact_num_params": (C.c_uint64, [C.c_void_p]),
    "gprx_exact_get_params": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_exact_set_params": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_exact_factor": (C.c_int32, [C.c_void_p]),
    "gprx_exact_eval": (C.c_int32, [C.c_void_p, D, C.c_uint64, D, D]),
    "gprx_exact_hessian": (C.c_int32, [C.c_void_p, D, C.c_uint64, D]),
    "gprx_exact_data": (C.c_int32, [C.c_void_p, D, D]),
    "gprx_exact_nlml": (C.c_int32, [C.c_void_p, D]),
    "gprx_exact_factor_jitter": (C.c_int32, [C.c_void_p, D]),
    "gprx_exact_predict": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_int32, D, D]),
    "gprx_exact_predict_group": (C.c_int32, [C.POINTER(C.c_void_p), C.c_uint64, C.POINTER(D), U64, C.c_int32,
                                             C.POINTER(D), C.POINTER(D)]),
    "gprx_exact_alpha": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_exact_fit": (C.c_int32, [C.c_void_p, C.POINTER(LbfgsOptions), C.POINTER(FitReport)]),
    "gprx_exact_fit_trust_region": (C.c_int32, [C.c_void_p, C.POINTER(TrustRegionOptions), C.POINTER(FitReport)]),
    "gprx_exact_value_gradient_hessian": (C.c_int32, [C.c_void_p, D, C.c_uint64, D, D, D]),
    "gprx_exact_stage_times": (C.c_int32, [C.c_void_p, D]),
    "gprx_exact_stream": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gprx_online_begin": (C.c_int32, [C.c_void_p]),
    "gprx_online_insert": (C.c_int32, [C.c_void_p, D, C.c_double, U64]),
    "gprx_online_delete": (C.c_int32, [C.c_void_p, C.c_uint64]),
    "gprx_online_n": (C.c_uint64, [C.c_void_p]),
    "gprx_online_point_ids": (C.c_int32, [C.c_void_p, U64, C.c_uint64]),
    "gprx_sgpr_create": (C.c_int32, [D, C.c_uint64, C.c_uint64, D, D, C.c_uint64, C.POINTER(KernelNode), C.c_int32,
                                     D, C.c_int32, C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "gprx_sgpr_destroy": (C.c_int32, [C.c_void_p]),
    "gprx_sgpr_num_params": (C.c_uint64, [C.c_void_p]),
    "gprx_sgpr_get_params": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_sgpr_factor": (C.c_int32, [C.c_void_p]),
    "gprx_sgpr_eval": (C.c_int32, [C.c_void_p, D, C.c_uint64, D, D]),
    "gprx_sgpr_nlml": (C.c_int32, [C.c_void_p, D]),
    "gprx_sgpr_set_params": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_sgpr_predict": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_int32, D, D]),
    "gprx_sgpr_predict_covariance": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_int32, D, D]),
    "gprx_sgpr_sample": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_int32, C.c_uint64, C.c_uint64, D]),
    "gprx_sgpr_fit": (C.c_int32, [C.c_void_p, C.POINTER(LbfgsOptions), C.POINTER(FitReport)]),
    "gprx_sgpr_insert": (C.c_int32, [C.c_void_p, D, C.c_double, U64]),
    "gprx_sgpr_delete": (C.c_int32, [C.c_void_p, C.c_uint64]),
    "gprx_sgpr_n": (C.c_uint64, [C.c_void_p]),
    "gprx_sgpr_last_step_in_place": (C.c_int32, [C.c_void_p]),
    "gprx_sgpr_point_ids": (C.c_int32, [C.c_void_p, U64, C.c_uint64]),
    "gprx_sgpr_set_inducing": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_sgpr_kmm_jitter": (C.c_int32, [C.c_void_p, D]),
    "gprx_sgpr_stream": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gprx_sgpr_stage_times": (C.c_int32, [C.c_void_p, D]),
    "gprx_batch_create": (C.c_int32, [D, D, U64, C.c_uint64, C.c_uint64, C.POINTER(KernelNode), C.c_int32,
                                      C.c_int32, C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "gprx_batch_destroy": (C.c_int32, [C.c_void_p]),
    "gprx_batch_num_params": (C.c_uint64, [C.c_void_p]),
    "gprx_batch_eval": (C.c_int32, [C.c_void_p, D, C.c_uint64, D, D, I32]),
    "gprx_batch_fit": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.POINTER(LbfgsOptions), D, C.POINTER(FitReport),
                                   I32]),
    "gprx_batch_stream": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gprx_exact_save": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_int32]),
    "gprx_exact_load": (C.c_int32, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "gprx_persist_inspect": (C.c_int32, [C.c_char_p, C.POINTER(PersistInfo)]),
    "gprx_persist_read": (C.c_int32, [C.c_char_p, C.POINTER(KernelNode), D, D, D, D, D, U64]),
    "gprx_persist_write": (C.c_int32, [C.c_char_p, D, C.c_uint64, C.c_uint64, D, C.POINTER(KernelNode), C.c_int32,
                                       D, C.c_int32, C.POINTER(Options), D, D, C.c_int32, C.c_double, U64,
                                       C.c_uint64]),
    "gprx_exact_loo": (C.c_int32, [C.c_void_p, C.c_int32, D, D]),
    "gprx_exact_predict_covariance": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_int32, D, D]),
    "gprx_exact_sample": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_int32, C.c_uint64, C.c_uint64, D]),
    "gprx_sgpr_insert_inducing": (C.c_int32, [C.c_void_p, D, U64]),
    "gprx_sgpr_delete_inducing": (C.c_int32, [C.c_void_p, C.c_uint64]),
    "gprx_sgpr_m": (C.c_uint64, [C.c_void_p]),
    "gprx_sgpr_inducing_ids": (C.c_int32, [C.c_void_p, U64, C.c_uint64]),
    "gprx_sgpr_shard_sizes": (C.c_int32, [C.c_void_p, U64, U64]),
    "gprx_sgpr_shard_assemble": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_void_p]),
    "gprx_sgpr_shard_nlml": (C.c_int32, [C.c_void_p, C.c_void_p, D, C.c_void_p]),
    "gprx_sgpr_shard_gradient": (C.c_int32, [C.c_void_p, C.c_void_p, D]),
    "gprx_batch_autotune": (C.c_int32, [C.c_void_p, D, C.c_uint64]),
    "gprx_batch_set_schedule": (C.c_int32, [C.c_void_p, I32]),
    "gprx_batch_schedule": (C.c_int32, [C.c_void_p, I32, C.POINTER(C.c_float), I32]),
    "gprx_server_options_default": (None, [C.POINTER(ServerOptions)]),
    "gprx_server_create": (C.c_int32, [C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "gprx_server_destroy": (C.c_int32, [C.c_void_p]),
    "gprx_server_fit": (C.c_int32, [C.c_void_p, D, C.c_uint64, C.c_uint64, D, C.POINTER(KernelNode), C.c_int32, D,
                                    C.c_int32, C.POINTER(Options), C.POINTER(LbfgsOptions), C.c_int32, U64]),
    "gprx_server_predict": (C.c_int32, [C.c_void_p, C.c_uint64, D, C.c_uint64, C.c_uint64, C.c_int32, D, D, U64]),
    "gprx_server_add": (C.c_int32, [C.c_void_p, C.c_uint64, D, D, C.c_uint64, C.c_uint64, U64, U64]),
    "gprx_server_remove": (C.c_int32, [C.c_void_p, C.c_uint64, U64, C.c_uint64, U64]),
    "gprx_server_wait": (C.c_int32, [C.c_void_p, C.c_uint64, C.POINTER(RequestInfo)]),
    "gprx_server_stats": (C.c_int32, [C.c_void_p, C.POINTER(ServerStats)]),
    "gprx_probe_dgemm": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, D]),
    "gprx_probe_potrf": (C.c_int32, [C.c_int32, C.c_int32, D]),
    "gprx_probe_emu_gemm": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, D]),
    "gprx_rng_seed": (None, [C.POINTER(Rng), C.c_uint64]),
    "gprx_rng_next_u64": (C.c_uint64, [C.POINTER(Rng)]),
    "gprx_rng_unit": (C.c_double, [C.POINTER(Rng)]),
    "gprx_rng_up_to": (C.c_uint64, [C.POINTER(Rng), C.c_uint64]),
    "gprx_rng_normal": (C.c_double, [C.POINTER(Rng)]),
    "gprx_rng_fill_unit": (None, [C.POINTER(Rng), D, C.c_uint64]),
    "gprx_rng_fill_normal": (None, [C.POINTER(Rng), D, C.c_uint64]),
    "gprx_rng_subset": (C.c_int32, [C.POINTER(Rng), C.c_uint64, C.c_uint64, U64]),
}


def lib():
    """The loaded library.  Raises when it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libgprx_cuda.so is not built (%s); run `python -m gprx_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def declared_symbols():
    """Every function name include/gprx_cuda.h declares."""
    import re
    hdr = os.path.join(os.path.dirname(PKG), "include", "gprx_cuda.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(gprx_[a-z0-9_]+)\s*\(", text)))


def ptr(a):
    return a.ctypes.data_as(D) if a is not None else None


def f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


def last_error():
    info = ErrorInfo()
    lib().gprx_last_error(C.byref(info))
    return info
