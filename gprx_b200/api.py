"""The gprx model API over the CUDA backend.

Mirrors gprx 0.2.0's public surface for the exact / VFE path
(src/lib.rs:33-55): `KernelSpec` trees built from `RbfKernel`,
`RbfArdKernel`, `ConstantKernel`, `PeriodicKernel` with `+` and `*`;
`GaussianLikelihood`; `Gpr` (trainer) → `FittedGpr` → `OnlineGpr`;
`Lbfgs` / `Fixed` optimizers; `PredictOptions` / `VarianceKind` /
`Prediction`; typed `GprError`s (src/error.rs).  Points are column-major
(`x[i + f*n_rows]`), as in the reference.  Every computation runs in
libgprx_cuda.so; this module only checks arguments and maps errors.
"""

import ctypes as C
import enum
import math

import numpy as np

from . import _lib as L


# ---------------------------------------------------------------------------
# errors (src/error.rs:308-500)
# ---------------------------------------------------------------------------
class GprError(Exception):
    """Base of every error the backend reports."""

    def __init__(self, message, status=None, info=None):
        super().__init__(message)
        self.status = status
        self.info = info


class CholeskyFailed(GprError):
    """GprError::CholeskyFailed { jitter, matrix_size, stage }."""

    @property
    def jitter(self):
        return self.info.jitter

    @property
    def matrix_size(self):
        return self.info.matrix_size

    @property
    def stage(self):
        return CholeskyStage(self.info.stage)


class NonFiniteKernelValue(GprError):
    pass


class ShapeMismatch(GprError):
    pass


class IndexOutOfRange(GprError):
    pass


class InsufficientData(GprError):
    pass


class InvalidHyperparameter(GprError):
    pass


class NonFiniteInput(GprError):
    pass


class EmptyInput(GprError):
    pass


class InvalidConfig(GprError):
    pass


class OptimizationNotConverged(GprError):
    pass


class CudaError(GprError):
    pass


class DeviceTimeout(GprError):
    pass


class NonPositiveDefiniteMatrix(GprError):
    """GprError::NonPositiveDefiniteMatrix (a leave-one-out [K⁻¹]_ii ≤ 0)."""


class PersistFailed(GprError):
    """GprError::PersistFailed (a saved model that cannot be read or written)."""


class UnsupportedPersistVersion(GprError):
    """GprError::UnsupportedPersistVersion."""


class OutOfDeviceMemory(GprError):
    pass


_ERRORS = {
    L.CHOLESKY_FAILED: CholeskyFailed,
    L.NONFINITE_KERNEL: NonFiniteKernelValue,
    L.SHAPE_MISMATCH: ShapeMismatch,
    L.INVALID_POINT_ID: IndexOutOfRange,
    L.INSUFFICIENT_DATA: InsufficientData,
    L.CUDA_ERROR: CudaError,
    L.TIMEOUT: DeviceTimeout,
    L.INVALID_HYPERPARAMETER: InvalidHyperparameter,
    L.NONFINITE_INPUT: NonFiniteInput,
    L.EMPTY_INPUT: EmptyInput,
    L.OUT_OF_MEMORY: OutOfDeviceMemory,
    L.INVALID_CONFIG: InvalidConfig,
    L.NOT_CONVERGED: OptimizationNotConverged,
    L.INVALID_ARGUMENT: ShapeMismatch,
    L.CAPACITY: InvalidConfig,
    L.NOT_POSITIVE_DEFINITE: NonPositiveDefiniteMatrix,
    L.PERSIST_FAILED: PersistFailed,
    L.UNSUPPORTED_PERSIST_VERSION: UnsupportedPersistVersion,
}


def check(status):
    if status == L.OK:
        return
    info = L.last_error()
    cls = _ERRORS.get(status, GprError)
    raise cls(info.message.decode(errors="replace") or "status %d" % status, status, info)


class CholeskyStage(enum.IntEnum):
    Fit = 0
    Predict = 1
    OnlineInsert = 2
    OnlineDelete = 3


# ---------------------------------------------------------------------------
# kernels (src/kernel/)
# ---------------------------------------------------------------------------
DEFAULT_LO, DEFAULT_HI = 1e-5, 1e5  # Interval::DEFAULT_POSITIVE (src/param.rs:91)


def _positive(v, what):
    v = float(v)
    if not (math.isfinite(v) and DEFAULT_LO < v < DEFAULT_HI):
        raise InvalidHyperparameter("%s must be in (1e-5, 1e5), got %r" % (what, v))
    return v


class KernelSpec:
    """A kernel tree: a leaf, or a Sum / Product of trees (flattened)."""

    def __init__(self, kind, children=(), params=(), dims=0):
        self.kind = kind
        self.children = list(children)
        self._params = list(params)  # log θ of a leaf
        self.dims = dims

    # tree building -------------------------------------------------------
    def _flat(self, op):
        return self.children if self.kind == op else [self]

    def __add__(self, other):
        return KernelSpec(L.NODE_SUM, self._flat(L.NODE_SUM) + other._flat(L.NODE_SUM))

    def __mul__(self, other):
        return KernelSpec(L.NODE_PRODUCT, self._flat(L.NODE_PRODUCT) + other._flat(L.NODE_PRODUCT))

    # parameters (log space, depth-first) ------------------------------------
    def num_params(self):
        if self.kind in (L.NODE_SUM, L.NODE_PRODUCT):
            return sum(c.num_params() for c in self.children)
        return len(self._params)

    def get_params(self):
        if self.kind in (L.NODE_SUM, L.NODE_PRODUCT):
            out = []
            for c in self.children:
                out += c.get_params()
            return out
        return list(self._params)

    def set_params(self, params):
        params = list(params)
        if len(params) != self.num_params():
            raise ShapeMismatch("expected %d parameters, got %d" % (self.num_params(), len(params)))
        if self.kind in (L.NODE_SUM, L.NODE_PRODUCT):
            at = 0
            for c in self.children:
                k = c.num_params()
                c.set_params(params[at:at + k])
                at += k
        else:
            for p in params:
                _positive(math.exp(p), "parameter")
            self._params = params

    def nodes(self):
        """Prefix node list for the C ABI."""
        if self.kind in (L.NODE_SUM, L.NODE_PRODUCT):
            out = [(self.kind, len(self.children))]
            for c in self.children:
                out += c.nodes()
            return out
        return [(self.kind, self.dims)]

    def node_array(self):
        ns = self.nodes()
        arr = (L.KernelNode * len(ns))()
        for i, (k, a) in enumerate(ns):
            arr[i].kind = k
            arr[i].arg = a
        return arr, len(ns)

    def input_dim(self):
        if self.kind == L.LEAF_RBF_ARD:
            return self.dims
        for c in self.children:
            d = c.input_dim()
            if d:
                return d
        return 0

    def copy(self):
        k = KernelSpec(self.kind, [c.copy() for c in self.children], self._params, self.dims)
        return k

    @staticmethod
    def from_nodes(nodes, log_theta):
        """The tree of a prefix node list [(kind, arg), …] with its log θ."""
        it = iter([(int(k), int(a)) for k, a in nodes])
        th = [float(v) for v in log_theta]

        def build():
            kind, arg = next(it)
            if kind in (L.NODE_SUM, L.NODE_PRODUCT):
                return KernelSpec(kind, [build() for _ in range(arg)])
            take = arg if kind == L.LEAF_RBF_ARD else (2 if kind == L.LEAF_PERIODIC else 1)
            params = [th.pop(0) for _ in range(take)]
            return KernelSpec(kind, params=params, dims=arg if kind == L.LEAF_RBF_ARD else 0)

        return build()


def RbfKernel(lengthscale):
    """k = exp(−r²/(2ℓ²)) (src/kernel/rbf.rs:18)."""
    return KernelSpec(L.LEAF_RBF, params=[math.log(_positive(lengthscale, "lengthscale"))])


def RbfArdKernel(lengthscales):
    """k = exp(−½ Σ_f Δ_f²/ℓ_f²) (src/kernel/rbf_ard.rs:16)."""
    ls = [_positive(v, "lengthscale") for v in lengthscales]
    if not ls:
        raise EmptyInput("RbfArdKernel needs at least one lengthscale")
    return KernelSpec(L.LEAF_RBF_ARD, params=[math.log(v) for v in ls], dims=len(ls))


def ConstantKernel(constant):
    """k = c (src/kernel/constant.rs:12)."""
    return KernelSpec(L.LEAF_CONSTANT, params=[math.log(_positive(constant, "constant"))])


def PeriodicKernel(lengthscale, period):
    """k = exp(−2 sin²(π r / p)/ℓ²) (src/kernel/periodic.rs:598)."""
    return KernelSpec(L.LEAF_PERIODIC, params=[math.log(_positive(lengthscale, "lengthscale")),
                                               math.log(_positive(period, "period"))])


class GaussianLikelihood:
    """θ = log σn² (src/likelihood.rs:72-194)."""

    def __init__(self, noise_variance):
        self.log_noise_variance = math.log(_positive(noise_variance, "noise variance"))

    @property
    def noise_variance(self):
        return math.exp(self.log_noise_variance)


# ---------------------------------------------------------------------------
# optimizers (src/optimizer/)
# ---------------------------------------------------------------------------
class Lbfgs:
    """L-BFGS with the Moré–Thuente line search (src/optimizer/lbfgs.rs:28-172)."""

    def __init__(self, max_iterations=100, tolerance=math.sqrt(2.220446049250313e-16), history_size=10,
                 restarts=0, seed=0):
        if not (math.isfinite(tolerance) and tolerance >= 0.0):
            raise InvalidConfig("L-BFGS gradient tolerance must be finite and >= 0")
        self.max_iterations = int(max_iterations)
        self.tolerance = float(tolerance)
        self.history_size = int(history_size)
        self.restarts = int(restarts)
        self.seed = int(seed)

    def with_max_iterations(self, n):
        self.max_iterations = int(n)
        return self

    def with_tolerance(self, tol):
        return Lbfgs(self.max_iterations, tol, self.history_size, self.restarts, self.seed)

    def with_history_size(self, m):
        self.history_size = int(m)
        return self

    def with_restarts(self, n, seed):
        self.restarts = int(n)
        self.seed = int(seed)
        return self

    def _c(self):
        o = L.LbfgsOptions()
        L.lib().gprx_lbfgs_options_default(C.byref(o))
        o.max_iterations = self.max_iterations
        o.tolerance = self.tolerance
        o.history_size = self.history_size
        o.restarts = self.restarts
        o.seed = self.seed
        return o


class TrustRegion:
    """Trust region with the Steihaug subproblem over the analytic Hessian, in
    logit coordinates (src/optimizer/trust_region.rs:19-130).  Exact models
    only: the Sgpr Hessian is not part of this backend."""

    def __init__(self, max_iterations=100, tolerance=math.sqrt(2.220446049250313e-16), initial_radius=1.0,
                 max_radius=100.0, restarts=0, seed=0):
        if not (math.isfinite(tolerance) and tolerance >= 0.0):
            raise InvalidConfig("trust-region gradient tolerance must be finite and >= 0")
        self._check_radii(initial_radius, max_radius)
        self.max_iterations = int(max_iterations)
        self.tolerance = float(tolerance)
        self.initial_radius = float(initial_radius)
        self.max_radius = float(max_radius)
        self.restarts = int(restarts)
        self.seed = int(seed)

    @staticmethod
    def _check_radii(initial_radius, max_radius):
        if not (math.isfinite(initial_radius) and math.isfinite(max_radius) and initial_radius > 0.0
                and initial_radius <= max_radius):
            raise InvalidConfig("trust radii must satisfy 0 < initial <= max and be finite")

    def with_max_iterations(self, n):
        self.max_iterations = int(n)
        return self

    def with_tolerance(self, tol):
        return TrustRegion(self.max_iterations, tol, self.initial_radius, self.max_radius, self.restarts, self.seed)

    def with_radii(self, initial_radius, max_radius):
        self._check_radii(initial_radius, max_radius)
        self.initial_radius = float(initial_radius)
        self.max_radius = float(max_radius)
        return self

    def with_restarts(self, n, seed):
        self.restarts = int(n)
        self.seed = int(seed)
        return self

    def _c(self):
        o = L.TrustRegionOptions()
        L.lib().gprx_trust_region_options_default(C.byref(o))
        o.max_iterations = self.max_iterations
        o.tolerance = self.tolerance
        o.initial_radius = self.initial_radius
        o.max_radius = self.max_radius
        o.restarts = self.restarts
        o.seed = self.seed
        return o


class Fixed:
    """No optimization: factor at the given θ (src/optimizer/mod.rs)."""


class VarianceKind(enum.IntEnum):
    Latent = L.VARIANCE_LATENT
    Observation = L.VARIANCE_OBSERVATION


class PredictOptions:
    def __init__(self, variance_kind=VarianceKind.Observation):
        self.variance_kind = VarianceKind(variance_kind)


class Prediction:
    """Predictive mean and diagonal variance (src/prediction.rs)."""

    def __init__(self, mean, variance, variance_kind):
        self.mean = mean
        self.variance = variance
        self.variance_kind = variance_kind


class PredictiveCovariance:
    """Predictive mean and the q×q query covariance (src/prediction.rs:172)."""

    def __init__(self, mean, covariance, variance_kind):
        self.mean = mean
        self.covariance = covariance  # q×q ndarray (symmetric)
        self.variance_kind = variance_kind


class Precision(enum.IntEnum):
    Fp64 = L.PRECISION_FP64
    Mixed = L.PRECISION_MIXED


def _check_points(x, n_rows, n_cols):
    x = L.f64(x)
    if n_rows <= 0:
        raise EmptyInput("no points")
    if n_cols <= 0:
        raise EmptyInput("no features")
    if x.size != n_rows * n_cols:
        raise ShapeMismatch("x has %d values, expected %d×%d" % (x.size, n_rows, n_cols))
    if not np.all(np.isfinite(x)):
        raise NonFiniteInput("non-finite x")
    return x


# ---------------------------------------------------------------------------
# exact GPR (src/gpr/)
# ---------------------------------------------------------------------------
class JitterPolicy:
    """The Cholesky stabilizer (src/policy.rs:130-397): fixed(j) retries once
    with j after an unregularized failure; adaptive(initial, multiplier,
    max_retries, max_jitter) retries with a growing sequence."""

    def __init__(self, kind, initial, multiplier, max_retries, max_jitter):
        self.kind, self.initial, self.multiplier = int(kind), float(initial), float(multiplier)
        self.max_retries, self.max_jitter = int(max_retries), float(max_jitter)

    @staticmethod
    def fixed(jitter):
        if not (math.isfinite(jitter) and jitter >= 0.0):
            raise InvalidConfig("jitter must be finite and non-negative, got %r" % jitter)
        return JitterPolicy(0, jitter, 1.0, 0, jitter)

    @staticmethod
    def adaptive(initial, multiplier, max_retries, max_jitter):
        if not (math.isfinite(initial) and initial > 0.0):
            raise InvalidConfig("adaptive initial jitter must be finite and positive, got %r" % initial)
        if not (math.isfinite(multiplier) and multiplier > 1.0):
            raise InvalidConfig("adaptive jitter multiplier must be finite and greater than 1, got %r" % multiplier)
        if int(max_retries) < 1:
            raise InvalidConfig("adaptive jitter max_retries must be at least 1")
        if not (math.isfinite(max_jitter) and max_jitter >= initial):
            raise InvalidConfig("adaptive max_jitter must be finite and at least initial (%r), got %r"
                                % (initial, max_jitter))
        return JitterPolicy(1, initial, multiplier, max_retries, max_jitter)

    def _tuple(self):
        return (self.kind, self.initial, self.multiplier, self.max_retries, self.max_jitter)

    def __eq__(self, other):
        return isinstance(other, JitterPolicy) and self._tuple() == other._tuple()


class KernelExp(enum.IntEnum):
    """exp in the kernel walks (src/policy.rs:104-110).  The device computes
    the FP64 exp; FastApprox (gprx's degree-7 polynomial) is not built."""
    Accurate = 0
    FastApprox = 1


class DistanceCachePolicy(enum.IntEnum):
    """Whether the host reference caches pairwise distances; the device path
    recomputes them inside each fill, so this is recorded only."""
    Uncached = 0
    Cached = 1


class CholeskyBuffer(enum.IntEnum):
    """Whether the host reference keeps L beside W; the device path keeps a
    dedicated inverse buffer, so this is recorded only."""
    Reuse = 0
    Retain = 1


class _TrainerPolicies:
    """The trainer's policy setters shared by Gpr and Sgpr (src/gpr/trainer.rs)."""

    def with_jitter_policy(self, policy):
        self.jitter = policy._tuple()
        return self

    def jitter_policy(self):
        if self.jitter is None:
            return JitterPolicy.fixed(0.0)
        return JitterPolicy(*self.jitter)

    def with_math(self, mode):
        mode = KernelExp(mode)
        if mode != KernelExp.Accurate:
            raise InvalidConfig("KernelExp.FastApprox is not built on the device; the kernel walks use FP64 exp")
        self._math = mode
        return self

    def math(self):
        return getattr(self, "_math", KernelExp.Accurate)

    def with_prefer_memory(self):
        self._cache, self._buffer = DistanceCachePolicy.Uncached, CholeskyBuffer.Reuse
        return self

    def with_prefer_speed(self):
        self._cache, self._buffer = DistanceCachePolicy.Cached, CholeskyBuffer.Retain
        return self

    def distance_cache_policy(self):
        return getattr(self, "_cache", DistanceCachePolicy.Cached)

    def cholesky_buffer(self):
        return getattr(self, "_buffer", CholeskyBuffer.Retain)

    def num_params(self):
        return self.kernel.num_params() + 1

    def get_params(self):
        return np.array(self.kernel.get_params() + [self.likelihood.log_noise_variance])

    def set_params(self, params):
        params = list(params)
        if len(params) != self.num_params():
            raise ShapeMismatch("expected %d parameters, got %d" % (self.num_params(), len(params)))
        self.kernel.set_params(params[:-1])
        self.likelihood = GaussianLikelihood(math.exp(params[-1]))

    def to_kernel(self):
        return self.kernel.copy()


class Gpr(_TrainerPolicies):
    """Exact GPR trainer (src/gpr/trainer.rs:533-613)."""

    def __init__(self, kernel, likelihood, optimizer=None, precision=Precision.Fp64, device=0):
        self.kernel = kernel
        self.likelihood = likelihood
        self.optimizer = optimizer if optimizer is not None else Lbfgs()
        self.precision = Precision(precision)
        self.device = device
        self.jitter = None  # (kind, initial, multiplier, retries, max); None = fixed(0)

    def with_optimizer(self, opt):
        g = Gpr(self.kernel, self.likelihood, opt, self.precision, self.device)
        g.jitter = self.jitter
        return g

    def with_precision(self, precision):
        g = Gpr(self.kernel, self.likelihood, self.optimizer, precision, self.device)
        g.jitter = self.jitter
        return g

    def with_jitter_fixed(self, jitter):
        self.jitter = (0, float(jitter), 1.0, 0, float(jitter))
        return self

    def with_jitter_adaptive(self, initial, multiplier, max_retries, max_jitter):
        self.jitter = (1, float(initial), float(multiplier), int(max_retries), float(max_jitter))
        return self

    def _options(self):
        o = L.Options()
        L.lib().gprx_options_default(C.byref(o))
        o.precision = int(self.precision)
        o.device = int(self.device)
        if self.jitter is not None:
            o.jitter_kind, o.jitter_initial, o.jitter_multiplier, o.jitter_max_retries, o.jitter_max = self.jitter
        return o

    def _create(self, x, n_rows, n_cols, y):
        x = _check_points(x, n_rows, n_cols)
        y = L.f64(y)
        if y.size != n_rows:
            raise ShapeMismatch("y has %d values, expected %d" % (y.size, n_rows))
        if not np.all(np.isfinite(y)):
            raise NonFiniteInput("non-finite y")
        nodes, nn = self.kernel.node_array()
        theta = L.f64(self.kernel.get_params() + [self.likelihood.log_noise_variance])
        h = C.c_void_p()
        opt = self._options()
        check(L.lib().gprx_exact_create(L.ptr(x), n_rows, n_cols, L.ptr(y), nodes, nn, L.ptr(theta), theta.size,
                                        C.byref(opt), C.byref(h)))
        return FittedGpr(h, n_cols, self.kernel.copy(), self)

    def factor(self, x, n_rows, n_cols, y):
        """Factor at the given θ (Gpr<Fixed>::factor)."""
        f = self._create(x, n_rows, n_cols, y)
        check(L.lib().gprx_exact_factor(f._h))
        f.optimizer = Fixed()
        return f

    def fit(self, x, n_rows, n_cols, y):
        """Optimize θ with the trainer's optimizer, then factor at the best θ."""
        f = self._create(x, n_rows, n_cols, y)
        if isinstance(self.optimizer, Fixed):
            check(L.lib().gprx_exact_factor(f._h))
            return f
        rep = L.FitReport()
        opt = self.optimizer._c()
        if isinstance(self.optimizer, TrustRegion):
            check(L.lib().gprx_exact_fit_trust_region(f._h, C.byref(opt), C.byref(rep)))
        else:
            check(L.lib().gprx_exact_fit(f._h, C.byref(opt), C.byref(rep)))
        f.report = rep
        return f


class FittedGpr:
    """A factored exact GPR (src/gpr/fitted.rs)."""

    def __init__(self, handle, d, kernel, trainer=None):
        self._h = handle
        self.d = d
        self.kernel = kernel
        self.report = None
        self._trainer = trainer
        self.optimizer = trainer.optimizer if trainer is not None else Fixed()

    def x(self):
        """Training features, column-major n × d (FittedGpr::x, src/gpr/fitted.rs:1091)."""
        n = self.n()
        x = np.zeros(n * self.d)
        y = np.zeros(n)
        check(L.lib().gprx_exact_data(self._h, L.ptr(x), L.ptr(y)))
        return x

    def y(self):
        """Training targets (FittedGpr::y, src/gpr/fitted.rs:324)."""
        n = self.n()
        x = np.zeros(n * self.d)
        y = np.zeros(n)
        check(L.lib().gprx_exact_data(self._h, L.ptr(x), L.ptr(y)))
        return y

    def likelihood(self):
        """The Gaussian likelihood at the current σn² (src/gpr/fitted.rs:308)."""
        return GaussianLikelihood(math.exp(self.get_params()[-1]))

    def to_kernel(self):
        """The kernel at the current θ (FittedGpr::kernel, src/gpr/fitted.rs:836)."""
        k = self.kernel.copy()
        k.set_params(list(self.get_params()[:-1]))
        return k

    def with_optimizer(self, optimizer):
        """Replaces the optimizer used by a later refit (src/gpr/fitted.rs:328)."""
        self.optimizer = optimizer
        return self

    def refit(self):
        """Re-runs the stored optimizer on the stored data from the current θ;
        with Fixed, refactors at the current θ (src/gpr/fitted.rs:1146-1166)."""
        if isinstance(self.optimizer, Fixed):
            check(L.lib().gprx_exact_factor(self._h))
            return
        rep = L.FitReport()
        opt = self.optimizer._c()
        if isinstance(self.optimizer, TrustRegion):
            check(L.lib().gprx_exact_fit_trust_region(self._h, C.byref(opt), C.byref(rep)))
        else:
            check(L.lib().gprx_exact_fit(self._h, C.byref(opt), C.byref(rep)))
        self.report = rep

    def into_trainer(self):
        """Drops the factor and the data; returns a trainer with the current
        kernel, likelihood, optimizer and options (src/gpr/fitted.rs:291-306)."""
        t = self._trainer
        g = Gpr(self.to_kernel(), self.likelihood(), self.optimizer,
                t.precision if t is not None else Precision.Fp64, t.device if t is not None else 0)
        if t is not None:
            g.jitter = t.jitter
        self.__del__()
        return g

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                L.lib().gprx_exact_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def num_params(self):
        return int(L.lib().gprx_exact_num_params(self._h))

    def get_params(self):
        p = np.zeros(self.num_params())
        check(L.lib().gprx_exact_get_params(self._h, L.ptr(p), p.size))
        return p

    def set_params(self, params):
        p = L.f64(params)
        check(L.lib().gprx_exact_set_params(self._h, L.ptr(p), p.size))

    def value_and_gradient(self, params):
        """NLML and its gradient at `params` (ExactFit::value_and_gradient_into)."""
        p = L.f64(params)
        if p.size != self.num_params():
            raise ShapeMismatch("expected %d parameters" % self.num_params())
        v = np.zeros(1)
        g = np.zeros(p.size)
        check(L.lib().gprx_exact_eval(self._h, L.ptr(p), p.size, L.ptr(v), L.ptr(g)))
        return float(v[0]), g

    def value(self, params):
        p = L.f64(params)
        v = np.zeros(1)
        check(L.lib().gprx_exact_eval(self._h, L.ptr(p), p.size, L.ptr(v), None))
        return float(v[0])

    def value_gradient_hessian(self, params):
        """NLML, gradient and Hessian of one evaluation at `params`
        (TwiceDifferentiable::value_gradient_hessian_into, src/objective.rs:427)."""
        p = L.f64(params)
        if p.size != self.num_params():
            raise ShapeMismatch("expected %d parameters" % self.num_params())
        v = np.zeros(1)
        g = np.zeros(p.size)
        h = np.zeros(p.size * p.size)
        check(L.lib().gprx_exact_value_gradient_hessian(self._h, L.ptr(p), p.size, L.ptr(v), L.ptr(g), L.ptr(h)))
        return float(v[0]), g, h.reshape(p.size, p.size)

    def hessian(self, params):
        """Hessian of the NLML at `params`, p × p (FittedGpr::hessian_into,
        src/gpr/fitted.rs:665; src/gpr/exact_fit.rs:443-637)."""
        p = L.f64(params)
        if p.size != self.num_params():
            raise ShapeMismatch("expected %d parameters" % self.num_params())
        out = np.zeros(p.size * p.size)
        check(L.lib().gprx_exact_hessian(self._h, L.ptr(p), p.size, L.ptr(out)))
        return out.reshape(p.size, p.size)

    def neg_log_marginal_likelihood(self):
        v = np.zeros(1)
        check(L.lib().gprx_exact_nlml(self._h, L.ptr(v)))
        return float(v[0])

    def factor_jitter(self):
        v = np.zeros(1)
        check(L.lib().gprx_exact_factor_jitter(self._h, L.ptr(v)))
        return float(v[0])

    def alpha(self):
        n = self.n()
        out = np.zeros(n)
        check(L.lib().gprx_exact_alpha(self._h, L.ptr(out), n))
        return out

    def n(self):
        return int(L.lib().gprx_online_n(self._h))

    def predict(self, xs, n_rows, n_cols):
        return self.predict_with(xs, n_rows, n_cols, PredictOptions())

    def predict_with(self, xs, n_rows, n_cols, options):
        if n_cols != self.d:
            raise ShapeMismatch("query has %d features, model has %d" % (n_cols, self.d))
        xs = L.f64(xs)
        if xs.size != n_rows * n_cols:
            raise ShapeMismatch("xs has %d values, expected %d×%d" % (xs.size, n_rows, n_cols))
        mean = np.zeros(n_rows)
        var = np.zeros(n_rows)
        check(L.lib().gprx_exact_predict(self._h, L.ptr(xs), n_rows, int(options.variance_kind), L.ptr(mean),
                                         L.ptr(var)))
        return Prediction(mean, var, options.variance_kind)

    def _query(self, xs, n_rows, n_cols):
        if n_cols != self.d:
            raise ShapeMismatch("query has %d features, model has %d" % (n_cols, self.d))
        xs = L.f64(xs)
        if xs.size != n_rows * n_cols:
            raise ShapeMismatch("xs has %d values, expected %d×%d" % (xs.size, n_rows, n_cols))
        return xs

    def save(self, directory):
        """Writes <directory>/config.json and model.safetensors: x, y and the
        model's settings (FittedGpr::save, src/gpr/fitted.rs)."""
        check(L.lib().gprx_exact_save(self._h, str(directory).encode(), 0))

    def save_with_factor(self, directory):
        """save, plus the factor and α, so a load predicts without factoring."""
        check(L.lib().gprx_exact_save(self._h, str(directory).encode(), 1))

    def loo_predict(self):
        """Leave-one-out mean and variance at every training point
        (FittedGpr::loo_predict, src/gpr/fitted.rs:697)."""
        return self.loo_predict_with(PredictOptions())

    def loo_predict_with(self, options):
        n = self.n()
        mean = np.zeros(n)
        var = np.zeros(n)
        check(L.lib().gprx_exact_loo(self._h, int(options.variance_kind), L.ptr(mean), L.ptr(var)))
        return Prediction(mean, var, options.variance_kind)

    def predict_covariance(self, xs, n_rows, n_cols):
        """Mean and query covariance K** − VᵀV (src/gpr/fitted.rs:971)."""
        return self.predict_covariance_with(xs, n_rows, n_cols, PredictOptions())

    def predict_covariance_with(self, xs, n_rows, n_cols, options):
        xs = self._query(xs, n_rows, n_cols)
        mean = np.zeros(n_rows)
        cov = np.zeros(n_rows * n_rows)
        check(L.lib().gprx_exact_predict_covariance(self._h, L.ptr(xs), n_rows, int(options.variance_kind),
                                                    L.ptr(mean), L.ptr(cov)))
        return PredictiveCovariance(mean, cov.reshape(n_rows, n_rows, order="F"), options.variance_kind)

    def sample(self, xs, n_rows, n_cols, n_draws, seed):
        """n_draws posterior draws, column-major n_rows × n_draws
        (src/gpr/fitted.rs:1038)."""
        return self.sample_with(xs, n_rows, n_cols, PredictOptions(), n_draws, seed)

    def sample_with(self, xs, n_rows, n_cols, options, n_draws, seed):
        xs = self._query(xs, n_rows, n_cols)
        out = np.zeros(n_rows * n_draws)
        check(L.lib().gprx_exact_sample(self._h, L.ptr(xs), n_rows, int(options.variance_kind), int(n_draws),
                                        int(seed), L.ptr(out)))
        return out

    def stream_ptr(self):
        """The cudaStream_t this model's kernels run on (for event timing)."""
        s = C.c_void_p()
        check(L.lib().gprx_exact_stream(self._h, C.byref(s)))
        return s.value or 0

    def set_data(self, x, y):
        """Re-uploads X and y of the same shape (gprx_exact_set_data)."""
        x = L.f64(x)
        y = L.f64(y)
        check(L.lib().gprx_exact_set_data(self._h, L.ptr(x), L.ptr(y)))

    def stage_times_ms(self):
        out = np.zeros(5)
        check(L.lib().gprx_exact_stage_times(self._h, L.ptr(out)))
        return dict(zip(("fill", "factor", "inverse", "gradient", "total"), out))

    def into_online(self):
        """FittedGpr::into_online (src/gpr/fitted.rs:757-765)."""
        check(L.lib().gprx_online_begin(self._h))
        on = OnlineGpr(self._h, self.d, self.kernel, self._trainer)
        on.optimizer = self.optimizer
        self._h = None
        return on


class OnlineGpr(FittedGpr):
    """Exact GPR with O(n²) point insert / delete (src/gpr/online.rs)."""

    def insert(self, x_new, y_new):
        x = L.f64(x_new)
        if x.size != self.d:
            raise ShapeMismatch("point has %d features, model has %d" % (x.size, self.d))
        pid = C.c_uint64(0)
        check(L.lib().gprx_online_insert(self._h, L.ptr(x), float(y_new), C.byref(pid)))
        return int(pid.value)

    def delete(self, point_id):
        check(L.lib().gprx_online_delete(self._h, int(point_id)))

    def point_ids(self):
        n = self.n()
        out = np.zeros(n, dtype=np.uint64)
        check(L.lib().gprx_online_point_ids(self._h, out.ctypes.data_as(L.U64), n))
        return out


# ---------------------------------------------------------------------------
# VFE sparse GPR (src/sgpr/)
# ---------------------------------------------------------------------------
class Sgpr(_TrainerPolicies):
    """VFE sparse GPR trainer (src/sgpr/model.rs:448-579).  The K_mm factor
    retries with JitterPolicy::adaptive(1e-8, 10, 5, 1e-3) by default."""

    def __init__(self, kernel, likelihood, optimizer=None, precision=Precision.Fp64, device=0):
        self.kernel = kernel
        self.likelihood = likelihood
        self.optimizer = optimizer if optimizer is not None else Lbfgs()
        self.precision = Precision(precision)
        self.device = device
        self.jitter = None  # None = JitterPolicy.adaptive(1e-8, 10, 5, 1e-3)

    def with_optimizer(self, opt):
        g = Sgpr(self.kernel, self.likelihood, opt, self.precision, self.device)
        g.jitter = self.jitter
        return g

    def jitter_policy(self):
        if self.jitter is None:
            return JitterPolicy.adaptive(1e-8, 10.0, 5, 1e-3)
        return JitterPolicy(*self.jitter)

    def _create(self, x, n_rows, n_cols, y, z, m):
        x = _check_points(x, n_rows, n_cols)
        z = _check_points(z, m, n_cols)
        y = L.f64(y)
        if y.size != n_rows:
            raise ShapeMismatch("y has %d values, expected %d" % (y.size, n_rows))
        if not np.all(np.isfinite(y)):
            raise NonFiniteInput("non-finite y")
        nodes, nn = self.kernel.node_array()
        theta = L.f64(self.kernel.get_params() + [self.likelihood.log_noise_variance])
        o = L.Options()
        L.lib().gprx_options_default_sparse(C.byref(o))
        o.precision = int(self.precision)
        o.device = int(self.device)
        if self.jitter is not None:
            o.jitter_kind, o.jitter_initial, o.jitter_multiplier, o.jitter_max_retries, o.jitter_max = self.jitter
        h = C.c_void_p()
        check(L.lib().gprx_sgpr_create(L.ptr(x), n_rows, n_cols, L.ptr(y), L.ptr(z), m, nodes, nn, L.ptr(theta),
                                       theta.size, C.byref(o), C.byref(h)))
        return FittedSgpr(h, n_cols, self)

    def factor(self, x, n_rows, n_cols, y, z, m):
        f = self._create(x, n_rows, n_cols, y, z, m)
        check(L.lib().gprx_sgpr_factor(f._h))
        return f

    def fit(self, x, n_rows, n_cols, y, z, m):
        if isinstance(self.optimizer, TrustRegion):
            raise InvalidConfig("TrustRegion needs the Hessian, which this backend builds for exact models only")
        f = self._create(x, n_rows, n_cols, y, z, m)
        if isinstance(self.optimizer, Fixed):
            check(L.lib().gprx_sgpr_factor(f._h))
            return f
        rep = L.FitReport()
        opt = self.optimizer._c()
        check(L.lib().gprx_sgpr_fit(f._h, C.byref(opt), C.byref(rep)))
        f.report = rep
        return f


class FittedSgpr:
    """An assembled VFE model (src/sgpr/fitted.rs)."""

    def __init__(self, handle, d, trainer=None):
        self._h = handle
        self.d = d
        self.report = None
        self._trainer = trainer
        self.optimizer = trainer.optimizer if trainer is not None else Fixed()

    def set_params(self, params):
        """Writes θ and reassembles (FittedSgpr::set_params)."""
        p = L.f64(params)
        check(L.lib().gprx_sgpr_set_params(self._h, L.ptr(p), p.size))

    def likelihood(self):
        """The Gaussian likelihood at the current σn²."""
        return GaussianLikelihood(math.exp(self.get_params()[-1]))

    def to_kernel(self):
        """The kernel at the current θ."""
        if self._trainer is None:
            raise InvalidConfig("this model has no kernel description")
        k = self._trainer.kernel.copy()
        k.set_params(list(self.get_params()[:-1]))
        return k

    def with_optimizer(self, optimizer):
        """Replaces the optimizer used by a later refit."""
        self.optimizer = optimizer
        return self

    def refit(self):
        """Re-runs the stored optimizer from the current θ on the stored data
        (Fixed: reassembles at the current θ)."""
        if isinstance(self.optimizer, Fixed):
            check(L.lib().gprx_sgpr_factor(self._h))
            return
        if isinstance(self.optimizer, TrustRegion):
            raise InvalidConfig("TrustRegion needs the Hessian, which this backend builds for exact models only")
        rep = L.FitReport()
        opt = self.optimizer._c()
        check(L.lib().gprx_sgpr_fit(self._h, C.byref(opt), C.byref(rep)))
        self.report = rep

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                L.lib().gprx_sgpr_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def num_params(self):
        return int(L.lib().gprx_sgpr_num_params(self._h))

    def get_params(self):
        p = np.zeros(self.num_params())
        check(L.lib().gprx_sgpr_get_params(self._h, L.ptr(p), p.size))
        return p

    def value_and_gradient(self, params):
        p = L.f64(params)
        v = np.zeros(1)
        g = np.zeros(p.size)
        check(L.lib().gprx_sgpr_eval(self._h, L.ptr(p), p.size, L.ptr(v), L.ptr(g)))
        return float(v[0]), g

    def value(self, params):
        p = L.f64(params)
        v = np.zeros(1)
        check(L.lib().gprx_sgpr_eval(self._h, L.ptr(p), p.size, L.ptr(v), None))
        return float(v[0])

    def neg_log_marginal_likelihood(self):
        v = np.zeros(1)
        check(L.lib().gprx_sgpr_nlml(self._h, L.ptr(v)))
        return float(v[0])

    def kmm_jitter(self):
        v = np.zeros(1)
        check(L.lib().gprx_sgpr_kmm_jitter(self._h, L.ptr(v)))
        return float(v[0])

    def n(self):
        return int(L.lib().gprx_sgpr_n(self._h))

    def predict(self, xs, n_rows, n_cols):
        return self.predict_with(xs, n_rows, n_cols, PredictOptions())

    def predict_with(self, xs, n_rows, n_cols, options):
        if n_cols != self.d:
            raise ShapeMismatch("query has %d features, model has %d" % (n_cols, self.d))
        xs = L.f64(xs)
        mean = np.zeros(n_rows)
        var = np.zeros(n_rows)
        check(L.lib().gprx_sgpr_predict(self._h, L.ptr(xs), n_rows, int(options.variance_kind), L.ptr(mean),
                                        L.ptr(var)))
        return Prediction(mean, var, options.variance_kind)

    def predict_covariance(self, xs, n_rows, n_cols):
        """Mean and query covariance of the VFE posterior (src/sgpr/fitted.rs:795-850)."""
        return self.predict_covariance_with(xs, n_rows, n_cols, PredictOptions())

    def predict_covariance_with(self, xs, n_rows, n_cols, options):
        if n_cols != self.d:
            raise ShapeMismatch("query has %d features, model has %d" % (n_cols, self.d))
        xs = L.f64(xs)
        mean = np.zeros(n_rows)
        cov = np.zeros(n_rows * n_rows)
        check(L.lib().gprx_sgpr_predict_covariance(self._h, L.ptr(xs), n_rows, int(options.variance_kind),
                                                   L.ptr(mean), L.ptr(cov)))
        return PredictiveCovariance(mean, cov.reshape(n_rows, n_rows, order="F"), options.variance_kind)

    def sample(self, xs, n_rows, n_cols, n_draws, seed):
        """n_draws posterior draws, column-major n_rows × n_draws (src/sgpr/fitted.rs:855-900)."""
        return self.sample_with(xs, n_rows, n_cols, PredictOptions(), n_draws, seed)

    def sample_with(self, xs, n_rows, n_cols, options, n_draws, seed):
        if n_cols != self.d:
            raise ShapeMismatch("query has %d features, model has %d" % (n_cols, self.d))
        xs = L.f64(xs)
        out = np.zeros(n_rows * n_draws)
        check(L.lib().gprx_sgpr_sample(self._h, L.ptr(xs), n_rows, int(options.variance_kind), int(n_draws),
                                       int(seed), L.ptr(out)))
        return out

    def stream_ptr(self):
        s = C.c_void_p()
        check(L.lib().gprx_sgpr_stream(self._h, C.byref(s)))
        return s.value or 0

    def stage_times_ms(self):
        out = np.zeros(3)
        check(L.lib().gprx_sgpr_stage_times(self._h, L.ptr(out)))
        return dict(zip(("kmm_and_a", "b_and_sums", "gradient"), out))

    # -- one shard of an evaluation over n split across processes ---------
    # The model holds this process's points and the shared inducing inputs;
    # the two exchange buffers are float64 tensors on the model's device that
    # the caller sums over the processes between the calls
    # (sharded_value_and_gradient does the sequence).

    def shard_sizes(self):
        """Lengths (doubles) of the two exchange buffers."""
        a = np.zeros(1, dtype=np.uint64)
        b = np.zeros(1, dtype=np.uint64)
        check(L.lib().gprx_sgpr_shard_sizes(self._h, a.ctypes.data_as(L.U64), b.ctypes.data_as(L.U64)))
        return int(a[0]), int(b[0])

    def shard_assemble(self, params, exchange1):
        """This shard's sums over n at θ = params, written to exchange1."""
        p = L.f64(params)
        check(L.lib().gprx_sgpr_shard_assemble(self._h, L.ptr(p), p.size, C.c_void_p(exchange1.data_ptr())))

    def shard_nlml(self, exchange1, exchange2=None):
        """NLML from the summed exchange1; with exchange2, this shard's
        gradient sums are written there."""
        v = np.zeros(1)
        e2 = C.c_void_p(exchange2.data_ptr()) if exchange2 is not None else None
        check(L.lib().gprx_sgpr_shard_nlml(self._h, C.c_void_p(exchange1.data_ptr()), L.ptr(v), e2))
        return float(v[0])

    def shard_gradient(self, exchange2):
        """Gradient from the summed exchange2."""
        g = np.zeros(self.num_params())
        check(L.lib().gprx_sgpr_shard_gradient(self._h, C.c_void_p(exchange2.data_ptr()), L.ptr(g)))
        return g

    def into_online(self):
        """FittedSgpr::into_online: the same device state, now updatable."""
        on = OnlineSgpr(self._h, self.d, self._trainer)
        on.optimizer = self.optimizer
        self._h = None
        return on


class LoadedGpr:
    """LoadedGpr::load (src/persist/mod.rs): a saved exact model as a
    resident FittedGpr (factor_kind llt) or OnlineGpr (ldlt)."""

    @staticmethod
    def inspect(directory):
        info = L.PersistInfo()
        check(L.lib().gprx_persist_inspect(str(directory).encode(), C.byref(info)))
        return info

    @staticmethod
    def load(directory, device=0):
        info = LoadedGpr.inspect(directory)
        nodes = (L.KernelNode * info.n_nodes)()
        theta = np.zeros(info.n_theta)
        x = np.zeros(info.n * info.d)
        y = np.zeros(info.n)
        check(L.lib().gprx_persist_read(str(directory).encode(), nodes, L.ptr(theta), L.ptr(x), L.ptr(y), None, None,
                                        None))
        kernel = KernelSpec.from_nodes([(nd.kind, nd.arg) for nd in nodes], theta[:-1])
        h = C.c_void_p()
        check(L.lib().gprx_exact_load(str(directory).encode(), int(device), C.byref(h)))
        cls = OnlineGpr if info.factor_kind == 1 else FittedGpr
        return cls(h, int(info.d), kernel)


def sharded_value_and_gradient(shard, params, all_reduce, device=None, gradient=True):
    """VFE NLML (and gradient) over n split across processes.

    shard: this process's FittedSgpr (its points, the shared inducing
    inputs); all_reduce(t): sums the tensor t over the processes in place
    (e.g. torch.distributed.all_reduce over NCCL).  Every process returns
    the same values, equal to the unsharded evaluation's.  The exchange
    buffers are float64 tensors on `device` (the CUDA device of the model;
    the work of each call has finished when it returns, and the all-reduce
    is waited for before the next call reads its result)."""
    import torch

    n1, n2 = shard.shard_sizes()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    ex1 = torch.empty(n1, dtype=torch.float64, device=dev)
    ex2 = torch.empty(n2, dtype=torch.float64, device=dev) if gradient else None

    def reduce(t):
        all_reduce(t)
        if t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()

    shard.shard_assemble(params, ex1)
    reduce(ex1)
    nl = shard.shard_nlml(ex1, ex2)
    if not gradient:
        return nl, None
    reduce(ex2)
    return nl, shard.shard_gradient(ex2)


class OnlineSgpr(FittedSgpr):
    """VFE model with O(m²) point insert / delete (src/sgpr/online/mod.rs)."""

    def insert(self, x_new, y_new):
        x = L.f64(x_new)
        if x.size != self.d:
            raise ShapeMismatch("point has %d features, model has %d" % (x.size, self.d))
        pid = C.c_uint64(0)
        check(L.lib().gprx_sgpr_insert(self._h, L.ptr(x), float(y_new), C.byref(pid)))
        return int(pid.value)

    def delete(self, point_id):
        check(L.lib().gprx_sgpr_delete(self._h, int(point_id)))

    def point_ids(self):
        n = self.n()
        out = np.zeros(n, dtype=np.uint64)
        check(L.lib().gprx_sgpr_point_ids(self._h, out.ctypes.data_as(L.U64), n))
        return out

    def last_step_in_place(self):
        return bool(L.lib().gprx_sgpr_last_step_in_place(self._h))

    def set_inducing(self, z, m):
        """Replace the inducing set (inducing insert / delete by reassembly)."""
        z = _check_points(z, m, self.d)
        check(L.lib().gprx_sgpr_set_inducing(self._h, L.ptr(z), m))

    def m(self):
        return int(L.lib().gprx_sgpr_m(self._h))

    def inducing_ids(self):
        m = self.m()
        out = np.zeros(m, dtype=np.uint64)
        check(L.lib().gprx_sgpr_inducing_ids(self._h, out.ctypes.data_as(L.U64), m))
        return out

    def insert_inducing(self, z_new):
        """Appends one inducing point; returns its id (OnlineSgpr::insert_inducing)."""
        z = L.f64(z_new)
        if z.size != self.d:
            raise ShapeMismatch("inducing point has %d features, model has %d" % (z.size, self.d))
        iid = C.c_uint64(0)
        check(L.lib().gprx_sgpr_insert_inducing(self._h, L.ptr(z), C.byref(iid)))
        return int(iid.value)

    def delete_inducing(self, inducing_id):
        """Removes the inducing point with this id (OnlineSgpr::delete_inducing)."""
        check(L.lib().gprx_sgpr_delete_inducing(self._h, int(inducing_id)))


# ---------------------------------------------------------------------------
# batched exact GPR: many independent problems sharing one kernel tree
# ---------------------------------------------------------------------------
class BatchFit:
    """Per-problem results of GprBatch.fit."""

    def __init__(self, params, nlml, iterations, evaluations, grad_norm, converged, status):
        self.params = params            # n_problems × p, log space
        self.nlml = nlml
        self.iterations = iterations
        self.evaluations = evaluations
        self.grad_norm = grad_norm
        self.converged = converged
        self.status = status            # gprx_status per problem (0 = ok)


class GprBatch:
    """Independent exact GPs that share a kernel tree and d, evaluated in one
    persistent device launch per round; each problem is what Gpr does for one
    model (value_and_gradient, fit by L-BFGS).

    xs, ys: lists of per-problem arrays (x_i column-major n_i × d, y_i of n_i).
    """

    def __init__(self, kernel, xs, ys, d, jitter=None, device=0):
        self.kernel = kernel.copy()
        self.d = int(d)
        if len(xs) != len(ys) or len(xs) == 0:
            raise ShapeMismatch("xs and ys must be non-empty lists of the same length")
        ns = np.array([np.asarray(y).size for y in ys], dtype=np.uint64)
        x = np.concatenate([_check_points(xi, int(n), self.d) for xi, n in zip(xs, ns)])
        y = np.concatenate([L.f64(yi) for yi in ys])
        self.n = ns
        o = L.Options()
        L.lib().gprx_options_default(C.byref(o))
        o.device = int(device)
        if jitter is not None:
            o.jitter_kind, o.jitter_initial, o.jitter_multiplier, o.jitter_max_retries, o.jitter_max = jitter
        nodes, nn = self.kernel.node_array()
        self.p = self.kernel.num_params() + 1
        h = C.c_void_p()
        check(L.lib().gprx_batch_create(L.ptr(x), L.ptr(y), ns.ctypes.data_as(L.U64), ns.size, self.d, nodes, nn,
                                        self.p, C.byref(o), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().gprx_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def n_problems(self):
        return int(self.n.size)

    def _params(self, params):
        a = np.ascontiguousarray(np.asarray(params, dtype=np.float64))
        if a.shape != (self.n_problems, self.p):
            raise ShapeMismatch("params must be n_problems × %d" % self.p)
        return a

    def stream_ptr(self):
        """The handle's CUDA stream (for event timing)."""
        s = C.c_void_p()
        check(L.lib().gprx_batch_stream(self._h, C.byref(s)))
        return s.value or 0

    # size classes of the schedule (n ≤ 64, ≤ 128, …, ≤ 4096, larger) and the
    # in-CTA GEMM tile shapes (M, N, K) the autotuner chooses from
    SIZE_CLASSES = 8
    TILE_SHAPES = ((64, 128, 32), (64, 64, 32), (32, 64, 32), (32, 32, 16))

    def autotune(self, params):
        """Times every tile shape on every size class present at θ = params
        and keeps the fastest (the first evaluation or fit does this by
        itself); returns schedule()."""
        a = self._params(params)
        check(L.lib().gprx_batch_autotune(self._h, L.ptr(a), self.p))
        return self.schedule()

    def set_schedule(self, tile_of_class):
        """Fixes the tile shape index of each size class (turns tuning off)."""
        t = np.ascontiguousarray(np.asarray(tile_of_class, dtype=np.int32))
        if t.shape != (self.SIZE_CLASSES,):
            raise ShapeMismatch("one tile shape index per size class (%d)" % self.SIZE_CLASSES)
        check(L.lib().gprx_batch_set_schedule(self._h, t.ctypes.data_as(L.I32)))

    def schedule(self):
        """(tile shape per size class, tuning ms per launch [class, shape],
        whether tuning ran)."""
        t = np.zeros(self.SIZE_CLASSES, dtype=np.int32)
        ms = np.zeros((self.SIZE_CLASSES, len(self.TILE_SHAPES)), dtype=np.float32)
        tuned = np.zeros(1, dtype=np.int32)
        check(L.lib().gprx_batch_schedule(self._h, t.ctypes.data_as(L.I32), ms.ctypes.data_as(C.POINTER(C.c_float)),
                                          tuned.ctypes.data_as(L.I32)))
        return t, ms, bool(tuned[0])

    def value_and_gradient(self, params):
        """NLML, gradient and status of every problem at its own θ (row i)."""
        a = self._params(params)
        nl = np.zeros(self.n_problems)
        g = np.zeros((self.n_problems, self.p))
        st = np.zeros(self.n_problems, dtype=np.int32)
        check(L.lib().gprx_batch_eval(self._h, L.ptr(a), self.p, L.ptr(nl), g.ctypes.data_as(L.D),
                                      st.ctypes.data_as(L.I32)))
        return nl, g, st

    def fit(self, params0, optimizer=None):
        """Fits every problem by L-BFGS (the optimizers run on the device)."""
        a = self._params(params0)
        opt = (optimizer if optimizer is not None else Lbfgs())._c()
        out = np.zeros_like(a)
        reps = (L.FitReport * self.n_problems)()
        st = np.zeros(self.n_problems, dtype=np.int32)
        check(L.lib().gprx_batch_fit(self._h, L.ptr(a), self.p, C.byref(opt), out.ctypes.data_as(L.D), reps,
                                     st.ctypes.data_as(L.I32)))
        return BatchFit(out, np.array([r.nlml for r in reps]), np.array([r.iterations for r in reps]),
                        np.array([r.evaluations for r in reps]), np.array([r.grad_norm for r in reps]),
                        np.array([r.converged for r in reps], dtype=bool), st)


def predict_group(models, xs_list, qs, kind=None):
    """Mean and variance for several requests against several fitted exact
    models in one launch (gprx_exact_predict_group): request i asks
    models[i] at qs[i] points xs_list[i] (column-major qs[i] × d).  Returns a
    list of Prediction.  Every model has at most 1024 points and 16
    features, is not online, and all share d and the device."""
    k = len(models)
    if k == 0 or len(xs_list) != k or len(qs) != k:
        raise ShapeMismatch("one query array and one size per model")
    kind = VarianceKind.Observation if kind is None else kind
    hs = (C.c_void_p * k)(*[m._h.value for m in models])
    xs_a = [L.f64(x) for x in xs_list]
    for m, x, q in zip(models, xs_a, qs):
        if x.size != int(q) * m.d:
            raise ShapeMismatch("xs has %d values, expected %d×%d" % (x.size, q, m.d))
    means = [np.zeros(int(q)) for q in qs]
    vars_ = [np.zeros(int(q)) for q in qs]
    xp = (L.D * k)(*[L.ptr(x) for x in xs_a])
    mp = (L.D * k)(*[L.ptr(v) for v in means])
    vp = (L.D * k)(*[L.ptr(v) for v in vars_])
    qa = np.ascontiguousarray(np.asarray(qs, dtype=np.uint64))
    check(L.lib().gprx_exact_predict_group(hs, k, xp, qa.ctypes.data_as(L.U64), int(kind), mp, vp))
    return [Prediction(mu, v, kind) for mu, v in zip(means, vars_)]


def partition_by_cost(sizes, parts):
    """Splits problem indices 0..len(sizes)-1 into `parts` shards balanced by
    Σ n_i³ (an evaluation's work per problem is O(n_i³)): longest processing
    time first — problems by decreasing n³ (ties by index), each to the shard
    with the least work so far (ties to the lower shard).  Returns one sorted
    index array per shard; every problem is in exactly one shard."""
    sizes = np.asarray(sizes, dtype=np.int64)
    parts = int(parts)
    if parts < 1:
        raise InvalidConfig("at least one shard")
    cost = sizes.astype(np.float64) ** 3
    order = sorted(range(sizes.size), key=lambda i: (-cost[i], i))
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in order:
        k = min(range(parts), key=lambda j: (load[j], j))
        out[k].append(i)
        load[k] += cost[i]
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def sharded_batch_fit(kernel, xs, ys, d, params0, rank, world, all_gather_object, optimizer=None, device=0,
                      jitter=None, batch_factory=None):
    """GprBatch.fit over problems split across processes (one GPU each).

    Every process passes the same problem list; partition_by_cost gives
    process `rank` its shard, which it fits on `device` in one GprBatch
    (batch_factory(kernel, xs, ys, d, jitter, device) builds it; GprBatch by
    default).  all_gather_object(out_list, obj) gathers one object per process
    (torch.distributed.all_gather_object); it is the only exchange, once at
    the end.  Returns the BatchFit of all problems in their original order,
    the same on every process."""
    n = len(xs)
    if len(ys) != n or n == 0:
        raise ShapeMismatch("xs and ys must be non-empty lists of the same length")
    p0 = np.asarray(params0, dtype=np.float64)
    if p0.ndim != 2 or p0.shape[0] != n:
        raise ShapeMismatch("params0 must hold one row per problem")
    sizes = [np.asarray(y).size for y in ys]
    shard = partition_by_cost(sizes, world)[int(rank)]
    mine = None
    if shard.size:
        make = batch_factory if batch_factory is not None else (
            lambda k, x, y, dd, j, dev: GprBatch(k, x, y, dd, jitter=j, device=dev))
        b = make(kernel, [xs[i] for i in shard], [ys[i] for i in shard], d, jitter, device)
        r = b.fit(p0[shard], optimizer)
        mine = (shard, r.params, r.nlml, r.iterations, r.evaluations, r.grad_norm, r.converged, r.status)
    got = [None] * int(world)
    all_gather_object(got, mine)
    p = p0.shape[1]
    params = np.zeros((n, p))
    nlml = np.zeros(n)
    iters = np.zeros(n, dtype=np.int64)
    evals = np.zeros(n, dtype=np.int64)
    gnorm = np.zeros(n)
    conv = np.zeros(n, dtype=bool)
    status = np.full(n, -1, dtype=np.int32)
    for part in got:
        if part is None:
            continue
        idx = part[0]
        params[idx], nlml[idx], iters[idx], evals[idx] = part[1], part[2], part[3], part[4]
        gnorm[idx], conv[idx], status[idx] = part[5], part[6], part[7]
    if np.any(status < 0):
        raise InvalidConfig("a problem came back from no shard (ranks passed different problem lists?)")
    return BatchFit(params, nlml, iters, evals, gnorm, conv, status)


# ---------------------------------------------------------------------------
# serving: a request loop over resident exact models
# ---------------------------------------------------------------------------
class Server:
    """Continuous request loop on one GPU (gprx_server_*): fit, predict and
    online add/remove requests against resident models, admitted by free
    workers and the HBM budget, overlapping on the device; consecutive
    predicts of one model share a launch.  submit_* return a request id;
    wait(id) blocks until it completes and returns its info (the outputs of
    a predict / add are in the arrays submit_* returned)."""

    def __init__(self, device=0, workers=8, hbm_budget_bytes=150 << 30):
        o = L.ServerOptions()
        L.lib().gprx_server_options_default(C.byref(o))
        o.device, o.workers, o.hbm_budget_bytes = int(device), int(workers), int(hbm_budget_bytes)
        h = C.c_void_p()
        check(L.lib().gprx_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self._keep = {}  # request id → buffers the library writes on completion
        self.d = {}      # model id → d

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().gprx_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit_fit(self, kernel, likelihood, x, n, d, y, optimizer=None, precision=Precision.Fp64):
        x = _check_points(x, n, d)
        y = L.f64(y)
        nodes, nn = kernel.node_array()
        theta = L.f64(kernel.get_params() + [likelihood.log_noise_variance])
        o = L.Options()
        L.lib().gprx_options_default(C.byref(o))
        o.precision = int(precision)
        opt = optimizer if optimizer is not None else Lbfgs()
        lo = opt._c() if not isinstance(opt, Fixed) else Lbfgs()._c()
        rid = C.c_uint64()
        check(L.lib().gprx_server_fit(self._h, L.ptr(x), n, d, L.ptr(y), nodes, nn, L.ptr(theta), theta.size,
                                      C.byref(o), C.byref(lo), 0 if isinstance(opt, Fixed) else 1, C.byref(rid)))
        self.d[rid.value] = d
        return rid.value

    def submit_predict(self, model, xs, q, kind=VarianceKind.Observation):
        d = self.d[model]
        xs = _check_points(xs, q, d)
        mean = np.zeros(q)
        var = np.zeros(q)
        rid = C.c_uint64()
        check(L.lib().gprx_server_predict(self._h, model, L.ptr(xs), q, d, int(kind), L.ptr(mean), L.ptr(var),
                                          C.byref(rid)))
        self._keep[rid.value] = (mean, var)
        return rid.value, mean, var

    def submit_add(self, model, x, y, k):
        d = self.d[model]
        x = _check_points(x, k, d)
        y = L.f64(y)
        ids = np.zeros(k, dtype=np.uint64)
        rid = C.c_uint64()
        check(L.lib().gprx_server_add(self._h, model, L.ptr(x), L.ptr(y), k, d, ids.ctypes.data_as(L.U64),
                                      C.byref(rid)))
        self._keep[rid.value] = (ids,)
        return rid.value, ids

    def submit_remove(self, model, ids):
        ids = np.ascontiguousarray(np.asarray(ids, dtype=np.uint64))
        rid = C.c_uint64()
        check(L.lib().gprx_server_remove(self._h, model, ids.ctypes.data_as(L.U64), ids.size, C.byref(rid)))
        return rid.value

    def wait(self, rid):
        """Blocks until request rid completes; returns (status, info dict)."""
        info = L.RequestInfo()
        st = L.lib().gprx_server_wait(self._h, rid, C.byref(info))
        self._keep.pop(rid, None)
        return st, {"status": info.status, "model": info.model, "kind": info.kind,
                    "latency_ms": (info.end_ns - info.submit_ns) * 1e-6,
                    "queue_ms": (info.start_ns - info.submit_ns) * 1e-6, "merged": info.merged,
                    "message": info.message.decode(errors="replace")}

    def stats(self):
        s = L.ServerStats()
        check(L.lib().gprx_server_stats(self._h, C.byref(s)))
        return {"completed": s.completed, "merged_launches": s.merged_launches, "used_bytes": s.used_bytes,
                "resident_models": s.resident_models, "merged_fit_launches": s.merged_fit_launches}


# ---------------------------------------------------------------------------
# seeded RNG (src/rng.rs)
# ---------------------------------------------------------------------------
class SeededRng:
    """Xoshiro256++ seeded by SplitMix64, the reference's generator."""

    def __init__(self, seed):
        self._r = L.Rng()
        L.lib().gprx_rng_seed(C.byref(self._r), int(seed))

    def next_u64(self):
        return int(L.lib().gprx_rng_next_u64(C.byref(self._r)))

    def unit(self, count=None):
        if count is None:
            return float(L.lib().gprx_rng_unit(C.byref(self._r)))
        out = np.zeros(int(count))
        L.lib().gprx_rng_fill_unit(C.byref(self._r), L.ptr(out), out.size)
        return out

    def normal(self, count=None):
        if count is None:
            return float(L.lib().gprx_rng_normal(C.byref(self._r)))
        out = np.zeros(int(count))
        L.lib().gprx_rng_fill_normal(C.byref(self._r), L.ptr(out), out.size)
        return out

    def up_to(self, max_value):
        return int(L.lib().gprx_rng_up_to(C.byref(self._r), int(max_value)))

    def subset(self, n, count):
        out = np.zeros(int(count), dtype=np.uint64)
        check(L.lib().gprx_rng_subset(C.byref(self._r), int(n), int(count), out.ctypes.data_as(L.U64)))
        return out
