"""gprx_b200 — a B200 (sm_100a) backend for gprx's exact-GPR and VFE-SGPR
objective-and-prediction path.

The compute runs in libgprx_cuda.so (hand-written CUDA for sm_100a behind the
C ABI of include/gprx_cuda.h); this package mirrors the reference's model API
over it.  Importing works without a GPU; any computation needs the library
and a CUDA device, and fails loudly otherwise.
"""

from .api import (  # noqa: F401
    CholeskyFailed,
    CholeskyStage,
    BatchFit,
    ConstantKernel,
    CudaError,
    DeviceTimeout,
    EmptyInput,
    Fixed,
    FittedGpr,
    FittedSgpr,
    sharded_value_and_gradient,
    GaussianLikelihood,
    Gpr,
    GprBatch,
    GprError,
    IndexOutOfRange,
    InsufficientData,
    InvalidConfig,
    InvalidHyperparameter,
    KernelSpec,
    Lbfgs,
    TrustRegion,
    JitterPolicy,
    KernelExp,
    DistanceCachePolicy,
    CholeskyBuffer,
    LoadedGpr,
    PersistFailed,
    UnsupportedPersistVersion,
    NonPositiveDefiniteMatrix,
    PredictiveCovariance,
    NonFiniteInput,
    NonFiniteKernelValue,
    OnlineGpr,
    OnlineSgpr,
    OptimizationNotConverged,
    OutOfDeviceMemory,
    PeriodicKernel,
    Precision,
    Prediction,
    PredictOptions,
    RbfArdKernel,
    RbfKernel,
    SeededRng,
    Server,
    Sgpr,
    ShapeMismatch,
    VarianceKind,
)
