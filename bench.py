"""Benchmark: exact-GPR NLML + gradient evaluations per second at n = 8192.

Workload (the reference's exact objective, config "Exact Gpr,
ConstantKernel(2.0) * RbfArdKernel d = 8, n = 8192"): x ~ N(0, I₈), the eight
lengthscales log-uniform in [0.3, 3], c = 2, σn² = 0.05², y a draw from the
GP prior at those hyperparameters plus N(0, 0.05²) noise.  One step is one
NLML + gradient evaluation at a hyperparameter vector perturbed by N(0, 0.1²)
in log space (100 perturbations, cycled).  All data are synthetic, from the
restated SeededRng; no dataset is read.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
                    [--workload all|exact|c1|batched|serving|sgpr|hessian] [--impl ours|reference]

The default line's value is the mixed form (FP64 products emulated on the
int8 tensor cores); the plain FP64 form is timed beside it ("fp64") with the
largest error of the mixed results against it.  The other workloads ride in
the same line in brief: "c1" (exact RBF n = 512, d = 2: default L-BFGS fit
and a 256-point predict), "batched" (4096 ragged exact fits), "serving" (a
Poisson request stream, p50/p99), "sgpr" (VFE at n = 10⁶, m = 1024) and
"hessian" (the NLML Hessian at the exact workload's θ in both forms); each is
also available alone, in full, through --workload.  Floats in the default
line carry 4 significant digits so that the line stays within a few KB.

N > 1 runs N independent replicas (one exact problem does not shard; launched
by torchrun, one rank per GPU); `value` is the aggregate evals/s over ranks,
timed as the maximum over ranks.  `--impl reference` times the CPU
restatement of the reference's algorithm (oracle/) on the host cores, one
full n = 8192 evaluation per step; it draws its data from the Python
SynthRng below and never loads the CUDA library.
"""

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 8192
D = 8
NOISE = 0.05 ** 2
CONST = 2.0


_M64 = (1 << 64) - 1


class SynthRng:
    """Xoshiro256++ seeded by SplitMix64 with the reference's unit and
    Box–Muller normal draws (gprx src/rng.rs:10-87), in Python: the exact
    workloads' data come from here in both arms of this benchmark, so the
    reference arm never loads the CUDA library.  Scalar libm log/cos keep the
    draws bit-identical to the library's gprx_rng_* (tests/test_bench_cpu.py)."""

    def __init__(self, seed):
        x = int(seed) & _M64
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _M64
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
            s.append(z ^ (z >> 31))
        self.s = s

    def next_u64(self):
        s = self.s
        r = (s[0] + s[3]) & _M64
        r = (((r << 23) | (r >> 41)) & _M64) + s[0] & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = ((s[3] << 45) | (s[3] >> 19)) & _M64
        return r

    def _unit1(self):
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)

    def _open_unit(self):
        u = self._unit1()
        eps = 1.0 / 9007199254740992.0
        return eps if u <= eps else (1.0 - eps if u >= 1.0 - eps else u)

    def _normal1(self):
        u1 = max(self._open_unit(), 2.2250738585072014e-308)
        u2 = self._open_unit()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)

    def unit(self, count):
        return np.array([self._unit1() for _ in range(int(count))])

    def normal(self, count):
        return np.array([self._normal1() for _ in range(int(count))])


def synth(n, d, seed=0):
    """x, y, true θ for the C2 workload (seeded Xoshiro256++)."""
    rng = SynthRng(seed)
    x = rng.normal(n * d)                      # column-major n×d, N(0, 1)
    u = rng.unit(d)
    ls = np.exp(math.log(0.3) + u * (math.log(3.0) - math.log(0.3)))
    xm = x.reshape(d, n).T
    z = xm / ls
    sq = np.sum(z * z, axis=1)
    k = CONST * np.exp(-0.5 * np.maximum(sq[:, None] + sq[None, :] - 2.0 * (z @ z.T), 0.0))
    k[np.diag_indices(n)] = CONST + NOISE
    chol = np.linalg.cholesky(k)
    y = chol @ rng.normal(n)                   # prior draw plus noise (the NOISE on the diagonal)
    theta = np.array([math.log(CONST)] + list(np.log(ls)) + [math.log(NOISE)])
    return x, y, theta


def perturbations(theta, count=100, seed=1):
    rng = SynthRng(seed)
    return [theta + 0.1 * rng.normal(theta.size) for _ in range(count)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return {}


def fp64_peak_tflops(torch, dev):
    """cuBLAS DGEMM throughput on this GPU (the FP64 denominator; measured
    here because MEASURED_PEAKS.json has no FP64 figure)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def int8_peak_tops(torch, dev):
    """Dense int8 tensor throughput of this GPU through cuBLASLt
    (torch._int_mm, 8192³, int32 accumulate): the denominator of the
    emulated GEMM, whose work is int8 slice products.  None when the call
    is not available."""
    try:
        n = 8192
        a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev)
        b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev)
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        del a, b
        torch.cuda.empty_cache()
        return best
    except Exception:
        return None


def load_traffic():
    path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return None


def emu_kernel_roofline(n, peaks, traffic, int8_peak=None):
    """The dominant kernel of the mixed form, emu_gemm_kernel<7>, timed with
    CUDA events on its own stream (gprx_probe_emu_gemm) at the shape of the
    evaluation's largest product: the top-level coupling L21 = A21 X11ᵀ,
    (n/2)³.  Work per launch: 28 int8 slice products of 2·(n/2)³ ops (the
    FP64-equivalent rate is that ÷ 28).  Peak: cuBLASLt's dense int8 GEMM
    measured in the same run; without it, twice the measured dense bf16 rate
    (B200's int8 dense rate is twice its bf16 rate), else twice the fallback
    1.59 PFLOP/s."""
    from gprx_b200 import _lib as L

    h = n // 2
    out = np.zeros(5)
    st = L.lib().gprx_probe_emu_gemm(h, h, h, 7, 10, L.ptr(out))
    if st != 0 or out[0] <= 0:
        return None
    eq = 2.0 * h ** 3 / (out[0] * 1e-3) / 1e12
    achieved = 28 * eq
    bf16 = peaks.get("bf16_tflops")
    if int8_peak:
        peak, src = int8_peak, "cuBLASLt int8 GEMM 8192^3 measured in this run (torch._int_mm; of measured)"
    elif bf16:
        peak, src = 2.0 * bf16, "2 x measured dense bf16 burst (MEASURED_PEAKS.json bf16_tflops, of measured)"
    else:
        peak, src = 2.0 * 1590.0, "2 x the fallback dense bf16 1.59 PFLOP/s (of fallback)"
    return {"bound": "tensor", "kernel": "emu_gemm_kernel<7> (tcgen05.mma kind::i8, TMEM accumulators)",
            "shape": "%d^3, 7 slices (the top-level coupling product at n = %d)" % (h, n),
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s (int8 tensor ops)", "frac": achieved / peak,
            "peak_source": src, "ms_per_launch": out[0], "fp64_equivalent_tflops": eq,
            "work": "28 int8 slice products x 2 (n/2)^3 ops per launch",
            "traffic": traffic.get("emu_gemm_bytes_per_launch") if traffic else None,
            "max_rel_err_vs_dmma": out[3]}


def cpu_reference(n, d, x, y, thetas, steps, warmup):
    """Times the oracle (a CPU restatement of the reference's algorithm) on
    the full workload: each step is one NLML + gradient evaluation at n."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    lib = O.lib()
    cores = int(lib.orc_num_threads())
    nodes = [[2, 2], [12, 0], [11, d]]
    for i in range(warmup):
        O.exact_eval(nodes, thetas[i % len(thetas)], x, n, d, y)
    t0 = time.perf_counter()
    for i in range(steps):
        O.exact_eval(nodes, thetas[i % len(thetas)], x, n, d, y)
    dt = (time.perf_counter() - t0) / steps
    sample = "%d NLML+gradient evaluation(s) at n=%d, the full workload" % (steps, n)
    return 1.0 / dt, dt, cores, sample


# ---------------------------------------------------------------------------
# C1: exact RBF, n = 512, d = 2, default L-BFGS fit, then predict 256 points
# ---------------------------------------------------------------------------
C1_N, C1_D, C1_Q = 512, 2, 256


def c1_synth(seed=10):
    """x ~ U[0,10]² (column-major), y = sin(x0) + 0.5 cos(x1) + N(0, 0.1²),
    256 query points ~ U[0,10]²."""
    rng = SynthRng(seed)
    x = 10.0 * rng.unit(C1_N * C1_D)
    y = np.sin(x[:C1_N]) + 0.5 * np.cos(x[C1_N:]) + 0.1 * rng.normal(C1_N)
    xs = 10.0 * rng.unit(C1_Q * C1_D)
    return x, y, xs


def c1_measure(torch, local, steps=10, warm=3):
    """Fit + predict through the public API with host buffers (a step = one
    Gpr(RbfKernel(1.0), GaussianLikelihood(0.1)).fit by the default L-BFGS
    and one predict of mean and variance at 256 points), and the oracle beside
    it: its evaluation at n = 512 times the fit's evaluations, plus its
    prediction."""
    import gprx_b200 as gx

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    x, y, xs = c1_synth()

    def step():
        m = gx.Gpr(gx.RbfKernel(1.0), gx.GaussianLikelihood(0.1), device=local).fit(x, C1_N, C1_D, y)
        p = m.predict(xs, C1_Q, C1_D)
        return m, p

    for _ in range(warm):
        step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        m, p = step()
    dt = (time.perf_counter() - t0) / steps
    theta = np.array(m.get_params())
    evals = int(m.report.evaluations)
    # the predict alone, on the fitted model
    t0 = time.perf_counter()
    for _ in range(steps):
        m.predict(xs, C1_Q, C1_D)
    pred_ms = (time.perf_counter() - t0) / steps * 1e3
    nodes = [[10, 0]]
    t0 = time.perf_counter()
    reps = 20
    for _ in range(reps):
        O.exact_eval(nodes, theta, x, C1_N, C1_D, y)
    orc_eval = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    mo, vo = O.exact_predict(nodes, theta, x, C1_N, C1_D, y, xs, C1_Q, 1)
    orc_pred = time.perf_counter() - t0
    err = max(float(np.max(O.rel_err(p.mean, mo))), float(np.max(O.rel_err(p.variance, vo))))
    return {"value": 1.0 / dt, "unit": "fits/s", "ms_per_fit_predict": dt * 1e3, "predict_ms": pred_ms,
            "evaluations": evals, "iterations": int(m.report.iterations), "converged": bool(m.report.converged),
            "grad_norm": float(m.report.grad_norm),
            "nlml": m.neg_log_marginal_likelihood(), "predict_err_vs_oracle": err,
            "cpu_baseline": {"value": 1.0 / (evals * orc_eval + orc_pred), "unit": "fits/s",
                             "cores": int(O.lib().orc_num_threads()), "kind": "port",
                             "sample": "oracle eval x the fit's evaluations + oracle predict"}}


# ---------------------------------------------------------------------------
# batched fits (4096 ragged problems, Rbf + Periodic, d = 3)
# ---------------------------------------------------------------------------
BATCH_P = 4096
BATCH_D = 3


def batched_synth(torch, dev, count=BATCH_P, seed=3):
    """Sizes log-uniform in [32, 1024], x ~ U[0,5]³, period ~ U[10, 20]
    (shorter periods make the Euclidean-distance periodic kernel indefinite
    in 3-d), θ_true = (ℓ_rbf 1, ℓ_per 1, p, σn² 0.1); y a draw from each
    problem's GP prior (Cholesky on the device, data generation only)."""
    import gprx_b200 as gx

    rng = gx.SeededRng(seed)
    u = rng.unit(count)
    sizes = np.floor(np.exp(math.log(32) + u * (math.log(1024) - math.log(32)))).astype(np.int64)
    periods = 10.0 + 10.0 * rng.unit(count)
    xs, ys = [], []
    for n, per in zip(sizes, periods):
        x = 5.0 * rng.unit(int(n) * BATCH_D)
        z = rng.normal(int(n))
        xt = torch.from_numpy(x.reshape(BATCH_D, int(n)).T.copy()).to(dev)
        r2 = torch.cdist(xt, xt).pow(2)
        k = torch.exp(-0.5 * r2) + torch.exp(-2.0 * torch.sin(math.pi * torch.sqrt(r2) / per) ** 2)
        k += 0.1 * torch.eye(int(n), dtype=torch.float64, device=dev)
        y = torch.linalg.cholesky(k) @ torch.from_numpy(z).to(dev)
        xs.append(x)
        ys.append(y.cpu().numpy())
    theta0 = np.stack([np.zeros(count), np.zeros(count), np.log(periods), np.full(count, math.log(0.1))], axis=1)
    return sizes, xs, ys, theta0


def batched_measure(torch, dev, count=BATCH_P, single_sample=32, cpu_sample=48, fp64_peak=None):
    import gprx_b200 as gx
    from gprx_b200 import _lib as L

    sizes, xs, ys, theta0 = batched_synth(torch, dev, count)
    spec = gx.RbfKernel(1.0) + gx.PeriodicKernel(1.0, 15.0)
    opt = gx.Lbfgs().with_tolerance(1e-6)
    # end to end through the public API: upload, fit, results back
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = gx.GprBatch(spec, xs, ys, BATCH_D, device=dev.index or 0)
    res = b.fit(theta0, opt)
    e2e_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.stream_ptr(), device=dev)
    # device-timed fit (inputs resident)
    l0 = L.lib().gprx_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = b.fit(theta0, opt)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = int(L.lib().gprx_launch_count() - l0)
    fit_s = e0.elapsed_time(e1) * 1e-3
    # one evaluation round at θ0 for the roofline (Σ n³ flop per round)
    e0.record(stream)
    nl, g, st = b.value_and_gradient(theta0)
    e1.record(stream)
    torch.cuda.synchronize()
    round_ms = e0.elapsed_time(e1)
    # the autotuned schedule against the one fixed 64×128 tile shape
    tiles, tune_ms, _ = b.schedule()
    b.set_schedule([0] * gx.GprBatch.SIZE_CLASSES)
    e0.record(stream)
    b.value_and_gradient(theta0)
    e1.record(stream)
    torch.cuda.synchronize()
    round_ms_fixed = e0.elapsed_time(e1)
    b.set_schedule(tiles)
    flops = float((sizes.astype(np.float64) ** 3).sum())
    achieved = flops / (round_ms * 1e-3) / 1e12
    # one model per launch: the single-model path on every k-th problem
    idx = list(range(0, count, max(1, count // single_sample)))[:single_sample]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in idx:
        m = gx.Gpr(gx.RbfKernel(1.0) + gx.PeriodicKernel(1.0, math.exp(theta0[i][2])), gx.GaussianLikelihood(0.1),
                   optimizer=opt, device=dev.index or 0)
        m.fit(xs[i], int(sizes[i]), BATCH_D, ys[i])
    single_s = time.perf_counter() - t0
    single_fps = len(idx) / single_s
    # CPU: the oracle's evaluations on a sample, times evaluations per fit
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    nodes = [[1, 2], [10, 0], [13, 0]]
    cidx = list(range(0, count, max(1, count // cpu_sample)))[:cpu_sample]
    t0 = time.perf_counter()
    for i in cidx:
        O.exact_eval(nodes, theta0[i], xs[i], int(sizes[i]), BATCH_D, ys[i])
    cpu_eval_s = (time.perf_counter() - t0) / len(cidx)
    evals_per_fit = float(res.evaluations.mean())
    cpu_fps = 1.0 / (cpu_eval_s * evals_per_fit)
    bytes_in = int(sum(x.nbytes + y.nbytes for x, y in zip(xs, ys)) + theta0.nbytes)
    return {
        "metric": "batched fits/s (4096 ragged exact GPs, L-BFGS to |g| < 1e-6)",
        "value": count / fit_s, "unit": "fits/s", "ms_per_fit_batch": fit_s * 1e3,
        "config": {"workload": "batched_exact_fit_4096_ragged_rbf_periodic_d3", "problems": count,
                   "n": "log-uniform [32, 1024]", "sum_n3": flops, "d": BATCH_D,
                   "kernel": "RbfKernel(1.0) + PeriodicKernel(1.0, p), p ~ U[10, 20]", "noise_variance": 0.1,
                   "tolerance": 1e-6},
        "status_ok": int((res.status == 0).sum()), "converged": int(res.converged.sum()),
        "converged_share": float(res.converged.mean()),
        "grad_norm_median": float(np.median(res.grad_norm)),
        "evaluations_mean": evals_per_fit, "evaluations_max": int(res.evaluations.max()),
        "gpu_launches": launches,
        "e2e": {"value": count / e2e_s, "unit": "fits/s", "h2d_bytes_per_step": bytes_in,
                "d2h_bytes_per_step": int(theta0.nbytes + count * (8 * 4 + 4 * 2))},
        "one_model_per_launch": {"value": single_fps, "unit": "fits/s",
                                 "sample": "%d problems (every %d-th), Gpr.fit each" % (len(idx), count // single_sample)},
        "speedup_vs_one_model_per_launch": (count / fit_s) / single_fps,
        "schedule": {"size_classes": "n <= 64, 128, 256, ..., 4096, larger",
                     "tile_shapes": [list(t) for t in gx.GprBatch.TILE_SHAPES],
                     "tile_of_class": [int(v) for v in tiles],
                     "round_ms_autotuned": round_ms, "round_ms_fixed_64x128": round_ms_fixed},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp64_peak if fp64_peak else None, "kernel": "batch_eval_kernel",
                     "work": "sum of n_i^3 flop per evaluation round", "round_ms": round_ms},
        "cpu_baseline": {"value": cpu_fps, "unit": "fits/s", "cores": int(O.lib().orc_num_threads()), "kind": "port",
                         "sample": "oracle NLML+gradient of %d problems (every %d-th) at θ0, times the batched run's "
                                   "mean evaluations per fit (%.1f)" % (len(cidx), count // cpu_sample,
                                                                         evals_per_fit)},
    }


# ---------------------------------------------------------------------------
# sparse VFE at n = 10⁶, m = 1024 (Sgpr, RbfArd d = 4)
# ---------------------------------------------------------------------------
def sgpr_synth(n=1_000_000, m=1024, d=4, seed=2):
    """x ~ U[0,1]⁴, y = Σ_k sin(2π f_k x_k) + N(0, 0.1²) with f_k ~ U[0.5, 2];
    lengthscales log-uniform in [0.5, 2]; Z a seeded subset of m rows of x
    (up_to without replacement)."""
    import gprx_b200 as gx

    rng = gx.SeededRng(seed)
    x = rng.unit(n * d)
    f = 0.5 + 1.5 * rng.unit(d)
    ls = np.exp(math.log(0.5) + rng.unit(d) * (math.log(2.0) - math.log(0.5)))
    xm = x.reshape(d, n)
    y = np.sin(2 * math.pi * f[:, None] * xm).sum(0) + 0.1 * rng.normal(n)
    idx = rng.subset(n, m)
    z = xm[:, idx].reshape(-1).copy()
    return x, y, z, ls


def sgpr_measure(torch, dev, steps, warm, n=1_000_000, m=1024, d=4, cpu_n=5_000, fp64_peak=None):
    """FP64 and mixed NLML + gradient evaluations of the VFE objective; the
    mixed value is the headline, with its error against the FP64 results."""
    import gprx_b200 as gx

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    x, y, z, ls = sgpr_synth(n, m, d)
    spec = gx.RbfArdKernel(list(ls))
    theta = np.array(list(np.log(ls)) + [math.log(0.1)])
    rng = gx.SeededRng(6)
    thetas = [theta + 0.1 * rng.normal(theta.size) for _ in range(16)]
    flops = 7.0 * m * m * n + 2.0 * m ** 3 / 3.0
    res = {}
    for prec in ("fp64", "mixed"):
        pr = gx.Precision.Fp64 if prec == "fp64" else gx.Precision.Mixed
        mdl = gx.Sgpr(spec, gx.GaussianLikelihood(0.1), precision=pr).with_optimizer(gx.Fixed()).factor(
            x, n, d, y, z, m)
        stream = torch.cuda.ExternalStream(mdl.stream_ptr(), device=dev)
        for i in range(warm):
            mdl.value_and_gradient(thetas[i % len(thetas)])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        outs = [mdl.value_and_gradient(thetas[i % len(thetas)]) for i in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        res[prec] = {"value": 1000.0 / ms, "ms_per_step": ms, "stage_ms": mdl.stage_times_ms(), "outs": outs,
                     "tflops": flops / (ms * 1e-3) / 1e12}
        del mdl
        torch.cuda.empty_cache()
    nl_err = max(abs(a[0] - b[0]) / max(abs(b[0]), 1.0) for a, b in zip(res["mixed"]["outs"], res["fp64"]["outs"]))
    g_err = max(float(np.max(np.abs(a[1] - b[1]) / np.maximum(np.abs(b[1]), 1.0)))
                for a, b in zip(res["mixed"]["outs"], res["fp64"]["outs"]))
    # CPU oracle on the first cpu_n points (the evaluation is O(n m²)), scaled by n / cpu_n
    xs = x.reshape(d, n)[:, :cpu_n].reshape(-1).copy()
    t0 = time.perf_counter()
    orc = O.Sgpr([[11, d]], thetas[0], xs, cpu_n, d, y[:cpu_n].copy(), z, m)
    orc.nlml()
    orc.grad()
    cpu_s = (time.perf_counter() - t0) * n / cpu_n
    mx, fp = res["mixed"], res["fp64"]
    return {"metric": "Sgpr VFE NLML+grad evals/s (n=1e6, m=1024; mixed, FP64 beside)", "value": mx["value"],
            "unit": "evals/s", "ms_per_step": mx["ms_per_step"], "steps": steps, "stage_ms": mx["stage_ms"],
            "fp64": {"value": fp["value"], "ms_per_step": fp["ms_per_step"], "stage_ms": fp["stage_ms"],
                     "tflops": fp["tflops"]},
            "mixed_vs_fp64": mx["value"] / fp["value"],
            "mixed_error_vs_fp64": {"nlml_rel_max": nl_err, "grad_rel_max": g_err},
            "config": {"workload": "sgpr_vfe_n1e6_m1024_rbfard_d4", "n": n, "m": m, "d": d,
                       "inducing": "seeded subset of x (up_to without replacement)", "noise_variance": 0.1,
                       "mixed": "B = A A^T and H = G A^T as FP64 products emulated on int8 tensor cores (7 "
                                "slices, split-K parts of 32768); the m x n triangular solves (A = L^-1 K_mn, "
                                "G = B^-1 A, L^-T G) stay FP64, by recursive halving"},
            "roofline": {"bound": "tensor", "work": "7 m^2 n + 2 m^3 / 3 flop per evaluation",
                         "achieved": mx["tflops"], "unit": "TFLOP/s (FP64-equivalent)", "peak": fp64_peak,
                         "frac": mx["tflops"] / fp64_peak if fp64_peak else None,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured); 5 of the 7 m^2 n "
                                        "run as FP64 DGEMMs, 2 on the int8 tensor cores"},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "evals/s", "cores": int(O.lib().orc_num_threads()),
                             "kind": "port", "sample": "oracle assembly + NLML + gradient on the first %d points, "
                                                       "time scaled by n / %d (O(n m²))" % (cpu_n, cpu_n)}}


# ---------------------------------------------------------------------------
# serving: Poisson stream of fit / predict / online requests
# ---------------------------------------------------------------------------
SERVE_D = 4


def serving_synth(torch, dev, count=12, seed=4):
    """Datasets for the fit requests: n log-uniform in [64, 4096], x ~ N(0, I₄),
    y a draw from the GP prior (RbfArd, ℓ = 1) plus N(0, 0.05²)."""
    import gprx_b200 as gx

    rng = gx.SeededRng(seed)
    out = []
    for _ in range(count):
        n = int(math.exp(math.log(64) + rng.unit(1)[0] * (math.log(4096) - math.log(64))))
        x = rng.normal(n * SERVE_D)
        xt = torch.from_numpy(x.reshape(SERVE_D, n).T.copy()).to(dev)
        k = torch.exp(-0.5 * torch.cdist(xt, xt).pow(2)) + 0.05 ** 2 * torch.eye(n, dtype=torch.float64, device=dev)
        y = (torch.linalg.cholesky(k) @ torch.from_numpy(rng.normal(n)).to(dev)).cpu().numpy()
        out.append((n, x, y))
    return out


def serving_measure(torch, dev, rate, duration, precision, datasets, seed=5, workers=8):
    """Requests arrive as a Poisson process of `rate` per second for
    `duration` seconds: 20% fits (a new model on one of the datasets), 60%
    predictions (1..10⁴ points, log-uniform) against a model, 20% online
    steps (add or remove 1..16 points).  Latency = submission to completion."""
    import concurrent.futures as cf

    import gprx_b200 as gx

    rs = np.random.RandomState(seed)
    prec = gx.Precision.Fp64 if precision == "fp64" else gx.Precision.Mixed
    srv = gx.Server(device=dev.index or 0, workers=workers)
    kern = gx.RbfArdKernel([1.0] * SERVE_D)
    lik = gx.GaussianLikelihood(0.05 ** 2)
    models = []  # (model id, n, removable original ids)
    for n, x, y in datasets[:3]:  # a few resident models before the stream starts
        mid = srv.submit_fit(kern, lik, x, n, SERVE_D, y, precision=prec)
        srv.wait(mid)
        models.append([mid, n, list(range(n))])
    pool = cf.ThreadPoolExecutor(max_workers=64)
    futs = []
    kinds = []
    t0 = time.perf_counter()
    t = 0.0
    while True:
        t += rs.exponential(1.0 / rate)
        if t > duration:
            break
        now = time.perf_counter() - t0
        if t > now:
            time.sleep(t - now)
        u = rs.rand()
        if u < 0.2:
            n, x, y = datasets[rs.randint(len(datasets))]
            rid = srv.submit_fit(kern, lik, x, n, SERVE_D, y, precision=prec)
            models.append([rid, n, list(range(n))])
            kinds.append("fit")
        elif u < 0.8:
            m = models[rs.randint(len(models))]
            q = int(math.exp(rs.uniform(0.0, math.log(1e4))))
            rid, _, _ = srv.submit_predict(m[0], rs.standard_normal(q * SERVE_D), q)
            kinds.append("predict")
        else:
            m = models[rs.randint(len(models))]
            k = int(rs.randint(1, 17))
            if rs.rand() < 0.5 or len(m[2]) <= k + 8:
                rid, _ = srv.submit_add(m[0], rs.standard_normal(k * SERVE_D), rs.standard_normal(k), k)
            else:
                take = [m[2].pop(rs.randint(len(m[2]))) for _ in range(k)]
                rid = srv.submit_remove(m[0], take)
            kinds.append("online")
        futs.append(pool.submit(srv.wait, rid))
    res = [f.result() for f in futs]
    wall = time.perf_counter() - t0
    pool.shutdown()
    stats = srv.stats()
    srv.close()
    lat = np.array([r[1]["latency_ms"] for r in res])
    ok = np.array([r[0] == 0 for r in res])
    per = {}
    for kind in ("fit", "predict", "online"):
        sel = np.array([k == kind for k in kinds]) & ok
        if sel.any():
            per[kind] = {"count": int(sel.sum()), "p50_ms": float(np.percentile(lat[sel], 50)),
                         "p99_ms": float(np.percentile(lat[sel], 99))}
    return {"arrival_rate_per_s": rate, "duration_s": duration, "precision": precision,
            "requests": len(res), "completed_ok": int(ok.sum()), "requests_per_s": float(ok.sum() / wall),
            "p50_ms": float(np.percentile(lat[ok], 50)) if ok.any() else None,
            "p99_ms": float(np.percentile(lat[ok], 99)) if ok.any() else None,
            "per_kind": per, "merged_predict_launches": stats["merged_launches"],
            "merged_fit_launches": stats["merged_fit_launches"], "workers": workers}


def hessian_measure(torch, dev, local, spec, x, y, theta, n, d, steps, warm, forms=("fp64", "mixed")):
    """NLML Hessians (gprx_exact_hessian) at the exact workload's θ, timed
    with CUDA events on the model's stream, per precision form."""
    import gprx_b200 as gx
    from gprx_b200 import _lib as L

    per = {}
    for f in forms:
        prec = gx.Precision.Fp64 if f == "fp64" else gx.Precision.Mixed
        model = gx.Gpr(spec, gx.GaussianLikelihood(NOISE), precision=prec, device=local) \
            .with_optimizer(gx.Fixed()).factor(x, n, d, y)
        stream = torch.cuda.ExternalStream(model.stream_ptr(), device=dev)
        for i in range(warm):
            model.hessian(theta)
        torch.cuda.synchronize()
        l0 = L.lib().gprx_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(steps):
            h = model.hessian(theta)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        per[f] = {"ms_per_hessian": ms, "launches_per_hessian": (L.lib().gprx_launch_count() - l0) / steps,
                  "h00": float(h[0, 0])}
        del model
        torch.cuda.empty_cache()
    head = per["mixed"] if "mixed" in per else per["fp64"]
    p = theta.size
    return {"metric": "NLML Hessians/s n=%d p=%d" % (n, p), "value": 1e3 / head["ms_per_hessian"],
            "unit": "hessians/s", "config": {"workload": "exact_gpr_nlml_hessian_n%d_d%d_const_rbfard" % (n, d),
                                             "n": n, "d": d, "p": p},
            "forms": per,
            "work": "one evaluation with gradient; per kernel parameter S_i = X dK/dθ_i X^T with X = L^-1 "
                    "(4 n^3 / 3 flop) and the second-order kernel walk over the n(n+1)/2 pairs (all parameters in "
                    "one launch)"}


def brief(d, keys):
    """The listed keys of a result dict (the default line stays within the
    few KB a log tail keeps)."""
    return {k: d[k] for k in keys if k in d}


def rounded(obj, digits=4):
    """Floats to `digits` significant digits, recursively."""
    if isinstance(obj, float):
        return float("%.*g" % (digits, obj)) if math.isfinite(obj) else obj
    if isinstance(obj, dict):
        return {k: rounded(v, digits) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [rounded(v, digits) for v in obj]
    return obj


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: the mixed form is the headline value, the FP64 form is timed beside it")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-evals", type=int, default=0,
                    help="only factor once and run this many evaluations (for an ncu launch list), no JSON line")
    ap.add_argument("--workload", default="all", choices=["all", "exact", "c1", "batched", "serving", "sgpr", "hessian"],
                    help="all: the exact line with the batched measurement as its 'batched' key")
    ap.add_argument("--batch-problems", type=int, default=BATCH_P)
    ap.add_argument("--serve-rates", default="8,16,32,64", help="arrival rates (requests/s) of the serving sweep")
    ap.add_argument("--serve-requests", type=int, default=300, help="requests per rate of the serving sweep")
    args = ap.parse_args()
    n, d = args.n, D
    warm = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    workload = "exact_gpr_nlml_grad_n%d_d%d_const_rbfard" % (n, d)
    config = {"workload": workload, "n": n, "d": d,
              "l2": "inputs > L2 (two n x n FP64 buffers of %d MiB)" % (n * n * 8 // 2 ** 20),
              "parallelism": "replicas" if args.gpus > 1 else "single"}
    metric = "NLML+grad evals/s n=%d (%s)" % (n, {"both": "mixed; FP64 beside", "mixed": "mixed",
                                                   "fp64": "FP64"}[args.precision])

    x, y, theta = synth(n, d)
    thetas = perturbations(theta)

    if args.impl == "reference":
        if rank != 0:
            return
        value, dt, cores, sample = cpu_reference(n, d, x, y, thetas, args.steps, args.warmup)
        line = {"metric": metric, "value": value, "unit": "evals/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import gprx_b200 as gx
    from gprx_b200 import _lib as L

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    if args.workload == "sgpr":
        if args.profile_evals > 0:
            x, yv, z, ls = sgpr_synth()
            prec = gx.Precision.Fp64 if args.precision == "fp64" else gx.Precision.Mixed
            mdl = gx.Sgpr(gx.RbfArdKernel(list(ls)), gx.GaussianLikelihood(0.1), precision=prec).with_optimizer(
                gx.Fixed()).factor(x, 1_000_000, 4, yv, z, 1024)
            theta = np.array(list(np.log(ls)) + [math.log(0.1)])
            for _ in range(args.profile_evals):
                mdl.value_and_gradient(theta)
            torch.cuda.synchronize()
            return
        out = sgpr_measure(torch, dev, args.steps, warm, fp64_peak=fp64_peak_tflops(torch, dev))
        out.update({"n_gpus": 1, "warmup": warm, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic"})
        print(json.dumps(out), flush=True)
        return

    if args.workload == "c1":
        out = c1_measure(torch, local, steps=args.steps, warm=warm)
        out.update({"metric": "exact RBF n=512 d=2: L-BFGS fit + predict 256 per second", "n_gpus": 1,
                    "steps": args.steps, "warmup": warm, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                    "config": {"workload": "exact_gpr_fit_predict_n512_d2_rbf"}})
        print(json.dumps(out), flush=True)
        return

    if args.workload == "serving":
        datasets = serving_synth(torch, dev)
        sweep = []
        for prec in ("fp64", "mixed"):
            for rate in [float(r) for r in args.serve_rates.split(",")]:
                sweep.append(serving_measure(torch, dev, rate, args.serve_requests / rate, prec, datasets))
        head = max((r for r in sweep if r["precision"] == "mixed"), key=lambda r: r["requests_per_s"])
        out = {"metric": "serving p99 latency (ms) at the highest sustained rate", "value": head["p99_ms"],
               "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": len(sweep), "warmup": 3,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": "serving_exact_rbfard_d4_poisson", "mix": "20% fit, 60% predict, 20% online",
                          "fit_n": "log-uniform [64, 4096]", "predict_q": "log-uniform [1, 1e4]",
                          "online_points": "1..16"},
               "sweep": sweep}
        print(json.dumps(out), flush=True)
        return

    if args.workload == "batched":
        if args.profile_evals > 0:
            sizes, xs, ys, theta0 = batched_synth(torch, dev, args.batch_problems)
            b = gx.GprBatch(gx.RbfKernel(1.0) + gx.PeriodicKernel(1.0, 15.0), xs, ys, BATCH_D, device=local)
            for _ in range(args.profile_evals):
                b.value_and_gradient(theta0)
            torch.cuda.synchronize()
            return
        peak = fp64_peak_tflops(torch, dev)
        out = batched_measure(torch, dev, args.batch_problems, fp64_peak=peak)
        out.update({"n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic"})
        print(json.dumps(out), flush=True)
        return

    spec = gx.ConstantKernel(CONST) * gx.RbfArdKernel(list(np.exp(theta[1:1 + d])))

    if args.workload == "hessian":
        forms = ["fp64"] if args.precision == "fp64" else ["mixed"] if args.precision == "mixed" else ["fp64", "mixed"]
        if args.profile_evals > 0:
            prec = gx.Precision.Fp64 if forms[0] == "fp64" else gx.Precision.Mixed
            model = gx.Gpr(spec, gx.GaussianLikelihood(NOISE), precision=prec, device=local) \
                .with_optimizer(gx.Fixed()).factor(x, n, d, y)
            for i in range(args.profile_evals):
                model.hessian(theta)
            torch.cuda.synchronize()
            return
        out = hessian_measure(torch, dev, local, spec, x, y, theta, n, d, args.steps, warm, forms)
        out.update({"n_gpus": 1, "steps": args.steps, "warmup": warm, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic"})
        print(json.dumps(out), flush=True)
        return

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def measure(precision):
        """Device-timed and end-to-end evaluations of one precision form."""
        prec = gx.Precision.Fp64 if precision == "fp64" else gx.Precision.Mixed
        model = gx.Gpr(spec, gx.GaussianLikelihood(NOISE), precision=prec, device=local) \
            .with_optimizer(gx.Fixed()).factor(x, n, d, y)
        stream = torch.cuda.ExternalStream(model.stream_ptr(), device=dev)
        for i in range(warm):
            model.value_and_gradient(thetas[i % len(thetas)])
        barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        l0 = L.lib().gprx_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        stage = np.zeros(5)
        outs = []
        for i in range(args.steps):
            outs.append(model.value_and_gradient(thetas[i % len(thetas)]))
            st = model.stage_times_ms()
            stage += np.array([st["fill"], st["factor"], st["inverse"], st["gradient"], st["total"]])
        e1.record(stream)
        torch.cuda.synchronize()
        launches = int(L.lib().gprx_launch_count() - l0)
        clk = clocks.stop()
        barrier()
        ms_max = max_over_ranks(e0.elapsed_time(e1))
        # end to end through the public API with host buffers
        xh = torch.from_numpy(x).pin_memory().numpy()
        yh = torch.from_numpy(y).pin_memory().numpy()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(args.steps):
            model.set_data(xh, yh)
            model.value_and_gradient(thetas[i % len(thetas)])
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        del model
        torch.cuda.empty_cache()
        return {"value": args.steps * world / (ms_max * 1e-3), "ms_per_step": ms_max / args.steps,
                "stage": stage / args.steps, "launches": launches, "clocks": clk, "outs": outs,
                "e2e": {"value": args.steps * world / e2e_s, "unit": "evals/s",
                        "h2d_bytes_per_step": int((n * d + n + theta.size) * 8),
                        "d2h_bytes_per_step": int((1 + theta.size) * 8)}}

    if args.profile_evals > 0:
        prec = gx.Precision.Fp64 if args.precision == "fp64" else gx.Precision.Mixed
        model = gx.Gpr(spec, gx.GaussianLikelihood(NOISE), precision=prec, device=local) \
            .with_optimizer(gx.Fixed()).factor(x, n, d, y)
        for i in range(args.profile_evals):
            model.value_and_gradient(thetas[i % len(thetas)])
        torch.cuda.synchronize()
        return

    forms = ["fp64"] if args.precision == "fp64" else ["mixed"] if args.precision == "mixed" else ["fp64", "mixed"]
    res = {f: measure(f) for f in forms}
    head = res["mixed"] if "mixed" in res else res["fp64"]
    stage = head["stage"]
    peaks = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch, dev) if rank == 0 else None
    dmma_ms = stage[1] + stage[2]
    achieved = (n ** 3) / (dmma_ms * 1e-3) / 1e12
    traffic = load_traffic()
    mixed = "mixed" in res
    stage_roofline = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                      "frac": achieved / fp64_peak if fp64_peak else None,
                      "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured; FP64 has no entry "
                                     "in MEASURED_PEAKS.json)",
                      "kernel": ("factor + inverse stages: emu_gemm_kernel<7> + dgemm_kernel + potrf_diag_kernel"
                                 if mixed else "dgemm_kernel (DMMA m16n8k4 f64) inside potrf/trtri/lauum"),
                      "work": "n^3 FP64(-equivalent) flops per evaluation (potrf n^3/3 + trtri n^3/3 + lauum "
                              "n^3/3) over the factor + inverse stage time",
                      "stage_ms": {"fill": stage[0], "factor": stage[1], "inverse": stage[2], "gradient": stage[3],
                                   "total": stage[4]}}
    roofline = {k: stage_roofline[k] for k in ("bound", "achieved", "peak", "unit", "frac")}
    roofline["kernel"] = "factor + inverse stages (n^3 flop)"
    roofline["traffic"] = traffic.get("dgemm_bytes_per_eval") if traffic else None
    if mixed and rank == 0:
        k = emu_kernel_roofline(n, peaks, traffic, int8_peak_tops(torch, dev))
        if k is not None:
            roofline = {"bound": "tensor", "kernel": "emu_gemm_kernel<7> at (n/2)^3", "achieved": k["achieved"],
                        "peak": k["peak"], "unit": "TOP/s int8", "frac": k["frac"], "traffic": k["traffic"],
                        "peak_src": "cuBLASLt int8 (of measured)" if "cuBLASLt" in k["peak_source"]
                        else k["peak_source"][:40], "fp64_eq_tflops": k["fp64_equivalent_tflops"]}
    roofline["stage_frac_of_dgemm"] = stage_roofline["frac"]
    clk = head["clocks"]
    line = {"metric": metric, "value": head["value"], "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not mixed else "f64 (int8-emulated products)",
            "data": "synthetic", "config": config, "e2e": head["e2e"], "gpu_launches": head["launches"],
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
            "roofline": roofline,
            "stage_ms": {k: stage[i] for i, k in enumerate(("fill", "factor", "inverse", "gradient", "total"))}}
    if mixed and "fp64" in res:
        f, m = res["fp64"], res["mixed"]
        nl_err = max(abs(a[0] - b[0]) / max(abs(b[0]), 1.0) for a, b in zip(m["outs"], f["outs"]))
        g_err = max(float(np.max(np.abs(a[1] - b[1]) / np.maximum(np.abs(b[1]), 1.0)))
                    for a, b in zip(m["outs"], f["outs"]))
        line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "e2e": f["e2e"]["value"],
                        "frac_of_dgemm": (n ** 3) / ((f["stage"][1] + f["stage"][2]) * 1e-3) / 1e12 / fp64_peak
                        if fp64_peak else None}
        line["mixed_vs_fp64"] = m["value"] / f["value"]
        line["mixed_error_vs_fp64"] = {"nlml": nl_err, "grad": g_err}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, dt, cores, sample = cpu_reference(n, d, x, y, thetas, steps=1, warmup=0)
        line["cpu_baseline"] = {"value": v, "unit": "evals/s", "cores": cores, "kind": "port", "sample": sample}
    if args.workload == "all" and world == 1:
        torch.cuda.empty_cache()
        c1 = c1_measure(torch, local)
        line["c1"] = brief(c1, ("value", "unit", "ms_per_fit_predict", "predict_ms", "evaluations", "converged",
                                "grad_norm", "predict_err_vs_oracle"))
        line["c1"]["cpu"] = c1["cpu_baseline"]["value"]
        bt = batched_measure(torch, dev, args.batch_problems, fp64_peak=fp64_peak)
        line["batched"] = brief(bt, ("value", "unit", "speedup_vs_one_model_per_launch", "status_ok", "converged",
                                     "converged_share", "grad_norm_median"))
        line["batched"].update({"e2e": bt["e2e"]["value"], "one_model_per_launch": bt["one_model_per_launch"]["value"],
                                "round_ms": bt["roofline"]["round_ms"], "frac_of_dgemm": bt["roofline"]["frac"],
                                "cpu": bt["cpu_baseline"]["value"]})
        datasets = serving_synth(torch, dev)
        # a sweep of Poisson arrival rates, 300 requests each (mixed; FP64 at
        # two of the rates): precision, rate, requests, req/s, p50 / p99 ms,
        # merged predict launches, merged fit launches
        sweep = [("mixed", r) for r in (8.0, 16.0, 32.0, 64.0)] + [("fp64", r) for r in (16.0, 64.0)]
        line["serving"] = []
        for prec, rate in sweep:
            r = serving_measure(torch, dev, rate, 300.0 / rate, prec, datasets)
            line["serving"].append([prec, rate, r["requests"], r["requests_per_s"], r["p50_ms"], r["p99_ms"],
                                    r["merged_predict_launches"], r["merged_fit_launches"]])
        torch.cuda.empty_cache()
        sg = sgpr_measure(torch, dev, 3, 2, fp64_peak=fp64_peak)
        line["sgpr"] = brief(sg, ("value", "unit", "mixed_vs_fp64"))
        line["sgpr"].update({"fp64": sg["fp64"]["value"], "err": [sg["mixed_error_vs_fp64"]["nlml_rel_max"],
                                                                  sg["mixed_error_vs_fp64"]["grad_rel_max"]],
                             "frac_of_dgemm": sg["roofline"]["frac"], "cpu": sg["cpu_baseline"]["value"]})
        torch.cuda.empty_cache()
        hs = hessian_measure(torch, dev, local, spec, x, y, theta, n, d, 3, 3)
        line["hessian"] = {"fp64_ms": hs["forms"]["fp64"]["ms_per_hessian"],
                           "mixed_ms": hs["forms"]["mixed"]["ms_per_hessian"]}
    line = rounded(line)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
