// exact.cu — exact-GPR objective, factor and prediction on the device.
//
// One evaluation (gprx ExactFit::value_and_gradient_into_fit,
// src/gpr/exact_fit.rs:319-341) is enqueued on the handle's stream as
//   fill  K + (σn² + j) I                      (factor.rs:515-542)
//   potrf L                                    (chol.rs:141-167)
//   logdet 2 Σ ln L_ii                          (factor.rs:555-568)
//   trtri X = L⁻¹, α = Xᵀ (X y), yᵀα
//   lauum K⁻¹ = Xᵀ X                            (workspace.rs:395-425)
//   contraction −½⟨ααᵀ − K⁻¹, ∂K/∂θ⟩, noise −½σn² Σ W_ii (exact_fit.rs:665-729)
// and drained with one synchronisation.  A non-positive pivot stops every
// later kernel through the device status word; the host then retries with the
// next jitter offset (retry_with_jitter, chol.rs:35-58) or restores the
// previous θ and its factor (exact_fit.rs:196-206).

#include <algorithm>
#include <cmath>

#include "exact.cuh"
#include "hessian.cuh"
#include "persist.h"

namespace gprx {

ExactState::~ExactState() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

static bool in_default_interval(double log_v) {
  // Interval::DEFAULT_POSITIVE = (1e-5, 1e5), open (src/param.rs:91)
  double v = std::exp(log_v);
  return std::isfinite(v) && v > 1e-5 && v < 1e5;
}

gprx_status ExactState::create(const double* xh, uint64_t nn, uint64_t dd, const double* yh,
                               const gprx_kernel_node* nodes, int n_nodes, const double* theta, int n_theta,
                               const gprx_options* o) {
  if (!xh || !yh || !nodes || (!theta && n_theta > 0)) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (nn == 0) return set_error(GPRX_EMPTY_INPUT, "no training points");
  if (dd == 0) return set_error(GPRX_EMPTY_INPUT, "no features (d = 0)");
  if (nn > (uint64_t)INT32_MAX / 2) return set_error(GPRX_CAPACITY, "n too large");
  if (!all_finite(xh, nn * dd) || !all_finite(yh, nn)) return set_error(GPRX_NONFINITE_INPUT, "non-finite input");
  if (o) opt = *o;
  else gprx_options_default(&opt);
  std::string why;
  // θ for the kernel comes first, then log σn²
  if (n_theta < 1) return set_error(GPRX_SHAPE_MISMATCH, "theta must hold the kernel parameters and log noise");
  gprx_status st = kern.init(nodes, n_nodes, theta, n_theta - 1, (int)dd, &why);
  if (st != GPRX_OK) return set_error(st, why);
  for (int i = 0; i < n_theta; ++i)
    if (!in_default_interval(theta[i]))
      return set_error(GPRX_INVALID_HYPERPARAMETER, "hyperparameter outside (1e-5, 1e5)");
  log_noise = theta[n_theta - 1];
  n = (int)nn;
  d = (int)dd;
  cap = n;
  ld = round_ld(cap);
  device = opt.device;
  GPRX_CUDA_TRY(cudaSetDevice(device));
  GPRX_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  for (auto& e : ev) GPRX_CUDA_TRY(cudaEventCreate(&e));
  int nblk = ceil_div(cap, NB);
  if (x.alloc((size_t)cap * d) != cudaSuccess || y.alloc(cap) != cudaSuccess ||
      A.alloc((size_t)ld * cap) != cudaSuccess || linv.alloc((size_t)nblk * NB * NB) != cudaSuccess ||
      alpha.alloc(cap) != cudaSuccess || z.alloc(cap) != cudaSuccess || tmpv.alloc(cap) != cudaSuccess ||
      partials.alloc((size_t)grad_max_blocks() * 64) != cudaSuccess || slot_param.alloc(64) != cudaSuccess ||
      res.alloc(64) != cudaSuccess || status.alloc(1) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "device allocation failed");
  GPRX_CUDA_TRY(res_h.ensure(64));
  GPRX_CUDA_TRY(status_h.ensure(1));
  GPRX_CUDA_TRY(cudaMemcpyAsync(x.p, xh, sizeof(double) * n * d, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(y.p, yh, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  std::vector<int> sp(64, -1);
  std::copy(kern.slot_param.begin(), kern.slot_param.end(), sp.begin());
  GPRX_CUDA_TRY(cudaMemcpyAsync(slot_param.p, sp.data(), sizeof(int) * 64, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  y_host.assign(yh, yh + n);
  for (int i = 0; i < n; ++i) ids.push_back(next_id++);
  return GPRX_OK;
}

void ExactState::get_params(double* out) const {
  for (int i = 0; i < kern.n_params; ++i) out[i] = kern.theta[i];
  out[kern.n_params] = log_noise;
}

gprx_status ExactState::write_params(const double* params) {
  int p = num_params();
  for (int i = 0; i < p; ++i)
    if (!in_default_interval(params[i]))
      return set_error(GPRX_INVALID_HYPERPARAMETER, "hyperparameter outside (1e-5, 1e5)");
  gprx_status st = kern.set_theta(params);
  if (st != GPRX_OK) return set_error(st, "invalid kernel hyperparameter");
  log_noise = params[p - 1];
  factor_ok = false;
  alpha_ok = false;
  return GPRX_OK;
}

gprx_status ExactState::reset_status() {
  GPRX_CUDA_TRY(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), stream));
  return GPRX_OK;
}

gprx_status ExactState::read_status(DevStatus* out) {
  GPRX_CUDA_TRY(cudaMemcpyAsync(status_h.p, status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  *out = *status_h.p;
  return GPRX_OK;
}

gprx_status ExactState::enqueue_factor(double j) {
  GPRX_CUDA_TRY(cudaEventRecord(ev[0], stream));
  GPRX_CUDA_TRY(fill_lower(kern, x.p, cap, n, A.p, ld, noise() + j, status.p, stream));
  GPRX_CUDA_TRY(cudaEventRecord(ev[1], stream));
  GPRX_CUDA_TRY(potrf_blocked(A.p, ld, n, linv.p, status.p, stream, &fctx));
  GPRX_CUDA_TRY(cudaEventRecord(ev[2], stream));
  return GPRX_OK;
}

// JitterPolicy retry offsets after the first attempt (src/policy.rs:306-397).
std::vector<double> retry_list(const gprx_options& o) {
  std::vector<double> out;
  if (o.jitter_kind == GPRX_JITTER_FIXED) {
    if (o.jitter_initial > 0.0) out.push_back(o.jitter_initial);
    return out;
  }
  double j = o.jitter_initial;
  for (int r = 0; r < o.jitter_max_retries; ++r) {
    if (!(j <= o.jitter_max)) break;
    out.push_back(j);
    double g = j * o.jitter_multiplier;
    if (!std::isfinite(g)) break;
    j = g;
  }
  return out;
}

std::vector<double> jitter_attempts(const gprx_options& o) {
  std::vector<double> js{0.0};
  auto r = retry_list(o);
  js.insert(js.end(), r.begin(), r.end());
  return js;
}

gprx_status ExactState::factor_with_retries(int stage) {
  std::vector<double> js{0.0};
  auto r = retry_list(opt);
  js.insert(js.end(), r.begin(), r.end());
  double last = 0.0;
  for (double j : js) {
    last = j;
    gprx_status st = reset_status();
    if (st != GPRX_OK) return st;
    st = enqueue_factor(j);
    if (st != GPRX_OK) return st;
    DevStatus ds;
    st = read_status(&ds);
    if (st != GPRX_OK) return st;
    if (ds.code == GPRX_OK) {
      jitter = j;
      factor_ok = true;
      linv_ok = true;
      online = false;
      return GPRX_OK;
    }
    if (ds.code != GPRX_CHOLESKY_FAILED) return status_to_error(ds, j, n, stage);
  }
  factor_ok = false;
  return set_cholesky_error(last, n, stage);
}

gprx_status ExactState::solve_alpha_from_l() {
  GPRX_CUDA_TRY(cudaMemcpyAsync(alpha.p, y.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(trsm_lower(A.p, ld, n, linv.p, alpha.p, n, 1, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower_t(A.p, ld, n, linv.p, alpha.p, n, 1, status.p, stream));
  alpha_ok = true;
  return GPRX_OK;
}

gprx_status ExactState::factor_current() {
  gprx_status st = factor_with_retries(GPRX_STAGE_FIT);
  if (st != GPRX_OK) return st;
  st = solve_alpha_from_l();
  if (st != GPRX_OK) return st;
  DevStatus ds;
  st = read_status(&ds);
  if (st != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, jitter, n, GPRX_STAGE_FIT);
  return GPRX_OK;
}

gprx_status ExactState::ensure_emu() {
  const size_t bytes = emu_slice_bytes(cap, cap, 7);
  const size_t rows = (size_t)emu_pad_rows(cap);
  if (emu_sa.ensure(bytes) || emu_sb.ensure(bytes) || emu_ea.ensure(rows) || emu_eb.ensure(rows) ||
      emu_ma.ensure(rows) || emu_mb.ensure(rows) || emu_err.ensure(1))
    return set_error(GPRX_OUT_OF_MEMORY, "device allocation of the emulated-product scratch failed");
  GPRX_CUDA_TRY(emu_err_h.ensure(1));
  return GPRX_OK;
}

gprx_status ExactState::eval(const double* params, double* nlml_out, double* grad) {
  const int p = num_params();
  std::vector<double> prev(p);
  get_params(prev.data());
  gprx_status st = write_params(params);
  if (st != GPRX_OK) return st;
  if (online) return set_error(GPRX_INVALID_CONFIG, "an online model takes no hyperparameter evaluation");
  std::vector<double> js{0.0};
  auto r = retry_list(opt);
  js.insert(js.end(), r.begin(), r.end());
  double last = 0.0;
  const size_t nn = (size_t)ld * cap;
  if (grad && Xinv.n < nn) {
    size_t half = (size_t)((n + 1) / 2) * ((n + 1) / 2);
    if (Xinv.alloc(nn) != cudaSuccess || scratch.alloc(std::max<size_t>(half, 1)) != cudaSuccess) {
      Xinv.reset();
      write_params(prev.data());
      return set_error(GPRX_OUT_OF_MEMORY, "device allocation of the inverse failed");
    }
    GPRX_CUDA_TRY(cudaMemsetAsync(Xinv.p, 0, sizeof(double) * nn, stream));
  }
  for (double j : js) {
    last = j;
    if ((st = reset_status()) != GPRX_OK) return st;
    const bool emu = grad && use_emu();
    EmuWork ew;
    if (emu) {
      // fill, then L and X = L⁻¹ together by recursive halving with the
      // coupling products emulated
      if ((st = ensure_emu()) != GPRX_OK) return st;
      ew.sa = emu_sa.p; ew.sb = emu_sb.p; ew.ea = emu_ea.p; ew.eb = emu_eb.p; ew.ma = emu_ma.p; ew.mb = emu_mb.p;
      ew.err = emu_err.p;
      ew.S = 7;
      GPRX_CUDA_TRY(cudaMemsetAsync(emu_err.p, 0, sizeof(int), stream));
      GPRX_CUDA_TRY(cudaEventRecord(ev[0], stream));
      GPRX_CUDA_TRY(fill_lower(kern, x.p, cap, n, A.p, ld, noise() + j, status.p, stream));
      GPRX_CUDA_TRY(cudaEventRecord(ev[1], stream));
      GPRX_CUDA_TRY(potrf_trtri_rec(A.p, ld, n, Xinv.p, ld, linv.p, scratch.p, ew, EMU_LEAF_N, EMU_MIN_N, status.p,
                                    stream, &fctx));
      GPRX_CUDA_TRY(cudaEventRecord(ev[2], stream));
    } else {
      if ((st = enqueue_factor(j)) != GPRX_OK) return st;
    }
    GPRX_CUDA_TRY(logdet_diag(A.p, ld, n, false, res.p + 0, status.p, stream));
    if (grad) {
      if (!emu)  // the mixed factor produced X = L⁻¹ already
        GPRX_CUDA_TRY(trtri_blocked(A.p, ld, n, linv.p, Xinv.p, ld, scratch.p, status.p, stream));
      GPRX_CUDA_TRY(trmv_lower(Xinv.p, ld, n, y.p, z.p, status.p, stream));
      GPRX_CUDA_TRY(gemv_t(Xinv.p, ld, n, n, true, z.p, alpha.p, status.p, stream));
      GPRX_CUDA_TRY(dot_dev(y.p, alpha.p, n, res.p + 1, status.p, stream));
      if (emu) {
        GPRX_CUDA_TRY(lauum_lower_emu(Xinv.p, ld, n, A.p, ld, ew, status.p, stream));
        GPRX_CUDA_TRY(cudaMemcpyAsync(emu_err_h.p, emu_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
      } else {
        GPRX_CUDA_TRY(lauum_lower(Xinv.p, ld, n, A.p, ld, status.p, stream));
      }
      GPRX_CUDA_TRY(cudaEventRecord(ev[3], stream));
      int blocks = 0;
      GPRX_CUDA_TRY(grad_contract(kern, x.p, cap, n, A.p, ld, alpha.p, partials.p, &blocks, status.p, stream));
      GPRX_CUDA_TRY(grad_finalize(kern, partials.p, blocks, slot_param.p, -0.5, -0.5 * noise(), res.p + 2,
                                  status.p, stream));
      GPRX_CUDA_TRY(cudaEventRecord(ev[4], stream));
    } else {
      GPRX_CUDA_TRY(cudaMemcpyAsync(alpha.p, y.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
      GPRX_CUDA_TRY(trsm_lower(A.p, ld, n, linv.p, alpha.p, n, 1, status.p, stream));
      GPRX_CUDA_TRY(trsm_lower_t(A.p, ld, n, linv.p, alpha.p, n, 1, status.p, stream));
      GPRX_CUDA_TRY(dot_dev(y.p, alpha.p, n, res.p + 1, status.p, stream));
      GPRX_CUDA_TRY(cudaEventRecord(ev[3], stream));
      GPRX_CUDA_TRY(cudaEventRecord(ev[4], stream));
    }
    GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p, sizeof(double) * (2 + p), cudaMemcpyDeviceToHost, stream));
    DevStatus ds;
    if ((st = read_status(&ds)) != GPRX_OK) return st;
    ev_recorded = true;
    if (ds.code == GPRX_OK && grad && use_emu() && *emu_err_h.p != 0) {
      write_params(prev.data());
      factor_current();
      return set_error(GPRX_TIMEOUT, "an emulated product's bounded wait ran out");
    }
    if (ds.code == GPRX_OK) {
      jitter = j;
      factor_ok = grad == nullptr;  // the gradient overwrote L with K⁻¹
      linv_ok = factor_ok;
      alpha_ok = true;
      online = false;
      double logdet = res_h.p[0], quad = res_h.p[1];
      *nlml_out = 0.5 * (quad + logdet + (double)n * std::log(2.0 * M_PI));
      if (grad)
        for (int i = 0; i < p; ++i) grad[i] = res_h.p[2 + i];
      if (!std::isfinite(*nlml_out)) return set_error(GPRX_NOT_CONVERGED, "non-finite NLML");
      return GPRX_OK;
    }
    if (ds.code != GPRX_CHOLESKY_FAILED) {
      gprx_status e = status_to_error(ds, j, n, GPRX_STAGE_FIT);
      write_params(prev.data());
      factor_current();
      return set_error(e, last_error().message);
    }
  }
  // every offset failed: restore θ and its factor (exact_fit.rs:196-206)
  write_params(prev.data());
  factor_current();
  return set_cholesky_error(last, n, GPRX_STAGE_FIT);
}

// ExactFit::hessian_into_fit (src/gpr/exact_fit.rs:443-637): one evaluation
// at θ leaves K⁻¹ (lower) in A, L⁻¹ in Xinv and α; the second-order part is
// −½ ⟨ααᵀ − K⁻¹, ∂²K/∂θ_i∂θ_j⟩ over the lower triangle (weight 2 off the
// diagonal), the first-order part −½ ⟨S_i, S_j⟩_F + v_iᵀ v_j with
// S_i = L⁻¹ A_i L⁻ᵀ and v_i = L⁻¹ A_i α (A_i = ∂K/∂θ_i, or σn² I for the
// noise), S_i formed from the explicit inverse X = L⁻¹ as (X A_i) Xᵀ with the
// triangles cut from both products.  out is row-major p × p.
gprx_status ExactState::hessian(const double* params, double* out, double* nlml_out, double* grad_out) {
  const int p = num_params(), pk = kern.n_params;
  if (online) return set_error(GPRX_INVALID_CONFIG, "an online model takes no hyperparameter evaluation");
  std::vector<double> g(p);
  double v = 0.0;
  gprx_status st = eval(params, &v, g.data());
  if (st != GPRX_OK) return st;
  if (nlml_out) *nlml_out = v;
  if (grad_out) std::copy(g.begin(), g.end(), grad_out);
  const size_t nn = (size_t)ld * n;
  const int SEC = 0, TR = HESS_MAX_PARAMS * HESS_MAX_PARAMS, AA = TR + 1, FRO = TR + 2, VD = FRO + p * p;
  const int FUS = VD + p * p, TRF = FUS + HESS_FUSE_SLOTS;
  const int nres = TRF + HESS_TRACE_SLOTS;
  const bool fuse_second = pk <= HESS_FUSE_K, fuse_trace = p <= HESS_FUSE_P;
  if (hs_s.ensure(nn * p) || hs_p.ensure(nn) || hs_d.ensure(nn) || hs_v.ensure((size_t)n * (p + 1)) ||
      hs_part.ensure((size_t)HESS_MAX_BLOCKS * std::max(HESS_MAX_PARAMS, HESS_TRACE_SLOTS)) || hs_res.ensure(nres)) {
    hs_s.reset();
    hs_p.reset();
    hs_d.reset();
    return set_error(GPRX_OUT_OF_MEMORY, "device allocation of the Hessian scratch failed");
  }
  GPRX_CUDA_TRY(hs_res_h.ensure(nres));
  if ((st = reset_status()) != GPRX_OK) return st;
  HessMap hm{};
  hm.n_par = pk;
  for (int l = 0; l < kern.tree.n_leaves; ++l) {
    const KLeaf& lf = kern.tree.leaf[l];
    const int cnt = lf.kind == GPRX_LEAF_PERIODIC ? 2 : lf.kind == GPRX_LEAF_RBF_ARD ? kern.tree.d : 1;
    unsigned tm = 0;
    for (int t = 0; t < kern.tree.n_terms; ++t)
      if ((kern.tree.term_mask[t] >> l) & 1u) tm |= 1u << t;
    for (int a = 0; a < cnt; ++a) {
      hm.leaf_of[lf.param + a] = l;
      hm.local_of[lf.param + a] = a;
      hm.terms_of[lf.param + a] = tm;
    }
  }
  // second-order part: every row in one launch, or one launch per row
  if (fuse_second && pk > 0) {
    int blocks = 0;
    GPRX_CUDA_TRY(hess_second_all(kern, hm, x.p, cap, n, A.p, ld, alpha.p, hs_part.p, &blocks, stream));
    GPRX_CUDA_TRY(reduce_slots(hs_part.p, blocks, HESS_FUSE_SLOTS, HESS_FUSE_SLOTS, hs_res.p + FUS, stream));
  } else {
    for (int i = 0; i < pk; ++i) {
      int blocks = 0;
      GPRX_CUDA_TRY(hess_second(kern, hm, i, x.p, cap, n, A.p, ld, alpha.p, hs_part.p, &blocks, stream));
      GPRX_CUDA_TRY(reduce_slots(hs_part.p, blocks, HESS_MAX_PARAMS, pk - i, hs_res.p + SEC + i * HESS_MAX_PARAMS,
                                 stream));
    }
  }
  GPRX_CUDA_TRY(trace_dev(A.p, ld, n, hs_res.p + TR, stream));
  GPRX_CUDA_TRY(dot_dev(alpha.p, alpha.p, n, hs_res.p + AA, status.p, stream));
  // first-order part with X = L⁻¹: S_i = X A_i Xᵀ (lower triangle; P = X A_i
  // with k up to the row, then P Xᵀ on the lower tiles with k up to the
  // column: 4n³/3 flop in place of 2n³), ⟨S_i, S_j⟩ over the lower triangles,
  // v_i = X (A_i α) and v_iᵀ v_j.  The noise's S is σn² X Xᵀ and its v is
  // σn² X α: both scaled on the host.
  double* P = hs_p.p;
  double* D = hs_d.p;
  double* V = hs_v.p;                   // n × p: v_i
  double* u = hs_v.p + (size_t)n * p;   // n: A_i α
  const bool emu = use_emu();
  EmuWork ew;
  EmuOperand ex;
  if (emu) {
    // the mixed form emulates both products on the int8 tensor cores
    if ((st = ensure_emu()) != GPRX_OK) return st;
    ew.sa = emu_sa.p; ew.sb = emu_sb.p; ew.ea = emu_ea.p; ew.eb = emu_eb.p; ew.ma = emu_ma.p; ew.mb = emu_mb.p;
    ew.err = emu_err.p;
    ew.S = 7;
    GPRX_CUDA_TRY(cudaMemsetAsync(emu_err.p, 0, sizeof(int), stream));
    ex = ew.op_a(n, n);
    GPRX_CUDA_TRY(emu_slice(Xinv.p, ld, false, ex, stream));  // rows of X
  }
  auto sandwich = [&](const double* Dm, double* S) -> gprx_status {
    if (emu) {
      EmuOperand eb = ew.op_b(n, n);
      GPRX_CUDA_TRY(emu_slice(Dm, ld, true, eb, stream));
      GPRX_CUDA_TRY(emu_gemm(ex, eb, P, ld, 1.0, 0.0, false, 0, 0, 3, ew.err, stream));
      GPRX_CUDA_TRY(emu_slice(P, ld, false, eb, stream));
      GPRX_CUDA_TRY(emu_gemm(eb, ex, S, ld, 1.0, 0.0, true, 0, 0, 4, ew.err, stream));
    } else {
      GemmParams p1 = gemm_params(n, n, n, Xinv.p, ld, Dm, ld, P, ld, 1.0, 0.0, status.p);
      p1.mode = GEMM_K_TO_ROW;
      GPRX_CUDA_TRY(dgemm(false, false, p1, stream));
      GemmParams p2 = gemm_params(n, n, n, P, ld, Xinv.p, ld, S, ld, 1.0, 0.0, status.p);
      p2.mode = GEMM_LOWER_TILES | GEMM_K_TO_COL;
      GPRX_CUDA_TRY(dgemm(false, true, p2, stream));
    }
    return GPRX_OK;
  };
  for (int i = 0; i < pk; ++i) {
    GPRX_CUDA_TRY(fill_deriv(kern, hm, i, x.p, cap, n, D, ld, stream));
    GPRX_CUDA_TRY(gemv_t(D, ld, n, n, false, alpha.p, u, status.p, stream));
    GPRX_CUDA_TRY(trmv_lower(Xinv.p, ld, n, u, V + (size_t)i * n, status.p, stream));
    if ((st = sandwich(D, hs_s.p + (size_t)i * nn)) != GPRX_OK) return st;
  }
  // noise: X Xᵀ (lower) and X α
  {
    double* Sn = hs_s.p + (size_t)pk * nn;
    GemmParams pn = gemm_params(n, n, n, Xinv.p, ld, Xinv.p, ld, Sn, ld, 1.0, 0.0, status.p);
    pn.mode = GEMM_LOWER_TILES | GEMM_K_TO_COL;
    GPRX_CUDA_TRY(dgemm(false, true, pn, stream));
    GPRX_CUDA_TRY(trmv_lower(Xinv.p, ld, n, alpha.p, V + (size_t)pk * n, status.p, stream));
  }
  // VD(i, j) = v_iᵀ v_j, p × p column-major
  GPRX_CUDA_TRY(dgemm(true, false, gemm_params(p, p, n, V, n, V, n, hs_res.p + VD, p, 1.0, 0.0, status.p), stream));
  if (fuse_trace) {
    HessMats mats{};
    for (int i = 0; i < p; ++i) mats.m[i] = hs_s.p + (size_t)i * nn;
    int blocks = 0;
    GPRX_CUDA_TRY(sym_products(mats, p, ld, n, hs_part.p, &blocks, stream));
    GPRX_CUDA_TRY(reduce_slots(hs_part.p, blocks, HESS_TRACE_SLOTS, HESS_TRACE_SLOTS, hs_res.p + TRF, stream));
  } else {
    for (int i = 0; i < p; ++i)
      for (int j = 0; j <= i; ++j) {
        HessMats mats{};
        mats.m[0] = hs_s.p + (size_t)j * nn;
        mats.m[1] = hs_s.p + (size_t)i * nn;
        int blocks = 0;
        GPRX_CUDA_TRY(sym_products(mats, 2, ld, n, hs_part.p, &blocks, stream));
        // slot 1 of the packed triangle is ⟨M_1, M_0⟩
        GPRX_CUDA_TRY(reduce_slots(hs_part.p + 1, blocks, HESS_TRACE_SLOTS, 1, hs_res.p + FRO + i * p + j, stream));
      }
  }
  if (emu) GPRX_CUDA_TRY(cudaMemcpyAsync(emu_err_h.p, emu_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(hs_res_h.p, hs_res.p, sizeof(double) * nres, cudaMemcpyDeviceToHost, stream));
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, jitter, n, GPRX_STAGE_FIT);
  if (use_emu() && *emu_err_h.p != 0) return set_error(GPRX_TIMEOUT, "an emulated product's bounded wait ran out");
  const double* r = hs_res_h.p;
  const double s2 = noise();
  std::vector<double> h((size_t)p * p, 0.0);
  // packed slots of the fused kernels: second-order (a ≤ b) row by row over
  // HESS_FUSE_K columns, trace products (j ≤ i) row by row
  auto sec = [&](int i, int j) {
    if (!fuse_second) return r[SEC + i * HESS_MAX_PARAMS + (j - i)];
    return r[FUS + i * HESS_FUSE_K - i * (i - 1) / 2 + (j - i)];
  };
  auto fro = [&](int i, int j) { return fuse_trace ? r[TRF + i * (i + 1) / 2 + j] : r[FRO + i * p + j]; };
  for (int i = 0; i < pk; ++i)
    for (int j = i; j < pk; ++j) h[(size_t)i * p + j] = h[(size_t)j * p + i] = -0.5 * sec(i, j);
  h[(size_t)pk * p + pk] = -0.5 * s2 * (r[AA] - r[TR]);
  for (int i = 0; i < p; ++i)
    for (int j = 0; j <= i; ++j) {
      const double sc = (i == pk ? s2 : 1.0) * (j == pk ? s2 : 1.0);
      const double add = sc * (-0.5 * fro(i, j) + r[VD + i + j * p]);
      h[(size_t)i * p + j] += add;
      if (i != j) h[(size_t)j * p + i] += add;
    }
  for (size_t e = 0; e < h.size(); ++e)
    if (!std::isfinite(h[e])) return set_error(GPRX_NOT_CONVERGED, "non-finite Hessian entry");
  std::copy(h.begin(), h.end(), out);
  return GPRX_OK;
}

gprx_status ExactState::nlml(double* out) {
  gprx_status st;
  if (online) {
    if (!alpha_ok && (st = online_alpha()) != GPRX_OK) return st;
  } else if (!factor_ok || !alpha_ok) {
    if ((st = factor_current()) != GPRX_OK) return st;
  }
  if ((st = reset_status()) != GPRX_OK) return st;
  GPRX_CUDA_TRY(logdet_diag(A.p, ld, n, online, res.p + 0, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(y.p, alpha.p, n, res.p + 1, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, jitter, n, GPRX_STAGE_FIT);
  *out = 0.5 * (res_h.p[1] + res_h.p[0] + (double)n * std::log(2.0 * M_PI));
  return GPRX_OK;
}

// var = max(0, k** − quad) (+ σn² for observation variance); shared.rs:792-806
__global__ void finish_var_kernel(const double* quad, int q, double kss, double noise, int kind, double* var,
                                  const DevStatus* st) {
  if (dev_failed(st)) return;
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= q) return;
  double lat = kss - quad[j];
  if (lat < 0.0) lat = 0.0;
  var[j] = kind == GPRX_VARIANCE_OBSERVATION ? lat + noise : lat;
}

__global__ void extract_diag_kernel(const double* A, long long ld, int n, double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = A[i + (long long)i * ld];
}

// ---------------------------------------------------------------------------
// leave-one-out, query covariance and posterior draws
// ---------------------------------------------------------------------------
static unsigned blocks_for(long long count) { return (unsigned)((count + 255) / 256); }

// The resident factor of the current θ: L (LLT) with α, or the online LDLT
// with α solved and the unit diagonal-block inverses in linv.
gprx_status ExactState::ready_for_query() {
  gprx_status st;
  if (online) {
    if (!alpha_ok && (st = online_alpha()) != GPRX_OK) return st;
    if (!linv_ok) {
      if ((st = reset_status()) != GPRX_OK) return st;
      GPRX_CUDA_TRY(tri_inv_blocks(A.p, ld, n, true, linv.p, status.p, stream));
      linv_ok = true;
    }
    GPRX_CUDA_TRY(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), stream));
    extract_diag_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(A.p, ld, n, tmpv.p);
    count_launch();
  } else if (!factor_ok || !alpha_ok) {
    if ((st = factor_current()) != GPRX_OK) return st;
  }
  return GPRX_OK;
}

// mean_i = y_i − α_i / Q_ii, variance from 1 / Q_ii (src/gpr/shared.rs:538-555)
__global__ void loo_kernel(const double* y, const double* alpha, const double* qd, int n, double noise, int kind,
                           double* out, DevStatus* st) {
  if (dev_failed(st)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double q = qd[i];
  if (!(q > 0.0) || !isfinite(q)) {
    dev_fail(st, GPRX_NOT_POSITIVE_DEFINITE, i);
    return;
  }
  out[i] = y[i] - alpha[i] / q;
  const double obs = 1.0 / q;
  out[n + i] = kind == GPRX_VARIANCE_OBSERVATION ? obs : fmax(obs - noise, 0.0);
}

gprx_status ExactState::loo(int kind, double* mean, double* var) {
  if (!mean || !var) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (kind != GPRX_VARIANCE_LATENT && kind != GPRX_VARIANCE_OBSERVATION)
    return set_error(GPRX_INVALID_ARGUMENT, "variance kind");
  gprx_status st;
  if ((st = ready_for_query()) != GPRX_OK) return st;
  const size_t nn = (size_t)ld * cap;
  if (Xinv.n < nn) {
    size_t half = (size_t)((n + 1) / 2) * ((n + 1) / 2);
    if (Xinv.alloc(nn) != cudaSuccess || scratch.alloc(std::max<size_t>(half, 1)) != cudaSuccess) {
      Xinv.reset();
      return set_error(GPRX_OUT_OF_MEMORY, "device allocation of the inverse failed");
    }
    GPRX_CUDA_TRY(cudaMemsetAsync(Xinv.p, 0, sizeof(double) * nn, stream));
  } else if (scratch.n < (size_t)((n + 1) / 2) * ((n + 1) / 2)) {
    if (scratch.alloc((size_t)((n + 1) / 2) * ((n + 1) / 2)) != cudaSuccess)
      return set_error(GPRX_OUT_OF_MEMORY, "scratch");
  }
  if (qx.ensure((size_t)3 * n) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "scratch");
  // Q_ii = Σ_k (L⁻¹)_ki² / w_k (w = 1 for LLT, D for the online LDLT)
  GPRX_CUDA_TRY(trtri_blocked(A.p, ld, n, linv.p, Xinv.p, ld, scratch.p, status.p, stream));
  GPRX_CUDA_TRY(col_sumsq(Xinv.p, ld, n, n, online ? tmpv.p : nullptr, qx.p, status.p, stream));
  GPRX_LAUNCH(loo_kernel, ceil_div(n, 256), 256, 0, stream, y.p, alpha.p, qx.p, n, noise(), kind, qx.p + n,
              status.p);
  std::vector<double> h(2 * (size_t)n);
  GPRX_CUDA_TRY(cudaMemcpyAsync(h.data(), qx.p + n, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, stream));
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code == GPRX_NOT_POSITIVE_DEFINITE)
    return set_error(GPRX_NOT_POSITIVE_DEFINITE, "leave-one-out: [K⁻¹]_ii ≤ 0 at row " + std::to_string(ds.info));
  if (ds.code != GPRX_OK) return status_to_error(ds, jitter, n, GPRX_STAGE_PREDICT);
  std::copy(h.begin(), h.begin() + n, mean);
  std::copy(h.begin() + n, h.end(), var);
  return GPRX_OK;
}

// V := V ⊘ √w (row i scaled by 1 / √w_i)
__global__ void scale_rows_kernel(double* V, long long ld, int n, int q, const double* w) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)n * q) return;
  const int i = (int)(e % n), c = (int)(e / n);
  V[i + c * ld] /= sqrt(w[i]);
}

// C (q×q, lower computed) → full symmetric; diagonal clipped at 0 (latent)
// or plus σn² (observation)
__global__ void cov_finish_kernel(double* C, int q, double noise, int kind) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)q * q) return;
  const int i = (int)(e % q), j = (int)(e / q);
  if (i < j) {
    C[i + (long long)j * q] = C[j + (long long)i * q];
  } else if (i == j) {
    double v = C[i + (long long)i * q];
    if (v < 0.0) v = 0.0;
    C[i + (long long)i * q] = kind == GPRX_VARIANCE_OBSERVATION ? v + noise : v;
  }
}

// covbuf (q×q, ld q) = predictive covariance; mean to the host
gprx_status ExactState::covariance_dev(const double* xs, uint64_t q, int kind, double* mean_host) {
  if (kind != GPRX_VARIANCE_LATENT && kind != GPRX_VARIANCE_OBSERVATION)
    return set_error(GPRX_INVALID_ARGUMENT, "variance kind");
  if (q > (uint64_t)INT32_MAX) return set_error(GPRX_CAPACITY, "too many query points");
  if (!all_finite(xs, q * d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite query");
  gprx_status st;
  if ((st = ready_for_query()) != GPRX_OK) return st;
  const int qi = (int)q;
  if (qbuf.ensure((size_t)ld * q) != cudaSuccess || qx.ensure((size_t)q * (d + 1)) != cudaSuccess ||
      covbuf.ensure((size_t)q * q) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "covariance buffers");
  double* xq = qx.p;  // q × d
  double* mdev = qx.p + (size_t)q * d;
  GPRX_CUDA_TRY(cudaMemcpyAsync(xq, xs, sizeof(double) * q * d, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(fill_cross(kern, x.p, cap, n, xq, qi, qi, qbuf.p, ld, status.p, stream));
  GPRX_CUDA_TRY(gemv_t(qbuf.p, ld, n, qi, false, alpha.p, mdev, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower(A.p, ld, n, linv.p, qbuf.p, ld, qi, status.p, stream));
  if (online) GPRX_LAUNCH(scale_rows_kernel, blocks_for((long long)n * qi), 256, 0, stream, qbuf.p, ld, n, qi, tmpv.p);
  // K** (lower), then K** − VᵀV on the lower tiles
  GPRX_CUDA_TRY(fill_lower(kern, xq, qi, qi, covbuf.p, qi, 0.0, status.p, stream));
  GemmParams p = gemm_params(qi, qi, n, qbuf.p, ld, qbuf.p, ld, covbuf.p, qi, -1.0, 1.0, status.p);
  p.mode = GEMM_LOWER_TILES;
  GPRX_CUDA_TRY(dgemm(true, false, p, stream));
  GPRX_LAUNCH(cov_finish_kernel, blocks_for((long long)qi * qi), 256, 0, stream, covbuf.p, qi, noise(), kind);
  GPRX_CUDA_TRY(cudaMemcpyAsync(mean_host, mdev, sizeof(double) * q, cudaMemcpyDeviceToHost, stream));
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, jitter, n, GPRX_STAGE_PREDICT);
  return GPRX_OK;
}

gprx_status ExactState::predict_covariance(const double* xs, uint64_t q, int kind, double* mean, double* cov) {
  if (!xs || !mean || !cov) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (q == 0) return GPRX_OK;
  gprx_status st = covariance_dev(xs, q, kind, mean);
  if (st != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpyAsync(cov, covbuf.p, sizeof(double) * q * q, cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  return GPRX_OK;
}

// out(:, k) = μ + L z_k (L lower, its upper part zeroed first)
__global__ void zero_upper_kernel(double* L, int q) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)q * q) return;
  const int i = (int)(e % q), j = (int)(e / q);
  if (i < j) L[i + (long long)j * q] = 0.0;
}
__global__ void add_mean_kernel(double* out, const double* mean, int q, long long count) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e < count) out[e] += mean[e % q];
}
__global__ void add_diag_q_kernel(double* C, int q, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < q) C[i + (long long)i * q] += v;
}

gprx_status ExactState::sample(const double* xs, uint64_t q, int kind, uint64_t n_draws, uint64_t seed,
                               double* out) {
  if (!xs || (n_draws > 0 && !out)) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (q == 0) return GPRX_OK;
  if (n_draws > (uint64_t)INT32_MAX) return set_error(GPRX_CAPACITY, "too many draws");
  std::vector<double> mean(q);
  gprx_status st = covariance_dev(xs, q, kind, mean.data());
  if (st != GPRX_OK || n_draws == 0) return st;
  return draw_posterior(covbuf.p, (int)q, mean.data(), n_draws, seed, jitter_attempts(opt), covl, covlinv, zbuf, status.p,
                        stream, [&] { return reset_status(); }, [&](DevStatus* ds) { return read_status(ds); }, out);
}

// LLT of the covariance with the model's jitter retries (src/linalg/chol.rs:20-43,83-103),
// q unit normals per draw from the seeded generator (src/rng.rs:83-87), out(:, k) = μ + L z_k
// (src/prediction.rs:206-243).
gprx_status draw_posterior(const double* cov, int qi, const double* mean_host, uint64_t n_draws, uint64_t seed,
                           const std::vector<double>& js, DevBuf<double>& covl, DevBuf<double>& covlinv,
                           DevBuf<double>& zbuf, DevStatus* st_dev, cudaStream_t stream,
                           const std::function<gprx_status()>& reset,
                           const std::function<gprx_status(DevStatus*)>& read, double* out) {
  if (n_draws == 0) return GPRX_OK;
  const size_t q = (size_t)qi;
  const int nd = (int)n_draws;
  const size_t nblk = (size_t)ceil_div(qi, NB);
  if (covl.ensure(q * q) != cudaSuccess || covlinv.ensure(nblk * NB * NB) != cudaSuccess ||
      zbuf.ensure(q * n_draws * 2 + q) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "draw buffers");
  gprx_status st;
  bool ok = false;
  double last = 0.0;
  for (double j : js) {
    last = j;
    if ((st = reset()) != GPRX_OK) return st;
    GPRX_CUDA_TRY(cudaMemcpyAsync(covl.p, cov, sizeof(double) * q * q, cudaMemcpyDeviceToDevice, stream));
    if (j != 0.0) GPRX_LAUNCH(add_diag_q_kernel, ceil_div(qi, 256), 256, 0, stream, covl.p, qi, j);
    GPRX_CUDA_TRY(potrf_blocked(covl.p, qi, qi, covlinv.p, st_dev, stream, nullptr));
    DevStatus ds;
    if ((st = read(&ds)) != GPRX_OK) return st;
    if (ds.code == GPRX_OK) {
      ok = true;
      break;
    }
    if (ds.code != GPRX_CHOLESKY_FAILED) return status_to_error(ds, j, q, GPRX_STAGE_PREDICT);
  }
  if (!ok) return set_cholesky_error(last, q, GPRX_STAGE_PREDICT);
  std::vector<double> z(q * n_draws);
  gprx_rng rng;
  gprx_rng_seed(&rng, seed);
  gprx_rng_fill_normal(&rng, z.data(), z.size());
  double* zd = zbuf.p;
  double* od = zbuf.p + q * n_draws;
  double* md = od + q * n_draws;
  GPRX_CUDA_TRY(cudaMemcpyAsync(zd, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(md, mean_host, sizeof(double) * q, cudaMemcpyHostToDevice, stream));
  GPRX_LAUNCH(zero_upper_kernel, blocks_for((long long)qi * qi), 256, 0, stream, covl.p, qi);
  GemmParams p = gemm_params(qi, nd, qi, covl.p, qi, zd, qi, od, qi, 1.0, 0.0, st_dev);
  p.mode = GEMM_K_TO_ROW;
  GPRX_CUDA_TRY(dgemm(false, false, p, stream));
  GPRX_LAUNCH(add_mean_kernel, blocks_for((long long)qi * nd), 256, 0, stream, od, md, qi, (long long)qi * nd);
  GPRX_CUDA_TRY(cudaMemcpyAsync(out, od, sizeof(double) * q * n_draws, cudaMemcpyDeviceToHost, stream));
  DevStatus ds;
  if ((st = read(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, 0.0, q, GPRX_STAGE_PREDICT);
  return GPRX_OK;
}

// ---------------------------------------------------------------------------
// saved models (FittedGpr::save / save_with_factor, OnlineGpr::save;
// LoadedGpr::load, src/persist/mod.rs)
// ---------------------------------------------------------------------------
gprx_status ExactState::save(const char* dir, bool with_factor) {
  if (!dir) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  gprx_status st;
  PersistModel m;
  m.n = n;
  m.d = d;
  m.nodes = kern.nodes;
  m.theta = kern.theta;
  m.log_noise = log_noise;
  m.jitter = opt;
  m.x.resize((size_t)n * d);
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(m.x.data(), sizeof(double) * n, x.p, sizeof(double) * cap, sizeof(double) * n, d,
                                  cudaMemcpyDeviceToHost, stream));
  m.y.resize(n);
  GPRX_CUDA_TRY(cudaMemcpyAsync(m.y.data(), y.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
  m.ldlt = online;
  if (online) {
    m.ids = ids;
    m.next_id = next_id;
  }
  if (with_factor) {
    if (online) {
      if (!alpha_ok && (st = online_alpha()) != GPRX_OK) return st;
    } else if (!factor_ok || !alpha_ok) {
      if ((st = factor_current()) != GPRX_OK) return st;
    }
    m.has_factor = true;
    m.factor_jitter = online ? 0.0 : jitter;
    m.l.resize((size_t)n * n);
    m.alpha.resize(n);
    GPRX_CUDA_TRY(cudaMemcpy2DAsync(m.l.data(), sizeof(double) * n, A.p, sizeof(double) * ld, sizeof(double) * n, n,
                                    cudaMemcpyDeviceToHost, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(m.alpha.data(), alpha.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
  }
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  if (m.has_factor)
    for (long long j = 0; j < n; ++j)  // the stored layout: zero above the diagonal
      for (long long i = 0; i < j; ++i) m.l[i + j * n] = 0.0;
  return persist_write(dir, m);
}

// L (LLT) or unit-lower L with D on the diagonal (LDLT), n×n column-major on
// the host (a file mapping), and α: the handle then predicts without factoring.
gprx_status ExactState::adopt_factor(const double* l_host, const double* alpha_host, bool ldlt, double factor_jitter,
                                     const std::vector<uint64_t>& point_ids, uint64_t next_point_id) {
  gprx_status st;
  if ((st = reset_status()) != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(A.p, sizeof(double) * ld, l_host, sizeof(double) * n, sizeof(double) * n, n,
                                  cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(alpha.p, alpha_host, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  if (ldlt) {
    online = true;
    factor_ok = false;
    linv_ok = false;
    alpha_ok = true;
    ids = point_ids;
    next_id = next_point_id;
  } else {
    GPRX_CUDA_TRY(tri_inv_blocks(A.p, ld, n, false, linv.p, status.p, stream));
    online = false;
    factor_ok = true;
    linv_ok = true;
    alpha_ok = true;
    jitter = factor_jitter;
  }
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, factor_jitter, n, GPRX_STAGE_PREDICT);
  return GPRX_OK;
}

gprx_status ExactState::predict(const double* xs, uint64_t q, int kind, double* mean, double* var) {
  if (!xs || !mean || !var) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (kind != GPRX_VARIANCE_LATENT && kind != GPRX_VARIANCE_OBSERVATION)
    return set_error(GPRX_INVALID_ARGUMENT, "variance kind");
  if (q == 0) return GPRX_OK;
  if (!all_finite(xs, q * d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite query");
  gprx_status st;
  if (online) {
    if (!alpha_ok && (st = online_alpha()) != GPRX_OK) return st;
    if (!linv_ok) {
      if ((st = reset_status()) != GPRX_OK) return st;
      GPRX_CUDA_TRY(tri_inv_blocks(A.p, ld, n, true, linv.p, status.p, stream));
      linv_ok = true;
    }
    GPRX_CUDA_TRY(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), stream));
    extract_diag_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(A.p, ld, n, tmpv.p);
    count_launch();
  } else if (!factor_ok || !alpha_ok) {
    if ((st = factor_current()) != GPRX_OK) return st;
  }
  const int qc_max = (int)std::max<long long>(1, std::min<long long>((long long)q, (1LL << 27) / std::max(n, 1)));
  if (qbuf.ensure((size_t)ld * qc_max) != cudaSuccess || qx.ensure((size_t)qc_max * (d + 3)) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "predict scratch");
  HostPinned<double> hm;
  GPRX_CUDA_TRY(hm.ensure(2 * (size_t)qc_max));
  const double kss = kern.diag_value();
  for (uint64_t c0 = 0; c0 < q; c0 += qc_max) {
    int qc = (int)std::min<uint64_t>(qc_max, q - c0);
    double* xq = qx.p;                  // qc × d
    double* mdev = qx.p + (size_t)qc_max * d;
    double* vdev = mdev + qc_max;
    double* quad = vdev + qc_max;
    GPRX_CUDA_TRY(cudaMemcpy2DAsync(xq, sizeof(double) * qc, xs + c0, sizeof(double) * q, sizeof(double) * qc, d,
                                    cudaMemcpyHostToDevice, stream));
    GPRX_CUDA_TRY(fill_cross(kern, x.p, cap, n, xq, qc, qc, qbuf.p, ld, status.p, stream));
    GPRX_CUDA_TRY(gemv_t(qbuf.p, ld, n, qc, false, alpha.p, mdev, status.p, stream));
    GPRX_CUDA_TRY(trsm_lower(A.p, ld, n, linv.p, qbuf.p, ld, qc, status.p, stream));
    GPRX_CUDA_TRY(col_sumsq(qbuf.p, ld, n, qc, online ? tmpv.p : nullptr, quad, status.p, stream));
    finish_var_kernel<<<ceil_div(qc, 256), 256, 0, stream>>>(quad, qc, kss, noise(), kind, vdev, status.p);
    count_launch();
    GPRX_CUDA_TRY(cudaMemcpyAsync(hm.p, mdev, sizeof(double) * qc, cudaMemcpyDeviceToHost, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(hm.p + qc_max, vdev, sizeof(double) * qc, cudaMemcpyDeviceToHost, stream));
    DevStatus ds;
    if ((st = read_status(&ds)) != GPRX_OK) return st;
    if (ds.code != GPRX_OK) return status_to_error(ds, jitter, n, GPRX_STAGE_PREDICT);
    std::copy(hm.p, hm.p + qc, mean + c0);
    std::copy(hm.p + qc_max, hm.p + qc_max + qc, var + c0);
  }
  return GPRX_OK;
}

gprx_status ExactState::stage_times(double* out5) {
  if (!ev_recorded) return set_error(GPRX_INVALID_CONFIG, "no evaluation recorded");
  float ms;
  for (int i = 0; i < 4; ++i) {
    GPRX_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
    out5[i] = ms;
  }
  GPRX_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[4]));
  out5[4] = ms;
  return GPRX_OK;
}

}  // namespace gprx
