// exact.cuh — the exact-GPR handle (device state of one Gpr / FittedGpr /
// OnlineGpr).
#pragma once

#include <cmath>
#include <functional>
#include <string>
#include <vector>

#include "dense_f64.cuh"
#include "emu_gemm.cuh"
#include "kernels.cuh"
#include "runtime.cuh"

struct gprx_exact;

namespace gprx {

// JitterPolicy retry offsets after the first attempt (src/policy.rs:306-397),
// and the whole list of attempts starting with no jitter.
std::vector<double> retry_list(const gprx_options& o);
std::vector<double> jitter_attempts(const gprx_options& o);

// out (q × n_draws, column k = draw k, host) = μ + L z_k: L the LLT of the
// q×q device covariance `cov` under the jitter attempts js, z_k standard
// normals from the seeded generator.  reset / read clear and read the
// caller's device status word st_dev.
gprx_status draw_posterior(const double* cov, int q, const double* mean_host, uint64_t n_draws, uint64_t seed,
                           const std::vector<double>& js, DevBuf<double>& covl, DevBuf<double>& covlinv,
                           DevBuf<double>& zbuf, DevStatus* st_dev, cudaStream_t stream,
                           const std::function<gprx_status()>& reset,
                           const std::function<gprx_status(DevStatus*)>& read, double* out);

struct ExactState {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n = 0, d = 0;
  long long ld = 0;        // leading dimension of the n×n buffers
  int cap = 0;             // online capacity (rows/cols the buffers hold)
  gprx_options opt{};
  HostKernel kern;
  double log_noise = 0.0;
  std::vector<double> y_host;  // y in buffer order (online compaction)

  DevBuf<double> x;        // cap×d (column-major, ld = cap)
  DevBuf<double> y;        // cap
  DevBuf<double> A;        // ld×cap: K → L (→ K⁻¹ after a gradient; → LDLT online)
  DevBuf<double> Xinv;     // ld×cap: L⁻¹ (gradient path; strict upper triangle kept zero)
  DevBuf<double> scratch;  // ceil(n/2)² doubles for the recursive triangular inverse
  DevBuf<double> linv;     // diagonal-block inverses
  DevBuf<double> alpha, z, tmpv;
  DevBuf<double> partials;
  DevBuf<int> slot_param;
  DevBuf<double> res;      // [0] logdet, [1] yᵀα, [2..] grad
  DevBuf<DevStatus> status;
  FactorCtx fctx;          // side stream + events of the look-ahead factor
  HostPinned<double> res_h;
  HostPinned<DevStatus> status_h;
  DevBuf<double> qbuf, qx;  // predict scratch
  DevBuf<unsigned char> group_dev;       // grouped-predict staging (this handle leads the group)
  HostPinned<unsigned char> group_host;
  // mixed precision: the inverse's products emulated on the int8 tensor cores
  DevBuf<int8_t> emu_sa, emu_sb;
  DevBuf<int> emu_ea, emu_eb, emu_err;
  DevBuf<unsigned long long> emu_ma, emu_mb;
  HostPinned<int> emu_err_h;

  bool factor_ok = false;   // A holds L (LLT) of the current θ
  bool alpha_ok = false;
  bool online = false;      // A holds LDLT
  bool linv_ok = false;     // linv matches A's diagonal blocks
  double jitter = 0.0;
  std::vector<uint64_t> ids;
  uint64_t next_id = 0;

  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  bool ev_recorded = false;

  ~ExactState();
  gprx_status create(const double* x, uint64_t n, uint64_t d, const double* y, const gprx_kernel_node* nodes,
                     int n_nodes, const double* theta, int n_theta, const gprx_options* o);
  int num_params() const { return kern.n_params + 1; }
  // smallest n whose inverse uses the emulated products
  static constexpr int EMU_MIN_N = 1024;
  // blocks the recursive mixed factor hands to the blocked DMMA factor (a
  // sweep at n = 8192 over 1024 / 2048 / 4096 measured 24.9 / 23.1 / 21.7 ms
  // per evaluation: the blocked factor's look-ahead beats the extra coupling
  // products of deeper recursion)
  static constexpr int EMU_LEAF_N = 4096;
  // largest n (the longest K of a product) whose 7-digit int32 sums stay
  // exact: K·7·2^12 < 2^31; larger n runs the FP64 products
  static constexpr int EMU_MAX_N = 65536;
  bool use_emu() const { return opt.precision == GPRX_PRECISION_MIXED && n >= EMU_MIN_N && n <= EMU_MAX_N; }
  gprx_status ensure_emu();
  void get_params(double* out) const;
  gprx_status write_params(const double* params);
  double noise() const { return std::exp(log_noise); }

  // Enqueues fill + potrf for one jitter attempt.
  gprx_status enqueue_factor(double j);
  // fill + potrf with the jitter retries; syncs; on success A holds L.
  gprx_status factor_with_retries(int stage);
  gprx_status solve_alpha_from_l();
  gprx_status factor_current();
  gprx_status eval(const double* params, double* nlml, double* grad);
  gprx_status nlml(double* out);
  // Hessian of the NLML at params (row-major p × p); the value and the
  // gradient of the same evaluation when nlml_out / grad_out are given
  DevBuf<double> hs_s, hs_p, hs_d, hs_v, hs_part, hs_res;
  HostPinned<double> hs_res_h;
  gprx_status hessian(const double* params, double* out, double* nlml_out = nullptr, double* grad_out = nullptr);
  gprx_status predict(const double* xs, uint64_t q, int kind, double* mean, double* var);
  // leave-one-out, query covariance and posterior draws from the resident factor
  DevBuf<double> covbuf, covl, covlinv, zbuf;
  gprx_status ready_for_query();
  gprx_status loo(int kind, double* mean, double* var);
  gprx_status covariance_dev(const double* xs, uint64_t q, int kind, double* mean_host);
  gprx_status predict_covariance(const double* xs, uint64_t q, int kind, double* mean, double* cov);
  gprx_status sample(const double* xs, uint64_t q, int kind, uint64_t n_draws, uint64_t seed, double* out);
  // saved models (persist.cpp): write this model; read a stored factor in
  gprx_status save(const char* dir, bool with_factor);
  gprx_status adopt_factor(const double* l_host, const double* alpha_host, bool ldlt, double factor_jitter,
                           const std::vector<uint64_t>& point_ids, uint64_t next_point_id);
  gprx_status reset_status();
  gprx_status read_status(DevStatus* out);
  gprx_status stage_times(double* out5);

  // online (LDLT)
  gprx_status online_begin();
  // Runs op (θ writes, evaluations, Hessians) on an online model through a
  // plain LLT: afterwards A is the LDLT at the model's θ again, and a failed
  // op leaves the LDLT, α and the jitter as they were
  // (with_llt_view, src/gpr/online.rs:1151-1185).
  DevBuf<double> ldlt_keep, alpha_keep;
  gprx_status with_llt_view(const std::function<gprx_status()>& op);
  gprx_status online_insert(const double* xnew, double ynew, uint64_t* id);
  gprx_status online_delete(uint64_t id);
  gprx_status online_alpha();
  gprx_status grow(int needed);
};

}  // namespace gprx

struct gprx_exact {
  gprx::ExactState s;
};
