// predict_group.cu — one launch that predicts for many small requests against
// different fitted exact models (the serving loop's same-phase batching of
// predicts; no counterpart in the reference, where each request is one
// FittedGpr::predict_with, src/gpr/shared.rs:754-820).
//
// A CTA takes one (request, 16-query tile) item and walks the model's
// training points in 128-row blocks b:
//   K*_b  = k(x_b, x*)                      (128 × 16, in shared memory)
//   mean += K*_bᵀ α_b
//   V_b   = L_bb⁻¹ (K*_b − Σ_{c<b} L_bc V_c)  (DMMA; L from the model's factor,
//                                           L_bb⁻¹ from its diagonal-block inverses)
// and ends with var = max(0, k(x*, x*) − Σ V²) (+ σn² for the observation
// variance).  V of the request stays in shared memory (n ≤ 1024 rows), so a
// model's L is read once per tile and no other buffer is written.  Every item
// is computed in a fixed order by one CTA: a request's results do not depend
// on the other requests of the launch.

#include <algorithm>
#include <vector>

#include "exact.cuh"
#include "gemm_f64.cuh"

namespace gprx {

constexpr int PG_THREADS = 256;
constexpr int PG_Q = 16;         // queries per CTA
constexpr int PG_NMAX = 1024;    // training points of a grouped model
constexpr int PG_DMAX = 16;      // features of a grouped model
constexpr int PG_B = 128;        // row block (= the factor's diagonal block)
constexpr int PG_VLD = PG_Q + 4;  // ld of V and of the block (≡ 4 mod 16: conflict-free fragments)

struct GroupReq {
  KTree t;
  const double* x;      // training points, column-major, ld ldx
  long long ldx;
  int n;
  int q;                // queries of the request
  const double* L;      // factor (lower), ld
  long long ld;
  const double* linv;   // diagonal-block inverses, PG_B × PG_B each
  const double* alpha;
  const double* xq;     // queries, column-major q × d (ld q)
  double* out;          // mean (q) then variance (q)
  double noise;
  double kss;           // k(x*, x*)
  int kind;
};

inline size_t pg_smem(int d) {
  return sizeof(double) * ((size_t)PG_NMAX * PG_VLD + (size_t)PG_B * PG_VLD + (size_t)PG_B * d + (size_t)PG_Q * d +
                           2 * PG_THREADS);
}


// One item per CTA: items[blockIdx.x] = (request, first query of the tile).
template <int ARD_D>
__global__ void __launch_bounds__(PG_THREADS) predict_group_kernel(const GroupReq* reqs, const int2* items,
                                                                    DevStatus* st) {
  extern __shared__ __align__(16) double sm[];
  if (dev_failed(st)) return;
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  const GroupReq& R = reqs[items[blockIdx.x].x];
  const int j0 = items[blockIdx.x].y;
  const KTree& t = R.t;
  const int d = t.d, n = R.n;
  double* V = sm;                          // PG_NMAX × PG_VLD (row i, query j)
  double* Kb = V + PG_NMAX * PG_VLD;       // PG_B × PG_VLD
  double* xb = Kb + PG_B * PG_VLD;         // PG_B × d (feature-major)
  double* xq = xb + PG_B * d;              // PG_Q × d (feature-major)
  double* red = xq + PG_Q * d;             // 2 × PG_THREADS
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  const int qj = tid & (PG_Q - 1), grp = tid / PG_Q;  // the thread's query and row group (16 groups)
  for (int e = tid; e < PG_Q * d; e += PG_THREADS) {
    const int j = e % PG_Q, f = e / PG_Q;
    xq[f * PG_Q + j] = (j0 + j < R.q) ? R.xq[(j0 + j) + (long long)f * R.q] : 0.0;
  }
  double mean_acc = 0.0, var_acc = 0.0;
  bool bad = false;
  const int nblk = (n + PG_B - 1) / PG_B;
  for (int b = 0; b < nblk; ++b) {
    const int r0 = b * PG_B, rows = min(PG_B, n - r0);
    __syncthreads();
    for (int e = tid; e < PG_B * d; e += PG_THREADS) {
      const int i = e % PG_B, f = e / PG_B;
      xb[f * PG_B + i] = (i < rows) ? R.x[(r0 + i) + (long long)f * R.ldx] : 0.0;
    }
    __syncthreads();
    // K*_b (rows beyond n are zero) and the mean's partial sums
    for (int e = tid; e < PG_B * PG_Q; e += PG_THREADS) {
      const int i = e / PG_Q, j = e % PG_Q;
      double v = 0.0;
      if (i < rows) {
        double dx[AD];
        double r2 = 0.0;
        for (int f = 0; f < d; ++f) {
          const double u = xb[f * PG_B + i] - xq[f * PG_Q + j];
          r2 = fma(u, u, r2);
          if (ARD_D > 0) {
#pragma unroll
            for (int h = 0; h < AD; ++h)
              if (h == f) dx[h] = u;
          }
        }
        v = kt_value<ARD_D>(t, dx, r2);
        if (!isfinite(v)) bad = true;
        mean_acc = fma(v, R.alpha[r0 + i], mean_acc);  // thread (i, j) with j = tid % 16: fixed rows per thread
      }
      Kb[i * PG_VLD + j] = v;
    }
    __syncthreads();
    // acc = K*_b − Σ_{c<b} L_bc V_c: warp w owns rows 16w..16w+15, two 8-query tiles
    {
      double c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
      const int ra = min(r0 + 16 * warp + g, n - 1), rb = min(r0 + 16 * warp + g + 8, n - 1);
      const double* La = R.L + ra;
      const double* Lb = R.L + rb;
#pragma unroll 4
      for (int k = 0; k < r0; k += 4) {
        const double a0 = La[(long long)(k + t4) * R.ld], a1 = Lb[(long long)(k + t4) * R.ld];
        dmma_16x8x4(c0, a0, a1, V[(k + t4) * PG_VLD + g]);
        dmma_16x8x4(c1, a0, a1, V[(k + t4) * PG_VLD + 8 + g]);
      }
      const int row = 16 * warp + g, col = 2 * t4;
      Kb[row * PG_VLD + col] -= c0[0];
      Kb[row * PG_VLD + col + 1] -= c0[1];
      Kb[(row + 8) * PG_VLD + col] -= c0[2];
      Kb[(row + 8) * PG_VLD + col + 1] -= c0[3];
      Kb[row * PG_VLD + 8 + col] -= c1[0];
      Kb[row * PG_VLD + 8 + col + 1] -= c1[1];
      Kb[(row + 8) * PG_VLD + 8 + col] -= c1[2];
      Kb[(row + 8) * PG_VLD + 8 + col + 1] -= c1[3];
    }
    __syncthreads();
    // V_b = L_bb⁻¹ acc (lower: k up to the warp's last row)
    {
      double c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
      const double* Li = R.linv + (long long)b * PG_B * PG_B + 16 * warp + g;
#pragma unroll 4
      for (int k = 0; k < 16 * warp + 16; k += 4) {
        const double a0 = Li[(k + t4) * PG_B], a1 = Li[8 + (k + t4) * PG_B];
        dmma_16x8x4(c0, a0, a1, Kb[(k + t4) * PG_VLD + g]);
        dmma_16x8x4(c1, a0, a1, Kb[(k + t4) * PG_VLD + 8 + g]);
      }
      const int row = 16 * warp + g, col = 2 * t4;
      const bool ok0 = row < rows, ok1 = row + 8 < rows;
      double* v0 = V + (r0 + row) * PG_VLD;
      double* v1 = V + (r0 + row + 8) * PG_VLD;
      v0[col] = ok0 ? c0[0] : 0.0;
      v0[col + 1] = ok0 ? c0[1] : 0.0;
      v1[col] = ok1 ? c0[2] : 0.0;
      v1[col + 1] = ok1 ? c0[3] : 0.0;
      v0[8 + col] = ok0 ? c1[0] : 0.0;
      v0[8 + col + 1] = ok0 ? c1[1] : 0.0;
      v1[8 + col] = ok1 ? c1[2] : 0.0;
      v1[8 + col + 1] = ok1 ? c1[3] : 0.0;
    }
  }
  __syncthreads();
  // ‖v_j‖²: thread (group, j) sums rows group, group + 16, …; the groups in order
  for (int i = grp; i < nblk * PG_B; i += PG_THREADS / PG_Q) {
    const double v = V[i * PG_VLD + qj];
    var_acc = fma(v, v, var_acc);
  }
  red[tid] = mean_acc;
  red[PG_THREADS + tid] = var_acc;
  __syncthreads();
  if (tid < PG_Q && j0 + tid < R.q) {
    double m = 0.0, s = 0.0;
    for (int gi = 0; gi < PG_THREADS / PG_Q; ++gi) {
      m += red[gi * PG_Q + tid];
      s += red[PG_THREADS + gi * PG_Q + tid];
    }
    double lat = R.kss - s;
    if (lat < 0.0) lat = 0.0;
    R.out[j0 + tid] = m;
    R.out[R.q + j0 + tid] = R.kind == GPRX_VARIANCE_OBSERVATION ? lat + R.noise : lat;
  }
  if (bad) dev_fail(st, GPRX_NONFINITE_KERNEL, 0);
}

static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Grouped prediction through the handles' factors; the first handle's stream,
// staging buffers and status word serve the launch.
static gprx_status predict_group(gprx_exact* const* hs, uint64_t k, const double* const* xs, const uint64_t* qs,
                                 int kind, double* const* means, double* const* vars) {
  if (!hs || !xs || !qs || !means || !vars || k == 0) return set_error(GPRX_INVALID_ARGUMENT, "null pointer or k = 0");
  if (kind != GPRX_VARIANCE_LATENT && kind != GPRX_VARIANCE_OBSERVATION)
    return set_error(GPRX_INVALID_ARGUMENT, "variance kind");
  for (uint64_t i = 0; i < k; ++i)
    if (!hs[i] || !xs[i] || !means[i] || !vars[i]) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  ExactState& s0 = hs[0]->s;
  const int d = s0.d, ard = s0.kern.ard_d;
  long long items = 0, qtot = 0;
  for (uint64_t i = 0; i < k; ++i) {
    ExactState& s = hs[i]->s;
    if (s.device != s0.device) return set_error(GPRX_INVALID_CONFIG, "grouped models must share a device");
    if (s.online) return set_error(GPRX_INVALID_CONFIG, "an online model does not take part in a grouped prediction");
    if (s.n > PG_NMAX || s.d > PG_DMAX)
      return set_error(GPRX_CAPACITY, "a grouped prediction takes models of at most 1024 points and 16 features");
    if (s.d != d || s.kern.ard_d != ard)
      return set_error(GPRX_INVALID_CONFIG, "grouped models must share d and the kernel's ARD width");
    if (qs[i] == 0 || qs[i] > (uint64_t)INT32_MAX) return set_error(GPRX_EMPTY_INPUT, "a request has no query points");
    if (!all_finite(xs[i], qs[i] * d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite query");
    items += (long long)((qs[i] + PG_Q - 1) / PG_Q);
    qtot += (long long)qs[i];
  }
  GPRX_CUDA_TRY(cudaSetDevice(s0.device));
  for (uint64_t i = 0; i < k; ++i) {
    ExactState& s = hs[i]->s;
    if (!s.factor_ok || !s.alpha_ok) {
      gprx_status st = s.factor_current();
      if (st != GPRX_OK) return st;
    }
    if (i > 0) GPRX_CUDA_TRY(cudaStreamSynchronize(s.stream));
  }
  // staging: requests, items, queries (one upload); outputs (one download)
  const size_t o_items = align256(sizeof(GroupReq) * k);
  const size_t o_q = o_items + align256(sizeof(int2) * items);
  const size_t up = o_q + align256(sizeof(double) * qtot * d);
  const size_t bytes = up + sizeof(double) * 2 * qtot;
  if (s0.group_dev.ensure(bytes) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "grouped-predict staging");
  GPRX_CUDA_TRY(s0.group_host.ensure(bytes));
  unsigned char* hb = s0.group_host.p;
  unsigned char* db = s0.group_dev.p;
  GroupReq* rq = reinterpret_cast<GroupReq*>(hb);
  int2* it = reinterpret_cast<int2*>(hb + o_items);
  double* xq = reinterpret_cast<double*>(hb + o_q);
  double* out_d = reinterpret_cast<double*>(db + up);
  long long qo = 0, ni = 0;
  for (uint64_t i = 0; i < k; ++i) {
    ExactState& s = hs[i]->s;
    const int q = (int)qs[i];
    GroupReq r;
    r.t = s.kern.tree;
    r.x = s.x.p;
    r.ldx = s.cap;
    r.n = s.n;
    r.q = q;
    r.L = s.A.p;
    r.ld = s.ld;
    r.linv = s.linv.p;
    r.alpha = s.alpha.p;
    r.xq = reinterpret_cast<const double*>(db + o_q) + qo * d;
    r.out = out_d + 2 * qo;
    r.noise = s.noise();
    r.kss = s.kern.diag_value();
    r.kind = kind;
    rq[i] = r;
    std::copy(xs[i], xs[i] + (size_t)q * d, xq + qo * d);
    for (int j0 = 0; j0 < q; j0 += PG_Q) it[ni++] = make_int2((int)i, j0);
    qo += q;
  }
  gprx_status st;
  if ((st = s0.reset_status()) != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpyAsync(db, hb, up, cudaMemcpyHostToDevice, s0.stream));
  const GroupReq* rq_d = reinterpret_cast<const GroupReq*>(db);
  const int2* it_d = reinterpret_cast<const int2*>(db + o_items);
  const size_t smem = pg_smem(d);
#define GPRX_PG(D)                                                                                         \
  GPRX_CUDA_TRY(cudaFuncSetAttribute(predict_group_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     (int)pg_smem(PG_DMAX)));                                              \
  GPRX_LAUNCH(predict_group_kernel<D>, (int)items, PG_THREADS, smem, s0.stream, rq_d, it_d, s0.status.p)
  switch (ard) {
    case 0: GPRX_PG(0); break;
    case 4: GPRX_PG(4); break;
    case 8: GPRX_PG(8); break;
    default: GPRX_PG(16); break;
  }
#undef GPRX_PG
  GPRX_CUDA_TRY(cudaGetLastError());
  double* outh = reinterpret_cast<double*>(hb + up);
  GPRX_CUDA_TRY(cudaMemcpyAsync(outh, out_d, sizeof(double) * 2 * qtot, cudaMemcpyDeviceToHost, s0.stream));
  DevStatus ds;
  if ((st = s0.read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, 0.0, s0.n, GPRX_STAGE_PREDICT);
  qo = 0;
  for (uint64_t i = 0; i < k; ++i) {
    const size_t q = qs[i];
    std::copy(outh + 2 * qo, outh + 2 * qo + q, means[i]);
    std::copy(outh + 2 * qo + q, outh + 2 * qo + 2 * q, vars[i]);
    qo += (long long)q;
  }
  return GPRX_OK;
}

}  // namespace gprx

extern "C" gprx_status gprx_exact_predict_group(gprx_exact* const* handles, uint64_t k, const double* const* xs,
                                                 const uint64_t* q, int32_t variance_kind, double* const* mean,
                                                 double* const* var) {
  return gprx::predict_group(handles, k, xs, q, variance_kind, mean, var);
}
