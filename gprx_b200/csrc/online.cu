// online.cu — OnlineGpr on the device: LLT → LDLT, bordered append, row /
// column delete, lazy α.
//
// Reference: FittedGpr::into_online / LdltStore::fill_ld_from_llt
// (gprx src/gpr/fitted.rs:757-765, src/gpr/factor_store.rs:157-179),
// OnlineGpr::insert_with + LdltStore::append_border (src/gpr/online.rs:794-900,
// factor_store.rs:210-237), OnlineGpr::delete + LdltStore::delete_index →
// faer ldlt::update::delete_rows_and_cols_clobber (online.rs:564-611,
// factor_store.rs:239-255, src/linalg/ldlt.rs:113-122), the stale α solve
// (src/linalg/ldlt.rs:146-204) and IdRegistry (src/points.rs:76-190).
//
// The row/column delete is restated as the rank-1 LDLT update of the
// trailing block by D_k l_k l_kᵀ (Gill, Golub, Murray & Saunders 1974, C1),
// blocked 32 columns at a time: one warp runs the 32-step scalar recurrence
// on the block's own rows, then every thread applies the 32 column updates to
// its rows below.

#include <algorithm>
#include <cmath>

#include "exact.cuh"

namespace gprx {

__global__ void llt_to_ldlt_kernel(double* A, long long ld, int n) {
  // column j: D_j = L_jj², L_ij ← L_ij / L_jj (i > j)
  int j = blockIdx.x;
  if (j >= n) return;
  double ljj = A[j + (long long)j * ld];
  for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[i + (long long)j * ld] /= ljj;
  __syncthreads();
  if (threadIdx.x == 0) A[j + (long long)j * ld] = ljj * ljj;
}

// Border of one appended point: w (in place in `w`) holds L⁻¹ k; writes
// v = D⁻¹ w into row n of A and δ = k_new − Σ w_i v_i onto the diagonal.
__global__ void ldlt_border_kernel(double* A, long long ld, int n, const double* w, double k_new, DevStatus* st) {
  __shared__ double red[32];
  if (dev_failed(st)) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double di = A[i + (long long)i * ld];
    double vi = w[i] / di;
    A[n + (long long)i * ld] = vi;
    acc = fma(vi * vi, di, acc);
  }
  double vtdv = block_sum(acc, red);
  if (threadIdx.x == 0) {
    double delta = k_new - vtdv;
    if (!(delta > 0.0) || !isfinite(delta)) dev_fail(st, GPRX_CHOLESKY_FAILED, n);
    else A[n + (long long)n * ld] = delta;
  }
}

// Rank-1 update L D Lᵀ + a·w wᵀ of the trailing block starting at row/col r0
// (size m), with w = L[r0.., idx] and a = D_idx.  Single CTA, 1024 threads.
constexpr int R1_THREADS = 256;
__global__ void __launch_bounds__(R1_THREADS) ldlt_rank1_kernel(double* A, long long ld, int r0, int m, int idx,
                                                                 DevStatus* st) {
  __shared__ double P[32], Bt[32];
  __shared__ double a_sh;
  if (dev_failed(st)) return;
  // w lives in column idx of A (rows r0..r0+m−1); it is updated in place
  // there (that column is dropped afterwards).
  double* w = A + (long long)idx * ld;
  if (threadIdx.x == 0) a_sh = A[idx + (long long)idx * ld];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int jb = 0; jb < m; jb += 32) {
    int nbk = min(32, m - jb);
    if (warp == 0) {
      // lane owns row r = r0 + jb + lane of the block
      int r = r0 + jb + lane;
      bool live = lane < nbk;
      double wr = live ? w[r] : 0.0;
      double Lr[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) Lr[c] = (live && c < lane) ? A[r + (long long)(r0 + jb + c) * ld] : 0.0;
      double a = a_sh;
      // D of the block's rows, read before any of them is rewritten
      double dmine = live ? A[r + (long long)r * ld] : 1.0;
      double dnew_mine = dmine;
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        if (c >= nbk) break;
        double p = __shfl_sync(0xffffffffu, wr, c);
        double dj = __shfl_sync(0xffffffffu, dmine, c);
        double dnew = fma(a * p, p, dj);
        double beta = p * a / dnew;
        a = dj * a / dnew;
        if (lane == c) {
          P[c] = p;
          Bt[c] = beta;
          dnew_mine = dnew;
        }
        if (live && lane > c) {
          wr = fma(-p, Lr[c], wr);
          Lr[c] = fma(beta, wr, Lr[c]);
        }
      }
      if (live) {
        w[r] = wr;
        A[r + (long long)r * ld] = dnew_mine;
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (c < lane) A[r + (long long)(r0 + jb + c) * ld] = Lr[c];
      }
      if (lane == 0) a_sh = a;
    }
    __syncthreads();
    for (int rr = jb + nbk + threadIdx.x; rr < m; rr += blockDim.x) {
      int r = r0 + rr;
      double wr = w[r];
      for (int c = 0; c < nbk; ++c) {
        double* l = A + r + (long long)(r0 + jb + c) * ld;
        wr = fma(-P[c], *l, wr);
        *l = fma(Bt[c], wr, *l);
      }
      w[r] = wr;
    }
    __syncthreads();
  }
}

// Out-of-place compaction of the lower triangle without row/column idx.
__global__ void drop_rowcol_kernel(const double* A, long long lda, int n, int idx, double* B, long long ldb) {
  long long total = (long long)(n - 1) * (n - 1);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % (n - 1)), j = (int)(e / (n - 1));
    if (i < j) continue;
    int si = i >= idx ? i + 1 : i, sj = j >= idx ? j + 1 : j;
    B[i + (long long)j * ldb] = A[si + (long long)sj * lda];
  }
}

__global__ void drop_row_kernel(const double* x, long long ldx, int n, int d, int idx, double* out, long long ldo) {
  long long total = (long long)(n - 1) * d;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % (n - 1)), f = (int)(e / (n - 1));
    int si = i >= idx ? i + 1 : i;
    out[i + (long long)f * ldo] = x[si + (long long)f * ldx];
  }
}

__global__ void div_by_diag_kernel(double* v, const double* A, long long ld, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] /= A[i + (long long)i * ld];
}

gprx_status ExactState::online_begin() {
  gprx_status st;
  if (online) return GPRX_OK;
  if (!factor_ok || !alpha_ok) {
    if ((st = factor_current()) != GPRX_OK) return st;
  }
  llt_to_ldlt_kernel<<<n, 256, 0, stream>>>(A.p, ld, n);
  count_launch();
  GPRX_CUDA_TRY(cudaGetLastError());
  online = true;
  factor_ok = false;
  linv_ok = false;
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  return GPRX_OK;
}

gprx_status ExactState::with_llt_view(const std::function<gprx_status()>& op) {
  if (!online) return op();
  // keep the LDLT: a failed operation leaves the online model as it was
  const size_t keep = (size_t)ld * n;
  if (ldlt_keep.ensure(std::max<size_t>(keep, 1)) != cudaSuccess || alpha_keep.ensure(std::max(n, 1)) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "device allocation of the online factor copy failed");
  GPRX_CUDA_TRY(cudaMemcpyAsync(ldlt_keep.p, A.p, sizeof(double) * keep, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(alpha_keep.p, alpha.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
  const bool alpha_was_ok = alpha_ok;
  const double jitter_was = jitter;
  std::vector<double> theta_was(num_params());
  get_params(theta_was.data());
  online = false;
  factor_ok = false;
  linv_ok = false;
  alpha_ok = false;
  gprx_status st = op();
  if (st == GPRX_OK && (!factor_ok || !alpha_ok)) st = factor_current();
  if (st == GPRX_OK) {
    llt_to_ldlt_kernel<<<n, 256, 0, stream>>>(A.p, ld, n);
    count_launch();
    GPRX_CUDA_TRY(cudaGetLastError());
  } else {
    gprx_error_info saved = last_error();
    write_params(theta_was.data());
    GPRX_CUDA_TRY(cudaMemcpyAsync(A.p, ldlt_keep.p, sizeof(double) * keep, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(alpha.p, alpha_keep.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    alpha_ok = alpha_was_ok;
    jitter = jitter_was;
    last_error() = saved;
  }
  online = true;
  factor_ok = false;
  linv_ok = false;
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  return st;
}

gprx_status ExactState::grow(int needed) {
  if (needed <= cap) return GPRX_OK;
  int new_cap = std::max(needed, std::max(cap, 1) * 2);
  long long new_ld = round_ld(new_cap);
  DevBuf<double> nA, nx, ny;
  if (nA.alloc((size_t)new_ld * new_cap) != cudaSuccess || nx.alloc((size_t)new_cap * d) != cudaSuccess ||
      ny.alloc(new_cap) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "online capacity growth");
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(nA.p, sizeof(double) * new_ld, A.p, sizeof(double) * ld, sizeof(double) * n, n,
                                  cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(nx.p, sizeof(double) * new_cap, x.p, sizeof(double) * cap, sizeof(double) * n, d,
                                  cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(ny.p, y.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  std::swap(A.p, nA.p);
  std::swap(A.n, nA.n);
  std::swap(x.p, nx.p);
  std::swap(x.n, nx.n);
  std::swap(y.p, ny.p);
  std::swap(y.n, ny.n);
  int nblk = ceil_div(new_cap, NB);
  if (linv.alloc((size_t)nblk * NB * NB) != cudaSuccess || alpha.alloc(new_cap) != cudaSuccess ||
      z.alloc(new_cap) != cudaSuccess || tmpv.alloc(new_cap) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "online capacity growth");
  Xinv.reset();
  qbuf.reset();
  cap = new_cap;
  ld = new_ld;
  linv_ok = false;
  alpha_ok = false;
  return GPRX_OK;
}

gprx_status ExactState::online_insert(const double* xnew, double ynew, uint64_t* id) {
  if (!online) return set_error(GPRX_INVALID_CONFIG, "call gprx_online_begin first");
  if (!xnew || !id) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (!all_finite(xnew, d) || !std::isfinite(ynew)) return set_error(GPRX_NONFINITE_INPUT, "non-finite point");
  gprx_status st;
  if ((st = grow(n + 1)) != GPRX_OK) return st;
  if (qx.ensure((size_t)d + 8) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "insert scratch");
  if ((st = reset_status()) != GPRX_OK) return st;
  if (!linv_ok) {
    GPRX_CUDA_TRY(tri_inv_blocks(A.p, ld, n, true, linv.p, status.p, stream));
    linv_ok = true;
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(qx.p, xnew, sizeof(double) * d, cudaMemcpyHostToDevice, stream));
  // k = K(X, x_new) into tmpv (n×1), then w = L⁻¹ k (unit lower)
  GPRX_CUDA_TRY(fill_cross(kern, x.p, cap, n, qx.p, 1, 1, tmpv.p, n, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower(A.p, ld, n, linv.p, tmpv.p, n, 1, status.p, stream));
  double k_new = kern.diag_value() + noise() + jitter;  // online.rs:855-862
  ldlt_border_kernel<<<1, 1024, 0, stream>>>(A.p, ld, n, tmpv.p, k_new, status.p);
  count_launch();
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, 0.0, n + 1, GPRX_STAGE_ONLINE_INSERT);
  // append x, y (the store keeps them in buffer order)
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(x.p + n, sizeof(double) * cap, xnew, sizeof(double), sizeof(double), d,
                                  cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(y.p + n, &ynew, sizeof(double), cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  y_host.push_back(ynew);
  n += 1;
  *id = next_id++;
  ids.push_back(*id);
  alpha_ok = false;
  // the appended row changes only the last diagonal block
  linv_ok = false;
  return GPRX_OK;
}

gprx_status ExactState::online_delete(uint64_t id) {
  if (!online) return set_error(GPRX_INVALID_CONFIG, "call gprx_online_begin first");
  if (n <= 1) return set_error(GPRX_INSUFFICIENT_DATA, "an online model keeps at least one point");
  auto it = std::lower_bound(ids.begin(), ids.end(), id);
  if (it == ids.end() || *it != id) return set_error(GPRX_INVALID_POINT_ID, "unknown point id");
  int idx = (int)(it - ids.begin());
  gprx_status st;
  if ((st = reset_status()) != GPRX_OK) return st;
  int m = n - idx - 1;
  if (m > 0) {
    ldlt_rank1_kernel<<<1, R1_THREADS, 0, stream>>>(A.p, ld, idx + 1, m, idx, status.p);
    count_launch();
  }
  DevBuf<double> nA, nx, ny;
  if (nA.alloc((size_t)ld * cap) != cudaSuccess || nx.alloc((size_t)cap * d) != cudaSuccess ||
      ny.alloc(cap) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "online delete scratch");
  long long tot = (long long)(n - 1) * (n - 1);
  int blocks = (int)std::max<long long>(1, std::min<long long>((tot + 255) / 256, 148LL * 16));
  drop_rowcol_kernel<<<blocks, 256, 0, stream>>>(A.p, ld, n, idx, nA.p, ld);
  drop_row_kernel<<<ceil_div((long long)(n - 1) * d, 256) + 1, 256, 0, stream>>>(x.p, cap, n, d, idx, nx.p, cap);
  drop_row_kernel<<<ceil_div(n, 256) + 1, 256, 0, stream>>>(y.p, cap, n, 1, idx, ny.p, cap);
  count_launch(3);
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, 0.0, n, GPRX_STAGE_ONLINE_DELETE);
  std::swap(A.p, nA.p);
  std::swap(A.n, nA.n);
  std::swap(x.p, nx.p);
  std::swap(x.n, nx.n);
  std::swap(y.p, ny.p);
  std::swap(y.n, ny.n);
  y_host.erase(y_host.begin() + idx);
  ids.erase(it);
  n -= 1;
  alpha_ok = false;
  linv_ok = false;
  return GPRX_OK;
}

gprx_status ExactState::online_alpha() {
  gprx_status st;
  if ((st = reset_status()) != GPRX_OK) return st;
  if (!linv_ok) {
    GPRX_CUDA_TRY(tri_inv_blocks(A.p, ld, n, true, linv.p, status.p, stream));
    linv_ok = true;
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(alpha.p, y.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(trsm_lower(A.p, ld, n, linv.p, alpha.p, n, 1, status.p, stream));
  div_by_diag_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(alpha.p, A.p, ld, n);
  count_launch();
  GPRX_CUDA_TRY(trsm_lower_t(A.p, ld, n, linv.p, alpha.p, n, 1, status.p, stream));
  DevStatus ds;
  if ((st = read_status(&ds)) != GPRX_OK) return st;
  if (ds.code != GPRX_OK) return status_to_error(ds, 0.0, n, GPRX_STAGE_ONLINE_INSERT);
  alpha_ok = true;
  return GPRX_OK;
}

}  // namespace gprx
