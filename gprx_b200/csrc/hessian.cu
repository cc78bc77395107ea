// hessian.cu — the pieces of the exact NLML's Hessian that need the kernel's
// second derivatives (ExactFit::hessian_into, src/gpr/exact_fit.rs:443-637):
//
//   H_ij = −½ ⟨W, ∂²A/∂θ_i∂θ_j⟩ − ½ ⟨S_i, S_j⟩_F + v_iᵀ v_j,
//   W = ααᵀ − A⁻¹,  S_i = L⁻¹ A_i L⁻ᵀ,  v_i = L⁻¹ A_i α,  A_i = ∂A/∂θ_i.
//
// This file computes the first term's contraction (every entry in one launch
// up to HESS_FUSE_K kernel parameters, else one launch per row i with all
// j ≥ i accumulated in registers), fills A_i as a full symmetric matrix for
// the products that form S_i, and takes the Frobenius products ⟨S_i, S_j⟩ of
// the lower-stored S_i in one pass.  Leaf second derivatives, in the log
// parameters (u = r²/ℓ², u_f = Δ_f²/ℓ_f², φ = π r / p, s = sin φ, c = cos φ):
//   constant  k = c                     ∂ = c,  ∂² = c
//   rbf       k = e^{−u/2}              ∂ = k u,  ∂² = k (u² − 2u)
//   rbf_ard   k = e^{−Σu_f/2}           ∂_f = k u_f,  ∂_fg = k u_f u_g − 2 δ_fg k u_f
//   periodic  k = e^{−2 s²/ℓ²}          a = 4 s²/ℓ², b = 4 s c φ/ℓ²:
//             ∂_ℓ = k a, ∂_p = k b, ∂_ℓℓ = k (a² − 2a), ∂_ℓp = k b (a − 2),
//             ∂_pp = k (b² + 4 (φ² (s² − c²) − s c φ)/ℓ²)
// and a product of leaves by the product rule over the sum-of-products tree.
#include "hessian.cuh"

namespace gprx {

constexpr int HT = 64;  // tile of points
constexpr int HESS_THREADS = 256;

__device__ __forceinline__ void hess_lower_tile(long long idx, int& ti, int& tj) {
  double r = floor((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
  long long t = (long long)r;
  while ((t + 1) * (t + 2) / 2 <= idx) ++t;
  while (t * (t + 1) / 2 > idx) --t;
  ti = (int)t;
  tj = (int)(idx - t * (t + 1) / 2);
}

// Per-pair quantities of one leaf.
struct PairGeom {
  double r2;
  double dx[GPRX_MAX_DIM];
};

template <int ARD_D>
__device__ __forceinline__ double leaf_d1(const KTree& t, int l, int a, const PairGeom& g, double v) {
  const KLeaf& lf = t.leaf[l];
  switch (lf.kind) {
    case GPRX_LEAF_CONSTANT:
      return lf.c0;
    case GPRX_LEAF_RBF:
      return v * (2.0 * lf.c0 * g.r2);
    case GPRX_LEAF_RBF_ARD:
      return v * (g.dx[a] * g.dx[a] * t.inv_ell2[a]);
    case GPRX_LEAF_PERIODIC: {
      const double phi = lf.c0 * sqrt(fmax(g.r2, 0.0));
      double s, c;
      sincos(phi, &s, &c);
      return a == 0 ? v * 4.0 * s * s * lf.c1 : v * 4.0 * s * c * phi * lf.c1;
    }
  }
  return 0.0;
}

template <int ARD_D>
__device__ __forceinline__ double leaf_d2(const KTree& t, int l, int a, int b, const PairGeom& g, double v) {
  const KLeaf& lf = t.leaf[l];
  switch (lf.kind) {
    case GPRX_LEAF_CONSTANT:
      return lf.c0;
    case GPRX_LEAF_RBF: {
      const double u = 2.0 * lf.c0 * g.r2;
      return v * (u * u - 2.0 * u);
    }
    case GPRX_LEAF_RBF_ARD: {
      const double ua = g.dx[a] * g.dx[a] * t.inv_ell2[a];
      const double ub = g.dx[b] * g.dx[b] * t.inv_ell2[b];
      return v * ua * ub - (a == b ? 2.0 * v * ua : 0.0);
    }
    case GPRX_LEAF_PERIODIC: {
      const double phi = lf.c0 * sqrt(fmax(g.r2, 0.0));
      double s, c;
      sincos(phi, &s, &c);
      const double A = 4.0 * s * s * lf.c1, B = 4.0 * s * c * phi * lf.c1;
      if (a == 0 && b == 0) return v * (A * A - 2.0 * A);
      if (a == 1 && b == 1) return v * (B * B + 4.0 * lf.c1 * (phi * phi * (s * s - c * c) - s * c * phi));
      return v * B * (A - 2.0);
    }
  }
  return 0.0;
}

// Pair geometry and leaf values for points a, b (tile-local rows ra / rb).
template <int ARD_D>
__device__ __forceinline__ void pair_setup(const KTree& t, const double* xa, const double* xb, PairGeom& g,
                                           double (&v)[KT_MAX_LEAVES]) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  double dxl[1][AD];
  double r2 = 0.0;
  for (int f = 0; f < t.d; ++f) {
    const double df = xa[f * HT] - xb[f * HT];
    r2 = fma(df, df, r2);
    g.dx[f] = df;
#pragma unroll
    for (int q = 0; q < AD; ++q)
      if (q == f) dxl[0][q] = df;
  }
  g.r2 = r2;
  const double r[1] = {r2};
  double vw[KT_MAX_LEAVES][1];
  kt_leaf_values_w<ARD_D, 1>(t, dxl, r, vw);
#pragma unroll
  for (int l = 0; l < KT_MAX_LEAVES; ++l) v[l] = vw[l][0];
}

// Σ_{a ≥ b} c_ab W_ab ∂²K_ab/∂θ_i∂θ_j for j = i .. n_par − 1 (c = 1 on the
// diagonal, 2 off it), W = ααᵀ − M with M = A⁻¹ (lower, ld).  One partial row
// of HESS_MAX_PARAMS per block.
template <int ARD_D>
__global__ void __launch_bounds__(HESS_THREADS) hess_second_kernel(KTree t, HessMap hm, int i, const double* x,
                                                                   long long ldx, int n, const double* kinv,
                                                                   long long ld, const double* alpha,
                                                                   double* partials) {
  __shared__ double xi[GPRX_MAX_DIM * HT];
  __shared__ double xj[GPRX_MAX_DIM * HT];
  __shared__ double red[HESS_THREADS / 32][HESS_MAX_PARAMS];
  const int li = hm.leaf_of[i], ai = hm.local_of[i];
  const int nj = hm.n_par - i;
  double acc[HESS_MAX_PARAMS];
#pragma unroll
  for (int q = 0; q < HESS_MAX_PARAMS; ++q) acc[q] = 0.0;
  const int nt = (n + HT - 1) / HT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    hess_lower_tile(idx, ti, tj);
    const int i0 = ti * HT, j0 = tj * HT;
    __syncthreads();
    for (int e = threadIdx.x; e < t.d * HT; e += blockDim.x) {
      const int r = e % HT, f = e / HT;
      xi[f * HT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * HT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % HT;
    const int pa = i0 + r;
    for (int c = threadIdx.x / HT; c < HT; c += HESS_THREADS / HT) {
      const int pb = j0 + c;
      if (pa >= n || pb >= n || pa < pb) continue;
      const double w = fma(alpha[pa], alpha[pb], -kinv[pa + (long long)pb * ld]);
      const double cw = pa == pb ? w : 2.0 * w;
      PairGeom g;
      double v[KT_MAX_LEAVES];
      pair_setup<ARD_D>(t, xi + r, xj + c, g, v);
      const double d1i = leaf_d1<ARD_D>(t, li, ai, g, v[li]);
      for (int q = 0; q < nj; ++q) {
        const int j = i + q, lj = hm.leaf_of[j], aj = hm.local_of[j];
        const double d1j = lj == li ? 0.0 : leaf_d1<ARD_D>(t, lj, aj, g, v[lj]);
        const double d2 = lj == li ? leaf_d2<ARD_D>(t, li, ai, aj, g, v[li]) : 0.0;
        double tot = 0.0;
        for (int tt = 0; tt < t.n_terms; ++tt) {
          const unsigned mask = t.term_mask[tt];
          if (!((mask >> li) & 1u) || !((mask >> lj) & 1u)) continue;
          double po = 1.0;
          for (int o = 0; o < t.n_leaves; ++o)
            if (((mask >> o) & 1u) && o != li && o != lj) po *= v[o];
          tot += (lj == li ? d2 : d1i * d1j) * po;
        }
#pragma unroll
        for (int s = 0; s < HESS_MAX_PARAMS; ++s)
          if (s == q) acc[s] = fma(cw, tot, acc[s]);
      }
    }
  }
  // block partials in a fixed order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
#pragma unroll
  for (int s = 0; s < HESS_MAX_PARAMS; ++s) {
    const double vs = warp_sum(acc[s]);
    if (lane == 0) red[warp][s] = vs;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < HESS_MAX_PARAMS; s += blockDim.x) {
    double tot = 0.0;
    for (int wq = 0; wq < HESS_THREADS / 32; ++wq) tot += red[wq][s];
    partials[(long long)blockIdx.x * HESS_MAX_PARAMS + s] = tot;
  }
}

// All rows at once.  With T_t the value of term t at the pair and, for
// parameter a of leaf l_a, ∂v_l/∂θ_a = v_l f_a (f = u for rbf, u_f for
// rbf_ard, 1 for constant, a / b for periodic), the pair's second derivative
// is Σ_{t ∋ l_a, l_b} T_t (f_a f_b + [l_a = l_b] ∂f_b/∂θ_a), with ∂f_b/∂θ_a =
// −2 f_b for the length-scale-type parameters, 0 across ARD dimensions and for
// a constant, and 4 (φ² (s² − c²) − s c φ)/ℓ² for a periodic leaf's period
// twice.
template <int ARD_D>
__global__ void __launch_bounds__(HESS_THREADS) hess_all_kernel(KTree t, HessMap hm, const double* x, long long ldx,
                                                                int n, const double* kinv, long long ld,
                                                                const double* alpha, double* partials) {
  constexpr int K = HESS_FUSE_K, NS = HESS_FUSE_SLOTS;
  __shared__ double xi[GPRX_MAX_DIM * HT];
  __shared__ double xj[GPRX_MAX_DIM * HT];
  __shared__ double red[HESS_THREADS / 32][NS];
  const int np = hm.n_par;
  double acc[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) acc[q] = 0.0;
  const int nt = (n + HT - 1) / HT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    hess_lower_tile(idx, ti, tj);
    const int i0 = ti * HT, j0 = tj * HT;
    __syncthreads();
    for (int e = threadIdx.x; e < t.d * HT; e += blockDim.x) {
      const int r = e % HT, f = e / HT;
      xi[f * HT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * HT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % HT;
    const int pa = i0 + r;
    for (int c = threadIdx.x / HT; c < HT; c += HESS_THREADS / HT) {
      const int pb = j0 + c;
      if (pa >= n || pb >= n || pa < pb) continue;
      const double w = fma(alpha[pa], alpha[pb], -kinv[pa + (long long)pb * ld]);
      const double cw = pa == pb ? w : 2.0 * w;
      PairGeom g;
      double v[KT_MAX_LEAVES];
      pair_setup<ARD_D>(t, xi + r, xj + c, g, v);
      // term values
      double tv[KT_MAX_TERMS];
#pragma unroll
      for (int tt = 0; tt < KT_MAX_TERMS; ++tt) {
        double pr = tt < t.n_terms ? 1.0 : 0.0;
#pragma unroll
        for (int l = 0; l < KT_MAX_LEAVES; ++l)
          if (tt < t.n_terms && l < t.n_leaves && ((t.term_mask[tt] >> l) & 1u)) pr *= v[l];
        tv[tt] = pr;
      }
      // per-parameter factors f_a and the periodic period's own term e_a
      double fa[K], ea[K];
#pragma unroll
      for (int a = 0; a < K; ++a) {
        fa[a] = 0.0;
        ea[a] = 0.0;
        if (a < np) {
          const KLeaf& lf = t.leaf[hm.leaf_of[a]];
          const int loc = hm.local_of[a];
          switch (lf.kind) {
            case GPRX_LEAF_CONSTANT:
              fa[a] = 1.0;
              break;
            case GPRX_LEAF_RBF:
              fa[a] = 2.0 * lf.c0 * g.r2;
              break;
            case GPRX_LEAF_RBF_ARD:
              fa[a] = g.dx[loc] * g.dx[loc] * t.inv_ell2[loc];
              break;
            case GPRX_LEAF_PERIODIC: {
              const double phi = lf.c0 * sqrt(fmax(g.r2, 0.0));
              double sn, cs;
              sincos(phi, &sn, &cs);
              fa[a] = loc == 0 ? 4.0 * sn * sn * lf.c1 : 4.0 * sn * cs * phi * lf.c1;
              ea[a] = 4.0 * lf.c1 * (phi * phi * (sn * sn - cs * cs) - sn * cs * phi);
              break;
            }
          }
        }
      }
      int q = 0;
#pragma unroll
      for (int a = 0; a < K; ++a) {
#pragma unroll
        for (int b = a; b < K; ++b, ++q) {
          if (b >= np) continue;
          const unsigned m = hm.terms_of[a] & hm.terms_of[b];
          double sum = 0.0;
#pragma unroll
          for (int tt = 0; tt < KT_MAX_TERMS; ++tt)
            if ((m >> tt) & 1u) sum += tv[tt];
          double dd = fa[a] * fa[b];
          if (hm.leaf_of[a] == hm.leaf_of[b]) {
            const int kind = t.leaf[hm.leaf_of[a]].kind;
            if (kind == GPRX_LEAF_RBF || kind == GPRX_LEAF_RBF_ARD) {
              if (a == b) dd -= 2.0 * fa[a];
            } else if (kind == GPRX_LEAF_PERIODIC) {
              dd += (hm.local_of[a] == 1 && hm.local_of[b] == 1) ? ea[b] : -2.0 * fa[b];
            }
          }
          acc[q] = fma(cw, sum * dd, acc[q]);
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const double vs = warp_sum(acc[q]);
    if (lane == 0) red[warp][q] = vs;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NS; q += blockDim.x) {
    double tot = 0.0;
    for (int wq = 0; wq < HESS_THREADS / 32; ++wq) tot += red[wq][q];
    partials[(long long)blockIdx.x * NS + q] = tot;
  }
}

// ⟨M_i, M_j⟩ for symmetric matrices held in their lower triangles: 64×64
// lower tiles, each thread one row of a column pass (coalesced), every
// matrix's element in registers and all products accumulated at once.
__global__ void __launch_bounds__(256) sym_products_kernel(HessMats mats, int np, long long ld, int n,
                                                           double* partials) {
  constexpr int P = HESS_FUSE_P, NS = HESS_TRACE_SLOTS;
  __shared__ double red[8 * NS];
  double acc[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) acc[q] = 0.0;
  const int nt = (n + HT - 1) / HT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  const int r = threadIdx.x % HT;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    hess_lower_tile(idx, ti, tj);
    const int a = ti * HT + r;
    for (int c = threadIdx.x / HT; c < HT; c += 256 / HT) {
      const int b = tj * HT + c;
      if (a >= n || b >= n || a < b) continue;
      const double w = a == b ? 1.0 : 2.0;
      double xv[P];
#pragma unroll
      for (int i = 0; i < P; ++i) xv[i] = i < np ? mats.m[i][a + (long long)b * ld] : 0.0;
      int q = 0;
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const double wx = w * xv[i];
#pragma unroll
        for (int j = 0; j <= i; ++j, ++q) acc[q] = fma(wx, xv[j], acc[q]);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const double vs = warp_sum(acc[q]);
    if (lane == 0) red[warp * NS + q] = vs;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NS; q += blockDim.x) {
    double tot = 0.0;
    for (int wq = 0; wq < 8; ++wq) tot += red[wq * NS + q];
    partials[(long long)blockIdx.x * NS + q] = tot;
  }
}

// out (full n×n, ld) = ∂K/∂θ_i
template <int ARD_D>
__global__ void __launch_bounds__(HESS_THREADS) fill_deriv_kernel(KTree t, HessMap hm, int i, const double* x,
                                                                  long long ldx, int n, double* out, long long ld) {
  __shared__ double xi[GPRX_MAX_DIM * HT];
  __shared__ double xj[GPRX_MAX_DIM * HT];
  const int li = hm.leaf_of[i], ai = hm.local_of[i];
  const int nt = (n + HT - 1) / HT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    hess_lower_tile(idx, ti, tj);
    const int i0 = ti * HT, j0 = tj * HT;
    __syncthreads();
    for (int e = threadIdx.x; e < t.d * HT; e += blockDim.x) {
      const int r = e % HT, f = e / HT;
      xi[f * HT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * HT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % HT;
    const int pa = i0 + r;
    for (int c = threadIdx.x / HT; c < HT; c += HESS_THREADS / HT) {
      const int pb = j0 + c;
      if (pa >= n || pb >= n || pa < pb) continue;
      PairGeom g;
      double v[KT_MAX_LEAVES];
      pair_setup<ARD_D>(t, xi + r, xj + c, g, v);
      const double d1 = leaf_d1<ARD_D>(t, li, ai, g, v[li]);
      double tot = 0.0;
      for (int tt = 0; tt < t.n_terms; ++tt) {
        const unsigned mask = t.term_mask[tt];
        if (!((mask >> li) & 1u)) continue;
        double po = 1.0;
        for (int o = 0; o < t.n_leaves; ++o)
          if (((mask >> o) & 1u) && o != li) po *= v[o];
        tot += d1 * po;
      }
      out[pa + (long long)pb * ld] = tot;
      out[pb + (long long)pa * ld] = tot;
    }
  }
}

// out[q] = Σ_b partials[b·stride + q] for q < nq (fixed order).
__global__ void reduce_slots_kernel(const double* partials, int blocks, int stride, int nq, double* out) {
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < blocks; ++b) s += partials[(long long)b * stride + q];
    out[q] = s;
  }
}

// out = Σ_i M(i, i)
__global__ void trace_kernel(const double* M, long long ld, int n, double* out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += M[i + (long long)i * ld];
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) *out = s;
}

static int hess_grid(long long ntiles) {
  return (int)std::max<long long>(1, std::min<long long>(ntiles, HESS_MAX_BLOCKS));
}

cudaError_t hess_second(const HostKernel& k, const HessMap& hm, int i, const double* x, long long ldx, int n,
                        const double* kinv, long long ld, const double* alpha, double* partials, int* blocks_out,
                        cudaStream_t s) {
  const int nt = (n + HT - 1) / HT;
  const int grid = hess_grid((long long)nt * (nt + 1) / 2);
  *blocks_out = grid;
#define GPRX_HS(D) \
  GPRX_LAUNCH(hess_second_kernel<D>, grid, HESS_THREADS, 0, s, k.tree, hm, i, x, ldx, n, kinv, ld, alpha, partials)
  switch (k.ard_d) {
    case 0: GPRX_HS(0); break;
    case 4: GPRX_HS(4); break;
    case 8: GPRX_HS(8); break;
    case 16: GPRX_HS(16); break;
    default: GPRX_HS(32); break;
  }
#undef GPRX_HS
  return cudaGetLastError();
}

cudaError_t hess_second_all(const HostKernel& k, const HessMap& hm, const double* x, long long ldx, int n,
                            const double* kinv, long long ld, const double* alpha, double* partials, int* blocks_out,
                            cudaStream_t s) {
  if (hm.n_par > HESS_FUSE_K) return cudaErrorInvalidValue;
  const int nt = (n + HT - 1) / HT;
  const int grid = hess_grid((long long)nt * (nt + 1) / 2);
  *blocks_out = grid;
#define GPRX_HA(D) \
  GPRX_LAUNCH(hess_all_kernel<D>, grid, HESS_THREADS, 0, s, k.tree, hm, x, ldx, n, kinv, ld, alpha, partials)
  switch (k.ard_d) {
    case 0: GPRX_HA(0); break;
    case 4: GPRX_HA(4); break;
    case 8: GPRX_HA(8); break;
    case 16: GPRX_HA(16); break;
    default: GPRX_HA(32); break;
  }
#undef GPRX_HA
  return cudaGetLastError();
}

cudaError_t sym_products(const HessMats& mats, int np, long long ld, int n, double* partials, int* blocks_out,
                         cudaStream_t s) {
  if (np > HESS_FUSE_P) return cudaErrorInvalidValue;
  const int nt = (n + HT - 1) / HT;
  const int grid = hess_grid((long long)nt * (nt + 1) / 2);
  *blocks_out = grid;
  GPRX_LAUNCH(sym_products_kernel, grid, 256, 0, s, mats, np, ld, n, partials);
  return cudaGetLastError();
}

cudaError_t fill_deriv(const HostKernel& k, const HessMap& hm, int i, const double* x, long long ldx, int n,
                       double* out, long long ld, cudaStream_t s) {
  const int nt = (n + HT - 1) / HT;
  const int grid = hess_grid((long long)nt * (nt + 1) / 2);
#define GPRX_FD(D) GPRX_LAUNCH(fill_deriv_kernel<D>, grid, HESS_THREADS, 0, s, k.tree, hm, i, x, ldx, n, out, ld)
  switch (k.ard_d) {
    case 0: GPRX_FD(0); break;
    case 4: GPRX_FD(4); break;
    case 8: GPRX_FD(8); break;
    case 16: GPRX_FD(16); break;
    default: GPRX_FD(32); break;
  }
#undef GPRX_FD
  return cudaGetLastError();
}

cudaError_t reduce_slots(const double* partials, int blocks, int stride, int nq, double* out, cudaStream_t s) {
  GPRX_LAUNCH(reduce_slots_kernel, 1, 64, 0, s, partials, blocks, stride, nq, out);
  return cudaGetLastError();
}

cudaError_t trace_dev(const double* M, long long ld, int n, double* out, cudaStream_t s) {
  GPRX_LAUNCH(trace_kernel, 1, 1024, 0, s, M, ld, n, out);
  return cudaGetLastError();
}

}  // namespace gprx
