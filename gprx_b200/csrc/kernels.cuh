// kernels.cuh — kernel-matrix fills and the NLML gradient contraction.
#pragma once

#include <vector>

#include "common.cuh"

namespace gprx {

// Host-side kernel description: the prefix node list, θ, and the device tree
// in sum-of-products form.
struct HostKernel {
  std::vector<gprx_kernel_node> nodes;
  std::vector<double> theta;  // log params, depth-first
  int n_params = 0;
  int d = 0;
  KTree tree{};
  int ard_d = 0;              // template width for the ARD leaf (0, 4, 8, 16, 32)
  // gradient slot → θ index (−1: unused)
  std::vector<int> slot_param;

  // Parses nodes, checks θ count and dimension; builds the device tree.
  gprx_status init(const gprx_kernel_node* nodes, int n_nodes, const double* theta, int n_theta, int d,
                   std::string* why);
  // Writes θ (log space) and refreshes the derived constants.
  gprx_status set_theta(const double* theta);
  double diag_value() const { return tree.diag_value; }
};

constexpr int GRAD_SLOTS_LEAF = KT_MAX_LEAVES * KT_ACC_PER_LEAF;  // 16
inline int grad_slots(int ard_d) { return GRAD_SLOTS_LEAF + (ard_d > 0 ? ard_d : 1) + 1; }  // + noise slot

// K(X, X) lower triangle (+ diag_add on the diagonal) into K (n×n, ld); X is
// n×d with leading dimension ldx.
cudaError_t fill_lower(const HostKernel& k, const double* x, long long ldx, int n, double* K, long long ld,
                       double diag_add, DevStatus* st, cudaStream_t s);
// K(X1, X2): n1×n2 into out (ld ≥ n1).  X1 is n1×d, X2 is n2×d (column-major,
// leading dimensions ldx1 / ldx2).
cudaError_t fill_cross(const HostKernel& k, const double* x1, long long ldx1, int n1, const double* x2,
                       long long ldx2, int n2, double* out, long long ld, DevStatus* st, cudaStream_t s);

// Partial sums of Σ_{i≥j} c_ij · W_ij · ∂K_ij/∂θ (c = 1 on the diagonal, 2 off
// it).  With alpha: W_ij = α_i α_j − M_ij (M = K⁻¹ lower in ld) and the last
// slot collects Σ W_ii; with alpha == nullptr: W_ij = M_ij.  x is n×d with
// leading dimension ldx.  Writes `blocks × grad_slots(ard_d)` partials.
cudaError_t grad_contract(const HostKernel& k, const double* x, long long ldx, int n, const double* kinv, long long ld,
                          const double* alpha, double* partials, int* blocks_out, DevStatus* st, cudaStream_t s);
// Partial sums of Σ_{i,c} W_ic ∂k(z_i, x_c)/∂θ over the m×n rectangle.
cudaError_t cross_contract(const HostKernel& k, const double* z, long long ldz, int m, const double* x, long long ldx,
                           int n, const double* W, long long ldw, double* partials, int* blocks_out, DevStatus* st,
                           cudaStream_t s);
// grad[p] = scale · (slot sums mapped to θ), grad[n_params] = noise_coef · Σ W_ii.
cudaError_t grad_finalize(const HostKernel& k, const double* partials, int blocks, const int* slot_param_dev,
                          double scale, double noise_coef, double* grad, DevStatus* st, cudaStream_t s);

// Maximum partial-block count of grad_contract (sizes the partials buffer).
int grad_max_blocks();

}  // namespace gprx
