// emu_gemm.cuh — FP64 matrix products emulated on the int8 tensor cores
// (tcgen05.mma kind::i8, TMEM accumulators).
//
// Every row r of an operand is scaled by a power of two, 2^e_r, so that its
// largest entry lies in [32, 64), and the scaled row is written exactly as a
// sum of S int8 slices with signed digits of 7 bits:
//   a·2^e = s_0 + s_1·2^-7 + … + s_{S-1}·2^-7(S-1),  |s_p| ≤ 64.
// A product Σ_k A(i,k) B(j,k) is then Σ_t 2^-7t C_t with
//   C_t = Σ_{p+q=t} Σ_k s_p(A)(i,k) s_q(B)(j,k)   (t < S),
// each C_t an exact int32 sum (|s_p s_q| ≤ 2^12, K·t·2^12 < 2^31), so the
// only rounding is the FP64 combination of the S terms and the dropped terms
// with p + q ≥ S (relative size 2^(6-7S) of the row/column maxima).  S = 6
// carries 41 bits.  This is the slicing scheme of Ozaki et al. (error-free
// transformation of matrix products) with int8 slices.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace gprx {

constexpr int EMU_M = 128;   // tile rows (TMEM lanes)
constexpr int EMU_N = 64;    // tile columns per term
constexpr int EMU_KC = 64;   // bytes of K per pipeline stage
constexpr int EMU_STAGES = 3;
constexpr int EMU_THREADS = 128;
constexpr int EMU_MAX_S = 8;  // S terms × 64 columns ≤ 512 TMEM columns

// Row slices of an FP64 operand op(M) with R rows and K columns:
//   op(M)(r, k) = trans ? M[k + r·ld] : M[r + k·ld].
// S planes of Rpad × Kpad int8 digits (zero padding), stored pre-tiled in
// 8 KB blocks of 128 rows × 64 bytes of K in the UMMA core-matrix order (see
// emu_gemm.cu); exps[r] the row's power-of-two exponent.
struct EmuOperand {
  int8_t* slices = nullptr;
  int* exps = nullptr;
  unsigned long long* rmax = nullptr;  // Rpad words of scratch (row maxima)
  int R = 0, K = 0, Rpad = 0, Kpad = 0, S = 0;
};

inline int emu_pad_rows(int R) { return (R + EMU_M - 1) / EMU_M * EMU_M; }
inline int emu_pad_k(int K) { return (K + EMU_KC - 1) / EMU_KC * EMU_KC; }
inline size_t emu_slice_bytes(int R, int K, int S) {
  return (size_t)S * emu_pad_rows(R) * emu_pad_k(K);
}

// Fills op.slices / op.exps from M (op.R, op.K, op.S, op.Rpad, op.Kpad set).
cudaError_t emu_slice(const double* M, long long ld, bool trans, const EmuOperand& op, cudaStream_t s);

// C(i, j) = beta·C + alpha · Σ_{k ∈ [kb, K)} A(i,k) B(j,k) for i < A.R, j < B.R.
// lower: only i + row0 ≥ j + col0 is written.  kmode (triangular operands):
// 0 full K; 1 k from the tile's first row; 2 k from the tile's first column;
// 3 k up to the tile's last row; 4 k up to the tile's last column.
// err: device int set to 1 when a bounded wait gave up (never expected).
cudaError_t emu_gemm(const EmuOperand& A, const EmuOperand& B, double* C, long long ldc, double alpha, double beta,
                     bool lower, long long row0, long long col0, int kmode, int* err, cudaStream_t s);

// Split K: part z (z < emu_splitk_parts(Kpad, kz)) of the full product,
// Σ over K chunks [z·kz, (z+1)·kz) of 64 bytes, is written (alpha 1, beta 0)
// to C + z·zstride; kz·64·S·2^12 < 2^31 keeps each part's int32 sums exact.
inline int emu_splitk_parts(int Kpad, int kz) { return (Kpad / EMU_KC + kz - 1) / kz; }
cudaError_t emu_gemm_splitk(const EmuOperand& A, const EmuOperand& B, double* C, long long ldc, long long zstride,
                            int kz, bool lower, int* err, cudaStream_t s);

size_t emu_gemm_smem(int S);

// Device scratch for the products of one handle: slice planes and exponents
// of two operands sized for n×n, and the bounded-wait error flag.
struct EmuWork {
  int8_t* sa = nullptr;
  int8_t* sb = nullptr;
  int* ea = nullptr;
  int* eb = nullptr;
  unsigned long long* ma = nullptr;
  unsigned long long* mb = nullptr;
  int* err = nullptr;
  int S = 6;
  EmuOperand op_a(int R, int K) const {
    EmuOperand o;
    o.slices = sa; o.exps = ea; o.rmax = ma; o.R = R; o.K = K; o.Rpad = emu_pad_rows(R); o.Kpad = emu_pad_k(K); o.S = S;
    return o;
  }
  EmuOperand op_b(int R, int K) const {
    EmuOperand o;
    o.slices = sb; o.exps = eb; o.rmax = mb; o.R = R; o.K = K; o.Rpad = emu_pad_rows(R); o.Kpad = emu_pad_k(K); o.S = S;
    return o;
  }
};

}  // namespace gprx
