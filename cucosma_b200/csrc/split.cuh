// split.cuh -- launchers of the operand pre-passes (BF16 split, Ozaki slices).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cucosma {

// FP32 rows x cols -> nterms BF16 planes.  transpose = false: planes are
// [nterms][rows][kpad] (A operand, cols = K).  transpose = true: the input is
// K x N (rows = K, cols = N) and planes are [nterms][N][kpad] (B operand).
//
// xform (backward pass): the value split is not A[i] but
//   kXformScale:        scale * A[i]
//   kXformSigmoidGrad:  scale * A[i] * Y[i] * (1 - Y[i])   (A = dY, Y = sigmoid output)
//   kXformReluGrad:     Y[i] > 0 ? scale * A[i] : 0        (Y = ReLU output)
// with Y read at the same (row, column) as A (row stride ldy).
enum SplitXform : int { kXformNone = 0, kXformScale = 1, kXformSigmoidGrad = 2, kXformReluGrad = 3 };
cudaError_t launch_split_bf16(const float* A, int64_t lda, int rows, int cols, int64_t kpad, int nterms, void* out,
                              bool transpose, int sms, cudaStream_t st, int xform = kXformNone,
                              const float* Y = nullptr, int64_t ldy = 0, float scale = 1.0f);

// Statistics of the adaptive Ozaki path (slice count or native FP64 chosen
// on the device from the operands), kept in the workspace.  The magnitude
// sum of a row of A is sum_k floor(|a_ik| 2^(30 - ea_i)) (a 2^-30 fixed-point
// form of ||a_i||_1 / 2^ea_i, below 2^31 K); of a column of B likewise.
struct OzakiStats {
  unsigned long long min_row;  // smallest sum over the nonzero rows of A (all ones: none)
  unsigned long long min_col;  // smallest sum over the nonzero columns of B
  unsigned int done_blocks;    // blocks of the decision kernel that have finished
  int choice;                  // slices used (8 or 9), 0 = native FP64, -1 = not decided
  unsigned long long pad[5];
};
static_assert(sizeof(OzakiStats) == 64, "stats block");

// Path choice of the adaptive Ozaki call.  Slicing row i of A at its
// exponent ea_i with s slices leaves each entry an absolute error below
// 2^(ea_i + 1 - 7 s), so |err_ij| <= 2^(1 - 7 s) (2^ea_i ||b_j||_1 +
// 2^eb_j ||a_i||_1).  With P_i = K 2^ea_i / ||a_i||_1 and Q_j likewise, and
// sum_k |a_ik||b_kj| ~ ||a_i||_1 ||b_j||_1 / K for entries of unrelated
// magnitudes, that is 2^(1 - 7 s) (P_i + Q_j) relative to sum_k |a_ik||b_kj|,
// the scale native FP64's own rounding error is measured against.  The
// smallest s in {8, 9} with 2^(1 - 7 s) (max P + max Q) <= 2^-52 is chosen;
// when neither reaches it the call runs native FP64.  (Uniform entries give
// P, Q ~ 2: s = 8.  Exponents spread by sign * exp(N(0, 8^2)) give P, Q ~ K:
// native.)  An operand pair whose large entries of A meet only small entries
// of B along K defeats the estimate; such callers should ask for native FP64.
__host__ __device__ inline int ozaki_choice(unsigned long long min_row, unsigned long long min_col, int64_t k) {
  if (min_row == ~0ull || min_col == ~0ull) return 8;  // A or B is zero: every product is exactly zero
  const double P = (double)k * 1073741824.0 / (double)min_row;
  const double Q = (double)k * 1073741824.0 / (double)min_col;
  const double need = 53.0 + log2(P + Q);
  for (int s = 8; s <= 9; ++s)
    if (7.0 * s >= need) return s;
  return 0;
}
constexpr int kOzakiLayoutAdaptive = 9;  // slices produced when the count is chosen on the device
// Rows of A longer than this (in padded columns) are prepared in chunks of
// this many columns by two kernels (exponents, then slices); shorter rows by
// one kernel that holds the row in registers.
constexpr int kOzakiRowChunk = 8192;

// B (k x n) -> per-column exponents eb (|b_kn| < 2^eb_n, 0 for zero columns)
// and s INT8 slices of the columns, stacked: byte (n, k, p) at
// ((k / 32) * s + p) * n * 32 + n * 32 + k % 32.  With colsum (n entries)
// also the columns' magnitude sums, and stats->min_col is reset.
cudaError_t launch_ozaki_prep_b(int s, const double* B, int64_t ldb, int k, int n, int64_t kpad, int32_t* eb,
                                int8_t* sb, unsigned long long* colsum, OzakiStats* stats, int sms, cudaStream_t st);

// A (m x k) -> row exponents ea and s INT8 slices of the rows, packed (four
// slices' 32-byte k-blocks per 128-byte row): byte (r, k, p) at
// r * kpad * s + (k / 32) * 32 * s + p * 32 + k % 32; kpad a multiple of 32.
// With stats, also the rows' magnitude sums into rowsum (m entries; the
// decision fields of stats are reset first).
cudaError_t launch_ozaki_prep_a(int s, const double* A, int64_t lda, int m, int k, int64_t kpad, int32_t* ea,
                                int8_t* sa, unsigned long long* rowsum, OzakiStats* stats, int sms, cudaStream_t st);

// After both preparations: stats->min_row / min_col from rowsum and colsum,
// then stats->choice.
cudaError_t launch_ozaki_decide(const unsigned long long* rowsum, int m, const unsigned long long* colsum, int n,
                                int64_t k, OzakiStats* stats, int sms, cudaStream_t st);

}  // namespace cucosma
