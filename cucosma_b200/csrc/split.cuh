// split.cuh -- launchers of the operand pre-passes (BF16 split, Ozaki slices).
#pragma once
#include <algorithm>
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

// Per-column exponents of B (k x n) into eb (the per-row exponents of A are
// written by launch_ozaki_slices, which must follow on the same stream).
cudaError_t launch_ozaki_exponents(const double* A, int64_t lda, const double* B, int64_t ldb, int m, int n, int k,
                                   int32_t* ea, int32_t* eb, int sms, cudaStream_t st);

// Row exponents of A into ea, then s INT8 slices of the rows of A, packed
// (four slices' 32-byte k-blocks per 128-byte row): byte (r, k, p) at
// r * kpad * s + (k / 32) * 32 * s + p * 32 + k % 32; and of the columns of B,
// stacked: byte (n, k, p) at ((k / 32) * s + p) * n_cols * 32 + n * 32 + k % 32.
// kpad a multiple of 32.
cudaError_t launch_ozaki_slices(int s, const double* A, int64_t lda, const double* B, int64_t ldb, int m, int n, int k,
                                int64_t kpad, int32_t* ea, int32_t* eb, int8_t* sa, int8_t* sb, int sms,
                                cudaStream_t st);

}  // namespace cucosma
