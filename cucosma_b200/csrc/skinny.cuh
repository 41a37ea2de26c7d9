// skinny.cuh -- native-precision kernels for the reference's skinny shapes
// (a tiny K, or a tiny M or N), where a 128 x 128 tile would do almost no
// useful work.  The shapes come from the reference's special benchmark list
// (Benchmarks/TESTS_TO_RUN/special.csv: 4 x 8 x 3,000,000, 4 x 3,000,000 x 4,
// 38416 x 38416 x 4), where they are HBM-bound.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cucosma {

struct SkinnyPlan {
  int kind;        // 0: not skinny (tile kernel), 1: small K, 2: thin M or N (8 x 8 blocks, K split)
  int splits;      // kind 2: K splits (partials reduced in split order)
  int64_t kchunk;  // kind 2: K extent of one split
  int64_t ldw;     // kind 2: row stride of the partial-sum workspace
  size_t ws_bytes;
  int tile_m, tile_n;  // output block of one CTA
};

namespace skinny {
constexpr int kMaxSmallK = 16;  // kind 1 when K <= this
constexpr int kThin = 8;        // kind 2 when M <= this or N <= this
}  // namespace skinny

// desc must describe a native-precision GEMM with m, n, k > 0.
SkinnyPlan plan_skinny(int64_t m, int64_t n, int64_t k, int dtype_bytes, int split_k, int tile, int sms);

template <typename T>
cudaError_t launch_skinny(const SkinnyPlan& pl, const T* A, int64_t lda, const T* B, int64_t ldb, T* C, int64_t ldc,
                          int m, int n, int k, double alpha, double beta, int epi, void* ws, int sms,
                          cudaStream_t st);

}  // namespace cucosma
