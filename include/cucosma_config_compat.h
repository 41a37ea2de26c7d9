// cucosma_config_compat.h -- build unchanged callers of the reference.
//
// Reference callers define the problem in a generated config.h
// (Kernel/cuda/src/config.h:9-31: TYPE, M, N, K, ALPHA, BETA, tiling macros)
// and call the six-argument cosmaSgemm(A, lda, B, ldb, C, ldc)
// (Kernel/cuda/src/cuCOSMAV100.cuh:2774).  Including this header after
// config.h (in place of cuCOSMAV100.cuh) provides exactly that function,
// backed by the library; the tiling macros (THREADBLOCK_TILE_*, WARP_TILE_*,
// THREAD_TILE_*, LOAD_K, SPLIT_K, SWIZZLE, ...) are accepted and ignored:
// the library chooses tiles and split-K at run time.
#pragma once

#include "cucosma.hpp"

#if !defined(M) || !defined(N) || !defined(K) || !defined(TYPE)
#error "cucosma_config_compat.h: include the caller's config.h (defining TYPE, M, N, K) first"
#endif
#ifndef ALPHA
#define ALPHA 1
#endif
#ifndef BETA
#define BETA 0
#endif

inline cublasStatus_t cosmaSgemm(const TYPE* A, const int lda, const TYPE* B, const int ldb, TYPE* C, const int ldc) {
  return cosmaSgemm<M, N, K, TYPE>(A, lda, B, ldb, C, ldc, (TYPE)(ALPHA), (TYPE)(BETA), 0);
}
