// cucosma.hpp -- compile-time drop-in for the reference's kernel API.
//
// The reference is used as
//     #include "config.h"          // M, N, K, ALPHA, BETA, TYPE, tiling macros
//     #include "cuCOSMAV100.cuh"
//     cublasStatus_t s = cosmaSgemm(A, lda, B, ldb, C, ldc);
// (Kernel/cuda/src/cuCOSMAV100.cuh:2774-2776).  This header keeps the call:
//     cublasStatus_t s = cosmaSgemm<M, N, K>(A, lda, B, ldb, C, ldc, alpha, beta);
// with M, N, K as template parameters and alpha, beta as arguments
// (defaults 1, 0), TYPE = float or double deduced from the pointers, an
// optional fused epilogue and precision, and the caller's stream.  Tiling and
// split-K are chosen by the library at run time (the reference fixed them in
// config.h from the ScheduleGenerator).  Link with -lcucosma.
//
// Status mapping: SUCCESS -> CUBLAS_STATUS_SUCCESS; INVALID_VALUE and
// MISALIGNED -> CUBLAS_STATUS_INVALID_VALUE (the reference returned it only for
// negative sizes); NOT_SUPPORTED -> CUBLAS_STATUS_NOT_SUPPORTED;
// ARCH_MISMATCH -> CUBLAS_STATUS_ARCH_MISMATCH; ALLOC_FAILED and
// WORKSPACE_TOO_SMALL -> CUBLAS_STATUS_ALLOC_FAILED; LAUNCH_FAILED, TIMEOUT and
// INTERNAL_ERROR -> CUBLAS_STATUS_EXECUTION_FAILED.
//
// Template parameters are named kM/kN/kK so that a config.h that #defines
// M, N, K may be included before this header (see cucosma_config_compat.h).
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "cucosma.h"

namespace cucosma {

inline cublasStatus_t to_cublas(cucosma_status s) {
  switch (s) {
    case CUCOSMA_STATUS_SUCCESS: return CUBLAS_STATUS_SUCCESS;
    case CUCOSMA_STATUS_INVALID_VALUE:
    case CUCOSMA_STATUS_MISALIGNED: return CUBLAS_STATUS_INVALID_VALUE;
    case CUCOSMA_STATUS_NOT_SUPPORTED: return CUBLAS_STATUS_NOT_SUPPORTED;
    case CUCOSMA_STATUS_ARCH_MISMATCH: return CUBLAS_STATUS_ARCH_MISMATCH;
    case CUCOSMA_STATUS_ALLOC_FAILED:
    case CUCOSMA_STATUS_WORKSPACE_TOO_SMALL: return CUBLAS_STATUS_ALLOC_FAILED;
    default: return CUBLAS_STATUS_EXECUTION_FAILED;
  }
}

// Full form: precision (cucosma_precision) and epilogue (cucosma_epilogue)
// selectable; the workspace is library-managed like the reference's split-K
// buffer (one per device and stream, grown on demand instead of allocated
// and freed per call: cucosma_gemm_managed).
template <int kM, int kN, int kK, class T>
cublasStatus_t cosmaGemm(const T* A, int lda, const T* B, int ldb, T* C, int ldc, T alpha, T beta,
                         int precision, int epilogue, cudaStream_t stream) {
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "TYPE must be float or double");
  if (kM < 0 || kN < 0 || kK < 0) return CUBLAS_STATUS_INVALID_VALUE;  // as cuCOSMAV100.cuh:2778-2780
  cucosma_gemm_desc d;
  cucosma_gemm_desc_init(&d);
  d.m = kM;
  d.n = kN;
  d.k = kK;
  d.lda = lda;
  d.ldb = ldb;
  d.ldc = ldc;
  d.dtype = std::is_same<T, float>::value ? CUCOSMA_R_32F : CUCOSMA_R_64F;
  d.precision = precision;
  d.epilogue = epilogue;
  d.alpha = (double)alpha;
  d.beta = (double)beta;
  if (precision == CUCOSMA_PRECISION_NATIVE && epilogue == CUCOSMA_EPILOGUE_NONE) {
    if (std::is_same<T, float>::value)
      return to_cublas(cucosma_sgemm(kM, kN, kK, (float)alpha, (const float*)A, lda, (const float*)B, ldb,
                                     (float)beta, (float*)C, ldc, stream));
    return to_cublas(cucosma_dgemm(kM, kN, kK, (double)alpha, (const double*)A, lda, (const double*)B, ldb,
                                   (double)beta, (double*)C, ldc, stream));
  }
  return to_cublas(cucosma_gemm_managed(&d, A, B, C, stream));
}

}  // namespace cucosma

// The reference's name and argument order; M, N, K at compile time.
template <int kM, int kN, int kK, class T>
inline cublasStatus_t cosmaSgemm(const T* A, int lda, const T* B, int ldb, T* C, int ldc, T alpha = T(1),
                                 T beta = T(0), cudaStream_t stream = 0) {
  return cucosma::cosmaGemm<kM, kN, kK, T>(A, lda, B, ldb, C, ldc, alpha, beta, CUCOSMA_PRECISION_NATIVE,
                                           CUCOSMA_EPILOGUE_NONE, stream);
}

// FP64 spelling of the same (the reference's TYPE=double instantiation).
template <int kM, int kN, int kK>
inline cublasStatus_t cosmaDgemm(const double* A, int lda, const double* B, int ldb, double* C, int ldc,
                                 double alpha = 1.0, double beta = 0.0, cudaStream_t stream = 0) {
  return cosmaSgemm<kM, kN, kK, double>(A, lda, B, ldb, C, ldc, alpha, beta, stream);
}
