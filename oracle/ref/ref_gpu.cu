// The reference kernel cosmaSgemm (Kernel/cuda/src/cuCOSMAV100.cuh:2774-2848)
// compiled unmodified for sm_100a with one compile-time configuration.
// oracle/build_ref.py passes the configuration as -D flags (the macro set of
// Kernel/cuda/src/config.h:9-31); CONFIG_H_ is predefined so the header's own
// config.h (include-guarded) is skipped.  TEST INFRASTRUCTURE ONLY.
#include <algorithm>
#include <cuda_runtime.h>
#include <cublas_v2.h>
#include "Util/helper_math.h"
#include "Util/helper_cuda.h"
#ifdef REF_FP64
// FP64 has never been built by the reference: helper_math.h lacks the
// double2/double4 operators the kernel uses, and the beta pre-scale calls
// cublasSscal on a double pointer.  This shim supplies both.
inline __host__ __device__ double4 operator*(double s, double4 a) { return make_double4(s * a.x, s * a.y, s * a.z, s * a.w); }
inline __host__ __device__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
inline __host__ __device__ void operator+=(double4& a, double4 b) { a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w; }
inline __host__ __device__ void operator+=(double2& a, double2 b) { a.x += b.x; a.y += b.y; }
inline cublasStatus_t cublasSscal_v2(cublasHandle_t h, int n, const float* alpha, double* x, int incx) {
  const double a = *alpha;
  return cublasDscal_v2(h, n, &a, x, incx);
}
#endif
#include "cuCOSMAV100.cuh"

extern "C" int ref_gpu_gemm(const void* A, int lda, const void* B, int ldb, void* C, int ldc) {
  return (int)cosmaSgemm((const TYPE*)A, lda, (const TYPE*)B, ldb, (TYPE*)C, ldc);
}
// m, n, k, tile_m, tile_n, tile_k, load_k, split_k, swizzle, atomic, sizeof(TYPE)
extern "C" void ref_gpu_config(long long* out) {
  out[0] = M; out[1] = N; out[2] = K; out[3] = THREADBLOCK_TILE_M; out[4] = THREADBLOCK_TILE_N;
  out[5] = THREADBLOCK_TILE_K; out[6] = LOAD_K; out[7] = SPLIT_K; out[8] = SWIZZLE;
  out[9] = ATOMIC_REDUCTION ? 1 : 0; out[10] = sizeof(TYPE);
}
extern "C" double ref_gpu_alpha(void) { return (double)(ALPHA); }
extern "C" double ref_gpu_beta(void) { return (double)(BETA); }
