// A reference-style caller: config.h macros + the six-argument cosmaSgemm,
// plus the template form, built against include/cucosma*.h and libcucosma.so.
// Prints "max_err <x>" per call and exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "cucosma.hpp"

// What the reference's run.sh writes into config.h (Kernel/cuda/run.sh:200-257).
#define TYPE float
#define VECTORTYPE2 float2
#define VECTORTYPE4 float4
#define M 300
#define N 200
#define K 100
#define THREADBLOCK_TILE_M 128
#define THREADBLOCK_TILE_N 128
#define THREADBLOCK_TILE_K 100
#define LOAD_K 8
#define SPLIT_K 1
#define SWIZZLE 1
#define ALPHA 1.5
#define BETA 0.5
#include "cucosma_config_compat.h"

template <class T>
static double run_case(bool compat) {
  const int m = M, n = N, k = K;
  std::mt19937 rng(1);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<T> a(m * k), b(k * n), c(m * n);
  for (auto& x : a) x = (T)u(rng);
  for (auto& x : b) x = (T)u(rng);
  for (auto& x : c) x = (T)u(rng);
  T *dA, *dB, *dC;
  size_t pa, pb, pc;  // pitched rows as the reference's callers allocate them (test_correctness.h:55-58)
  if (cudaMallocPitch(&dA, &pa, k * sizeof(T), m) || cudaMallocPitch(&dB, &pb, n * sizeof(T), k) ||
      cudaMallocPitch(&dC, &pc, n * sizeof(T), m))
    return 1e30;
  cudaMemcpy2D(dA, pa, a.data(), k * sizeof(T), k * sizeof(T), m, cudaMemcpyHostToDevice);
  cudaMemcpy2D(dB, pb, b.data(), n * sizeof(T), n * sizeof(T), k, cudaMemcpyHostToDevice);
  cudaMemcpy2D(dC, pc, c.data(), n * sizeof(T), n * sizeof(T), m, cudaMemcpyHostToDevice);
  cublasStatus_t s;
  if (compat)
    s = cosmaSgemm((const TYPE*)dA, (int)(pa / sizeof(T)), (const TYPE*)dB, (int)(pb / sizeof(T)), (TYPE*)dC,
                   (int)(pc / sizeof(T)));
  else
    s = cosmaSgemm<M, N, K>(dA, (int)(pa / sizeof(T)), dB, (int)(pb / sizeof(T)), dC, (int)(pc / sizeof(T)),
                            (T)ALPHA, (T)BETA);
  if (s != CUBLAS_STATUS_SUCCESS) {
    std::printf("status %d\n", (int)s);
    return 1e30;
  }
  std::vector<T> out(m * n);
  cudaMemcpy2D(out.data(), n * sizeof(T), dC, pc, n * sizeof(T), m, cudaMemcpyDeviceToHost);
  double err = 0;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      double acc = 0;
      for (int l = 0; l < k; ++l) acc += (double)a[i * k + l] * (double)b[l * n + j];
      const double ref = ALPHA * acc + BETA * (double)c[i * n + j];
      err = std::fmax(err, std::fabs(ref - (double)out[i * n + j]));
    }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dC);
  return err;
}

int main() {
  const double e1 = run_case<float>(true);
  const double e2 = run_case<float>(false);
  const double e3 = run_case<double>(false);
  std::printf("max_err compat_f32 %.3e template_f32 %.3e template_f64 %.3e\n", e1, e2, e3);
  // negative compile-time size: the reference's only error check
  const cublasStatus_t neg = cosmaSgemm<-1, 4, 4>((const float*)nullptr, 4, (const float*)nullptr, 4, (float*)nullptr, 4);
  std::printf("negative_size_status %d\n", (int)neg);
  const bool ok = e1 < 1e-4 && e2 < 1e-4 && e3 < 1e-12 && neg == CUBLAS_STATUS_INVALID_VALUE;
  return ok ? 0 : 1;
}
