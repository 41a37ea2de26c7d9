// common.cuh -- shared device helpers: epilogue functors and the output
// stage that applies C = epi(alpha*acc + beta*C).
#pragma once
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#include "ptx.cuh"

namespace cucosma {

// Raises a kernel's dynamic shared memory limit to `bytes` once per device
// (the attribute lives in each device's context, so a process that drives
// several GPUs sets it on each); `done` is the kernel's mask of devices
// already set.  Thread-safe: a race only repeats the idempotent call.
inline cudaError_t ensure_smem_attr(const void* fn, int bytes, std::atomic<uint64_t>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev >= 0 && dev < 64 ? (uint64_t(1) << dev) : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
  return e;
}

// With CUCOSMA_DEBUG set in the environment, a failing CUDA call inside the
// library is reported on stderr (the C ABI itself only returns a status).
inline cudaError_t debug_cuda(const char* what, cudaError_t e) {
  static const bool on = std::getenv("CUCOSMA_DEBUG") != nullptr;
  if (e != cudaSuccess && on) std::fprintf(stderr, "cucosma: %s: %s\n", what, cudaGetErrorString(e));
  return e;
}

enum Epilogue : int { kEpiNone = 0, kEpiSigmoid = 1, kEpiRelu = 2 };

// Fused activation applied to the final value (cuCOSMAV100.cuh:2466-2476
// holds the reference's ReLU / Sigmoid loops; sigmoid4.cuh:19-22 the formula).
// epi_t<EPI>: the activation fixed at compile time, for epilogues that
// dispatch once per block.
// FP32 sigmoid 1 / (1 + e^-v) without a division: the reciprocal of
// x = 1 + e^-v (x >= 1) from the hardware approximation refined by one
// Newton-Raphson step r <- r + r (1 - x r), which squares its relative error
// (from about 2^-23 to below 2^-44, so the result is within an ulp of the
// correctly rounded quotient); x = +inf (v below about -88) gives 0.  The
// IEEE division it replaces carries an out-of-line slow path whose call
// sites made the tensor-core epilogue (128 live accumulator registers a
// thread) several times slower on B200.
__device__ __forceinline__ float sigmoid_f32(float v) {
  const float x = 1.0f + expf(-v);
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  r = fmaf(r, fmaf(-x, r, 1.0f), r);
  return x == __int_as_float(0x7f800000) ? 0.0f : r;
}
template <int EPI>
__device__ __forceinline__ float epi_t(float v) {
  if constexpr (EPI == kEpiSigmoid) return sigmoid_f32(v);
  else if constexpr (EPI == kEpiRelu) return fmaxf(v, 0.0f);
  else return v;
}
template <int EPI>
__device__ __forceinline__ double epi_t(double v) {
  if constexpr (EPI == kEpiSigmoid) return 1.0 / (1.0 + exp(-v));
  else if constexpr (EPI == kEpiRelu) return fmax(v, 0.0);
  else return v;
}
// apply_epi: chosen at run time per value.  The sigmoid is a call, never
// inlined: inlined, the compiler if-converted it, evaluating the exponential
// and the division for every element of every epilogue (that made the FP32
// tensor-core epilogue five times slower on B200 with no activation at all).
__device__ __noinline__ float sigmoid_f32_call(float v);
__device__ __noinline__ double sigmoid_f64(double v);
__device__ __forceinline__ float apply_epi(float v, int epi) {
  if (epi == kEpiRelu) return fmaxf(v, 0.0f);
  if (epi == kEpiSigmoid) return sigmoid_f32_call(v);
  return v;
}
__device__ __forceinline__ double apply_epi(double v, int epi) {
  if (epi == kEpiRelu) return fmax(v, 0.0);
  if (epi == kEpiSigmoid) return sigmoid_f64(v);
  return v;
}
__device__ __noinline__ inline float sigmoid_f32_call(float v) { return sigmoid_f32(v); }
__device__ __noinline__ inline double sigmoid_f64(double v) { return epi_t<kEpiSigmoid>(v); }

// alpha/beta combination.  The reference scales the accumulator by ALPHA
// first and then adds BETA*C (cuCOSMAV100.cuh:1582-1593, :901); written here
// as one explicit FMA so every path (and the oracle) rounds the same way.
// C is not read when beta == 0.
template <typename T>
__device__ __forceinline__ T combine(T acc, T alpha, T beta, const T* cptr) {
  T v = alpha * acc;
  if (beta != T(0)) v = fma(beta, *cptr, v);
  return v;
}

template <typename T>
struct Vec;
template <>
struct Vec<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <>
struct Vec<double> {
  using type = double2;
  static constexpr int n = 2;
};

__host__ __device__ constexpr int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ constexpr int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

}  // namespace cucosma
