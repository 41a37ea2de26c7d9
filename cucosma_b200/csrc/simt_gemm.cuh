// simt_gemm.cuh -- parameters and launchers of the native FP32/FP64 kernels.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cucosma {

struct SimtParams {
  int m, n, k;
  int kchunk;    // K extent of one split (multiple of the stage depth BK)
  int splits;    // grid.z
  int swizzle;   // block-index remap width (1 = none)
  int tiles_m, tiles_n;
  int partial;   // 1: write raw partial sums to out[z] (split-K workspace)
  int epilogue;
  double alpha, beta;
  void* out;              // C, or the split-K workspace
  int64_t ldo;            // row stride of out (elements)
  int64_t ws_split_stride;  // elements between consecutive splits in the workspace
  WaitCtl ctl;
  // Optional device-side gate: when gate is set the kernel runs only if
  // *gate == gate_value (a path chosen on the device, e.g. the adaptive
  // Ozaki call's native FP64 fallback), and returns at once otherwise.
  const int* gate;
  int gate_value;
};

namespace simt {
constexpr int BM = 128, BN = 128, STAGES = 4;
// Eight warps, all computing; thread 0 also issues the TMA loads.  (A ninth,
// producer-only warp would put three warps in one register-file quadrant
// and cap every thread at 168 registers, which the FP64 8x8 tile exceeds.)
constexpr int kComputeWarps = 8;
constexpr int kThreads = kComputeWarps * 32;

template <typename T>
struct Cfg;
template <>
struct Cfg<float> {
  static constexpr int BK = 16;  // 64-byte A rows
  static constexpr int CTAS_PER_SM = 2;
  static constexpr CUtensorMapSwizzle A_SWIZZLE = CU_TENSOR_MAP_SWIZZLE_64B;
};
template <>
struct Cfg<double> {
  static constexpr int BK = 16;  // 128-byte A rows
  static constexpr int CTAS_PER_SM = 1;
  static constexpr CUtensorMapSwizzle A_SWIZZLE = CU_TENSOR_MAP_SWIZZLE_128B;
};

// CTA shapes of the FP32 kernel: BM_ x 128 tiles, 2 * BM_ threads, 128
// registers a thread; BM_ = 128 or 64.  The 64-row shape keeps 16 warps an
// SM (four CTAs) with three stages, so that four CTAs' shared memory fits.
template <int BM_>
struct SgemmShape {
  static constexpr int kThreads = 2 * BM_;
  static constexpr int kCtasPerSm = BM_ == 128 ? 2 : 4;
  static constexpr int kStages = BM_ == 128 ? 4 : 3;
  static constexpr int kLdT = BM_ + 4;  // k-major A row pitch (floats): 16-byte aligned rows
};
// CTA tile rows the native kernel of type T can run with (FP64: 128 only).
template <typename T>
inline bool tile_rows_supported(int bm) {
  return bm == BM || (sizeof(T) == 4 && bm == 64);
}

// Dynamic shared memory of the GEMM kernel with bm-row CTA tiles.
template <typename T>
size_t smem_bytes(int bm = BM);
// Resident CTAs per SM of the GEMM kernel (CUDA occupancy API).
template <typename T>
int occupancy(int bm = BM);
template <typename T>
cudaError_t launch_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const SimtParams& p, int bm,
                        cudaStream_t stream);
template <typename T>
cudaError_t launch_reduce(const T* ws, int64_t split_stride, int64_t ldw, int splits, T* C, int64_t ldc, int m, int n,
                          double alpha, double beta, int epi, int num_sms, cudaStream_t stream,
                          const int* gate = nullptr, int gate_value = 0);
template <typename T>
cudaError_t launch_scale(T* C, int64_t ldc, int m, int n, double beta, int epi, int num_sms, cudaStream_t stream);
}  // namespace simt

}  // namespace cucosma
