// noalloc.cu -- the allocation-free FP32 split-K entry point.
//
// cucosma_gemm needs a caller-provided workspace for split-K, and
// cucosma_sgemm grows a library-managed one with cudaMalloc.  Some callers
// can do neither: a plugin invoked by a host framework that owns the whole
// device memory pool and forbids its plugins to allocate, or a caller on a
// latency-critical path that must not hit cudaMalloc's implicit device
// synchronisation.  For them, cucosma_sgemm_splitk_static runs the same
// native FP32 split-K kernels with their partial sums in a fixed device
// array defined in this file, so a call allocates nothing.
//
// The array (CUCOSMA_STATIC_SCRATCH_BYTES) exists once per device that
// loads the library and stays allocated until the process exits.  Every call
// on a device shares it and it keeps the previous call's contents; the split
// kernels overwrite every element the reduction later reads, so nothing needs
// clearing.  Calls whose GPU execution overlaps (different streams, or
// different host threads) race on the array; the caller must order them.
#include <mutex>
#include <vector>

#include "../../include/cucosma.h"
#include "api_internal.cuh"
#include "simt_gemm.cuh"

namespace cucosma {

static __device__ __align__(256) unsigned char g_static_scratch[CUCOSMA_STATIC_SCRATCH_BYTES];

// Device address of g_static_scratch on the current device.  In host code
// the symbol names a host-side stand-in, not device memory, so the address
// comes from cudaGetSymbolAddress, once per device with that device current.
static cucosma_status static_scratch(void** out) {
  static std::mutex mu;
  static std::vector<void*> addr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)addr.size() <= dev) addr.resize(dev + 1, nullptr);
  if (!addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) return CUCOSMA_STATUS_LAUNCH_FAILED;
    addr[dev] = p;
  }
  *out = addr[dev];
  return CUCOSMA_STATUS_SUCCESS;
}

}  // namespace cucosma

using namespace cucosma;

extern "C" cucosma_status cucosma_sgemm_splitk_static(int m, int n, int k, float alpha, const float* A, int lda,
                                                      const float* B, int ldb, float beta, float* C, int ldc,
                                                      int split_k, void* stream) {
  cucosma_gemm_desc d;
  cucosma_gemm_desc_init(&d);
  d.m = m;
  d.n = n;
  d.k = k;
  d.lda = lda;
  d.ldb = ldb;
  d.ldc = ldc;
  d.dtype = CUCOSMA_R_32F;
  d.alpha = alpha;
  d.beta = beta;
  d.split_k = split_k;
  cucosma_status s = validate(&d, A, B, C);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (split_k < 0) return CUCOSMA_STATUS_INVALID_VALUE;
  if (m == 0 || n == 0) return CUCOSMA_STATUS_SUCCESS;
  if (k == 0 || alpha == 0.0f) {
    // No product term and no scratch: the library's regular path (a scale
    // kernel over C) allocates nothing either.
    return gemm(&d, A, B, C, nullptr, 0, static_cast<cudaStream_t>(stream));
  }
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (di->cc_major != 10 || di->cc_minor != 0) return CUCOSMA_STATUS_ARCH_MISMATCH;
  const NativePlan pl = plan_native(&d, di->sms, (size_t)CUCOSMA_STATIC_SCRATCH_BYTES);
  if (pl.ws_bytes > (size_t)CUCOSMA_STATIC_SCRATCH_BYTES) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  void* scratch = nullptr;
  if (pl.ws_bytes > 0) {
    s = static_scratch(&scratch);
    if (s != CUCOSMA_STATUS_SUCCESS) return s;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUtensorMap tmA, tmB;
  constexpr int BK = simt::Cfg<float>::BK;
  if (!encode_2d(&tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, A, k, m, lda, BK, pl.bm, simt::Cfg<float>::A_SWIZZLE))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (!encode_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, B, n, k, ldb, simt::BN, BK, CU_TENSOR_MAP_SWIZZLE_NONE))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  SimtParams p{};
  p.m = m;
  p.n = n;
  p.k = k;
  p.kchunk = (int)pl.kchunk;
  p.splits = pl.splits;
  p.swizzle = pl.swizzle;
  p.tiles_m = pl.tiles_m;
  p.tiles_n = pl.tiles_n;
  p.epilogue = CUCOSMA_EPILOGUE_NONE;
  p.alpha = alpha;
  p.beta = beta;
  wait_ctl(di, &p.ctl.status, &p.ctl.timeout_ns);
  if (pl.splits > 1) {
    p.partial = 1;
    p.out = scratch;
    p.ldo = pl.ldw;
    p.ws_split_stride = (int64_t)m * pl.ldw;
  } else {
    p.partial = 0;
    p.out = C;
    p.ldo = ldc;
  }
  if (simt::launch_gemm<float>(tmA, tmB, p, pl.bm, st) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  note_launches(1);
  if (pl.splits > 1) {
    if (simt::launch_reduce<float>(static_cast<const float*>(scratch), p.ws_split_stride, pl.ldw, pl.splits, C, ldc, m,
                                   n, alpha, beta, CUCOSMA_EPILOGUE_NONE, di->sms, st) != cudaSuccess)
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    note_launches(1);
  }
  return CUCOSMA_STATUS_SUCCESS;
}
