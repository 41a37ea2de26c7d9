// api.cu -- the C ABI (include/cucosma.h): validation, planning, tensor-map
// encoding and dispatch to the kernels.
//
// Reference host API being replaced: cosmaSgemm (cuCOSMAV100.cuh:2774-2848).
// Differences by design: sizes and scalars are runtime values, errors are
// returned (the reference exits through checkCudaErrors,
// Util/helper_cuda.h:574-586, and never checks its launches), the split-K
// workspace is the caller's (the reference cudaMallocs and frees it on every
// call, :2828-2838), and the beta pre-scale never needs cuBLAS.
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/cucosma.h"
#include "api_internal.cuh"
#include "simt_gemm.cuh"
#include "skinny.cuh"

namespace cucosma {

// Device status word (one per device that loads the library).
__device__ int g_device_status = 0;
static std::atomic<unsigned long long> g_wait_timeout_ns{4000000000ull};

void wait_ctl(const DeviceInfo* di, int** status, unsigned long long* timeout_ns) {
  *status = di->status;
  *timeout_ns = g_wait_timeout_ns.load();
}

// ---------------------------------------------------------------- device info
const DeviceInfo* device_info() {
  static std::mutex mu;
  static std::vector<DeviceInfo> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1);
  DeviceInfo& d = cache[dev];
  if (!d.valid) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return nullptr;
    d.sms = prop.multiProcessorCount;
    d.cc_major = prop.major;
    d.cc_minor = prop.minor;
    d.l2_bytes = prop.l2CacheSize;
    d.smem_optin = (int)prop.sharedMemPerBlockOptin;
    void* st = nullptr;
    if (cudaGetSymbolAddress(&st, g_device_status) != cudaSuccess) return nullptr;
    d.status = static_cast<int*>(st);
    d.valid = true;
  }
  return &d;
}

// ------------------------------------------------------------ tensor maps
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

bool encode_2d(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, const void* base, uint64_t inner,
               uint64_t outer, uint64_t row_stride_elems, uint32_t box_inner, uint32_t box_outer,
               CUtensorMapSwizzle swz) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {row_stride_elems * (uint64_t)elem_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool encode_3d(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, const void* base, uint64_t d0, uint64_t d1,
               uint64_t d2, uint64_t stride1_elems, uint64_t stride2_elems, uint32_t b0, uint32_t b1, uint32_t b2,
               CUtensorMapSwizzle swz) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {stride1_elems * (uint64_t)elem_bytes, stride2_elems * (uint64_t)elem_bytes};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, dt, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// ------------------------------------------------------------- validation
static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

cucosma_status validate(const cucosma_gemm_desc* d, const void* A, const void* B, const void* C) {
  if (!d) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->m < 0 || d->n < 0 || d->k < 0) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->m > INT32_MAX || d->n > INT32_MAX || d->k > INT32_MAX) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->dtype != CUCOSMA_R_32F && d->dtype != CUCOSMA_R_64F) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->precision < CUCOSMA_PRECISION_NATIVE || d->precision > CUCOSMA_PRECISION_OZAKI)
    return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->epilogue < CUCOSMA_EPILOGUE_NONE || d->epilogue > CUCOSMA_EPILOGUE_RELU) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->split_k < 0 || d->swizzle < 0) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->flags != 0 && (d->flags != CUCOSMA_FLAG_TEST_SKIP_STAGE || d->precision == CUCOSMA_PRECISION_NATIVE))
    return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->slices != 0 && (d->slices < 4 || d->slices > 9)) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->m == 0 || d->n == 0) return CUCOSMA_STATUS_SUCCESS;
  if (d->ldc < d->n) return CUCOSMA_STATUS_INVALID_VALUE;
  if (!C) return CUCOSMA_STATUS_INVALID_VALUE;
  const bool product = d->k > 0 && d->alpha != 0.0;
  if (product) {
    if (d->lda < d->k || d->ldb < d->n) return CUCOSMA_STATUS_INVALID_VALUE;
    if (!A || !B) return CUCOSMA_STATUS_INVALID_VALUE;
  }
  if ((d->precision == CUCOSMA_PRECISION_BF16X3 || d->precision == CUCOSMA_PRECISION_BF16X6) &&
      d->dtype != CUCOSMA_R_32F)
    return CUCOSMA_STATUS_NOT_SUPPORTED;
  if (d->precision == CUCOSMA_PRECISION_OZAKI && d->dtype != CUCOSMA_R_64F) return CUCOSMA_STATUS_NOT_SUPPORTED;
  const int es = d->dtype == CUCOSMA_R_32F ? 4 : 8;
  if (!aligned16(C) || (d->ldc * es) % 16) return CUCOSMA_STATUS_MISALIGNED;
  if (product) {
    if (!aligned16(A) || !aligned16(B) || (d->lda * es) % 16 || (d->ldb * es) % 16) return CUCOSMA_STATUS_MISALIGNED;
  }
  return CUCOSMA_STATUS_SUCCESS;
}

// --------------------------------------------------------------- planning
static int simt_bk(int dtype) { return dtype == CUCOSMA_R_32F ? simt::Cfg<float>::BK : simt::Cfg<double>::BK; }

// Modelled time (us) of the tile kernel with bm-row CTA tiles, `tiles` output
// tiles and `s` K splits of `kblocks` 16-deep k-blocks in all, plus the
// split-K reduction (s partial planes of per_split bytes in and out at HBM
// speed, and a launch).  Fitted to B200 measurements of both FP32 tile
// heights over square, flat, large-N and large-K shapes:
//   * a 128 x 128 x 16 k-block step takes kUnitUs of an SM holding 16 warps
//     (FP64: kUnitUsF64 a CTA, one CTA an SM);
//   * an SM holding fewer warps runs at occupancy_rate() of that (one 4-warp
//     CTA alone: 0.71; 8 warps: 0.91);
//   * the 64-row CTAs do a 64-row step in 0.95 of half a 128-row step (four
//     4-warp CTAs an SM stall less at the per-stage barrier than two 8-warp
//     ones);
//   * whole waves of resident CTAs run at full occupancy, and the last,
//     partial wave at the occupancy it leaves.
namespace {
constexpr double kUnitUs = 1.45, kUnitUsF64 = 2.4, kTile64Factor = 0.95;
double occupancy_rate(int warps) {
  return warps >= 16 ? 1.0 : warps >= 14 ? 0.99 : warps >= 12 ? 0.97 : warps >= 10 ? 0.95 : warps >= 8 ? 0.91
                       : warps >= 6 ? 0.8 : 0.71;
}
double native_time_us(int bm, bool fp32, int64_t tiles, int64_t s, int64_t kblocks, int sms, size_t per_split) {
  const int per_sm = fp32 ? (bm == 64 ? simt::SgemmShape<64>::kCtasPerSm : simt::SgemmShape<128>::kCtasPerSm)
                          : simt::Cfg<double>::CTAS_PER_SM;
  const int warps_per_cta = fp32 ? bm / 16 : 16;  // FP64: one CTA fills its SM's FP64 rate
  const double step = fp32 ? kUnitUs * (bm == 64 ? 0.5 * kTile64Factor : 1.0) : kUnitUsF64;  // one CTA k-block, full SM
  const int64_t ctas = tiles * s, slots = (int64_t)sms * per_sm;
  const double kbs = (double)ceil_div(kblocks, s);
  const int64_t waves = ctas / slots, rest = ctas - waves * slots;
  double t = (double)waves * kbs * per_sm * step;
  if (rest > 0) {
    const int r = (int)ceil_div(rest, (int64_t)sms);  // CTAs on the busiest SM of the last wave
    t += kbs * r * step / occupancy_rate(r * warps_per_cta);
  }
  if (s > 1) t += 2.0 + 2.0 * (double)s * (double)per_split / 6.0e6;
  return t;
}
}  // namespace

NativePlan plan_native(const cucosma_gemm_desc* d, int sms, size_t max_ws) {
  NativePlan p{};
  const bool fp32 = d->dtype == CUCOSMA_R_32F;
  const int bk = simt_bk(d->dtype);
  const int es = fp32 ? 4 : 8;
  const int vec = 16 / es;
  const int64_t kblocks = std::max<int64_t>(1, ceil_div(d->k, bk));
  const size_t per_split = (size_t)d->m * (size_t)round_up(d->n, vec) * es;
  // Tile heights to consider: tile id 1 = 128 rows, 2 = 64 rows (FP32), 0 = both.
  int heights[2] = {simt::BM, 64};
  int nh = 1;
  if (fp32 && d->tile == 2) heights[0] = 64;
  else if (fp32 && d->tile == 0) nh = 2;
  const int64_t tiles_n = ceil_div(d->n, simt::BN);
  int64_t splits = d->split_k;
  int bm = heights[0];
  if (splits <= 0) {
    // The (height, split) pair with the smallest modelled time wins; splits
    // keep >= 4 k-blocks each and fit max_ws, and a candidate must beat the
    // best so far by 2 % (ties keep the taller tile and the smaller split).
    const int64_t smax = std::max<int64_t>(1, std::min<int64_t>(kblocks / 4, 512));
    double best = 1e300;
    splits = 1;
    for (int h = 0; h < nh; ++h) {
      const int64_t tiles = ceil_div(d->m, heights[h]) * tiles_n;
      for (int64_t s = 1; s <= smax; ++s) {
        if (s > 1 && (size_t)s * per_split > max_ws) break;
        const double t = native_time_us(heights[h], fp32, tiles, s, kblocks, sms, per_split);
        if (t < best * 0.98) {
          best = t;
          splits = s;
          bm = heights[h];
        }
      }
    }
  } else if (nh == 2) {
    // forced split: the height with the smaller modelled time
    const int64_t s = std::min<int64_t>(splits, kblocks);
    const double t128 = native_time_us(128, fp32, ceil_div(d->m, 128) * tiles_n, s, kblocks, sms, per_split);
    const double t64 = native_time_us(64, fp32, ceil_div(d->m, 64) * tiles_n, s, kblocks, sms, per_split);
    bm = t64 < t128 * 0.98 ? 64 : 128;
  }
  p.bm = bm;
  p.tiles_m = (int)ceil_div(d->m, bm);
  p.tiles_n = (int)tiles_n;
  splits = std::max<int64_t>(1, std::min<int64_t>(splits, kblocks));
  splits = std::min<int64_t>(splits, 65535);
  int64_t kchunk = round_up(ceil_div(std::max<int64_t>(d->k, 1), splits), bk);
  splits = ceil_div(std::max<int64_t>(d->k, 1), kchunk);
  p.splits = (int)splits;
  p.kchunk = kchunk;
  int sw = d->swizzle > 0 ? d->swizzle : 1;
  p.swizzle = sw;
  p.ldw = round_up(d->n, vec);
  p.ws_bytes = p.splits > 1 ? (size_t)p.splits * (size_t)d->m * (size_t)p.ldw * es : 0;
  return p;
}

// ---------------------------------------------------------------- dispatch
template <typename T>
static cucosma_status run_native(const cucosma_gemm_desc* d, const NativePlan& pl, const T* A, const T* B, T* C,
                                 void* ws, const DeviceInfo* di, cudaStream_t st, const int* gate = nullptr,
                                 int gate_value = 0, bool profile = true) {
  constexpr int BK = simt::Cfg<T>::BK;
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  CUtensorMap tmA, tmB;
  if (!encode_2d(&tmA, dt, sizeof(T), A, d->k, d->m, d->lda, BK, pl.bm, simt::Cfg<T>::A_SWIZZLE))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (!encode_2d(&tmB, dt, sizeof(T), B, d->n, d->k, d->ldb, simt::BN, BK, CU_TENSOR_MAP_SWIZZLE_NONE))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  SimtParams p{};
  p.m = (int)d->m;
  p.n = (int)d->n;
  p.k = (int)d->k;
  p.kchunk = (int)pl.kchunk;
  p.splits = pl.splits;
  p.swizzle = pl.swizzle;
  p.tiles_m = pl.tiles_m;
  p.tiles_n = pl.tiles_n;
  p.epilogue = d->epilogue;
  p.alpha = d->alpha;
  p.beta = d->beta;
  p.gate = gate;
  p.gate_value = gate_value;
  wait_ctl(di, &p.ctl.status, &p.ctl.timeout_ns);
  if (pl.splits > 1) {
    p.partial = 1;
    p.out = ws;
    p.ldo = pl.ldw;
    p.ws_split_stride = (int64_t)d->m * pl.ldw;
  } else {
    p.partial = 0;
    p.out = C;
    p.ldo = d->ldc;
  }
  if (profile) prof_begin(st);
  if (simt::launch_gemm<T>(tmA, tmB, p, pl.bm, st) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (profile) prof_end(st);
  note_launches(pl.splits > 1 ? 2 : 1);
  if (pl.splits > 1) {
    if (simt::launch_reduce<T>(static_cast<const T*>(ws), p.ws_split_stride, pl.ldw, pl.splits, C, d->ldc, p.m, p.n,
                               d->alpha, d->beta, d->epilogue, di->sms, st, gate, gate_value) != cudaSuccess)
      return CUCOSMA_STATUS_LAUNCH_FAILED;
  }
  return CUCOSMA_STATUS_SUCCESS;
}

cucosma_status native_gemm_gated(const cucosma_gemm_desc* d, const NativePlan& pl, const void* A, const void* B,
                                 void* C, void* ws, const DeviceInfo* di, cudaStream_t st, const int* gate,
                                 int gate_value) {
  if (d->dtype == CUCOSMA_R_32F)
    return run_native<float>(d, pl, (const float*)A, (const float*)B, (float*)C, ws, di, st, gate, gate_value, false);
  return run_native<double>(d, pl, (const double*)A, (const double*)B, (double*)C, ws, di, st, gate, gate_value,
                            false);
}

// Skinny-shape kernels (skinny.cu) for native precision: tiny K, or tiny M or N.
static SkinnyPlan plan_skinny_for(const cucosma_gemm_desc* d, int sms) {
  return plan_skinny(d->m, d->n, d->k, d->dtype == CUCOSMA_R_32F ? 4 : 8, d->split_k, d->tile, sms);
}

template <typename T>
static cucosma_status run_skinny(const cucosma_gemm_desc* d, const SkinnyPlan& sp, const T* A, const T* B, T* C,
                                 void* ws, const DeviceInfo* di, cudaStream_t st) {
  prof_begin(st);
  const cudaError_t e = launch_skinny<T>(sp, A, d->lda, B, d->ldb, C, d->ldc, (int)d->m, (int)d->n, (int)d->k,
                                         d->alpha, d->beta, d->epilogue, ws, di->sms, st);
  prof_end(st);
  note_launches(sp.splits > 1 ? 2 : 1);
  return e == cudaSuccess ? CUCOSMA_STATUS_SUCCESS : CUCOSMA_STATUS_LAUNCH_FAILED;
}

cucosma_status workspace_size(const cucosma_gemm_desc* d, size_t* bytes, const DeviceInfo* di) {
  *bytes = 0;
  if (d->m == 0 || d->n == 0 || d->k == 0 || d->alpha == 0.0) return CUCOSMA_STATUS_SUCCESS;
  switch (d->precision) {
    case CUCOSMA_PRECISION_NATIVE: {
      const SkinnyPlan sp = plan_skinny_for(d, di->sms);
      *bytes = sp.kind ? sp.ws_bytes : plan_native(d, di->sms).ws_bytes;
      return CUCOSMA_STATUS_SUCCESS;
    }
    default:
      return tc_workspace_size(d, bytes, di);
  }
}

cucosma_status gemm(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws, size_t ws_bytes,
                    cudaStream_t st) {
  return gemm_ex(d, A, B, C, ws, ws_bytes, st, kPrepA | kPrepB);
}

cucosma_status gemm_ex(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws, size_t ws_bytes,
                       cudaStream_t st, int prep) {
  cucosma_status s = validate(d, A, B, C);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (d->m == 0 || d->n == 0) return CUCOSMA_STATUS_SUCCESS;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (di->cc_major != 10 || di->cc_minor != 0) return CUCOSMA_STATUS_ARCH_MISMATCH;
  cucosma_gemm_desc tuned;
  d = apply_tuning(d, &tuned, di);
  const bool fp32 = d->dtype == CUCOSMA_R_32F;
  if (d->k == 0 || d->alpha == 0.0) {
    cudaError_t e = fp32 ? simt::launch_scale<float>((float*)C, d->ldc, (int)d->m, (int)d->n, d->beta, d->epilogue,
                                                     di->sms, st)
                         : simt::launch_scale<double>((double*)C, d->ldc, (int)d->m, (int)d->n, d->beta, d->epilogue,
                                                      di->sms, st);
    note_launches(1);
    return e == cudaSuccess ? CUCOSMA_STATUS_SUCCESS : CUCOSMA_STATUS_LAUNCH_FAILED;
  }
  size_t need = 0;
  s = workspace_size(d, &need, di);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (need > 0 && (ws == nullptr || ws_bytes < need)) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  if (need > 0 && !aligned16(ws)) return CUCOSMA_STATUS_MISALIGNED;
  if (d->precision == CUCOSMA_PRECISION_NATIVE) {
    const SkinnyPlan sp = plan_skinny_for(d, di->sms);
    if (sp.kind)
      return fp32 ? run_skinny<float>(d, sp, (const float*)A, (const float*)B, (float*)C, ws, di, st)
                  : run_skinny<double>(d, sp, (const double*)A, (const double*)B, (double*)C, ws, di, st);
    const NativePlan pl = plan_native(d, di->sms);
    return fp32 ? run_native<float>(d, pl, (const float*)A, (const float*)B, (float*)C, ws, di, st)
                : run_native<double>(d, pl, (const double*)A, (const double*)B, (double*)C, ws, di, st);
  }
  return tc_gemm_ex(d, A, B, C, ws, ws_bytes, di, st, prep);
}

// ---------------------------------------------- launch count and profiling
static std::atomic<unsigned long long> g_launches{0};
static std::mutex g_prof_mu;
static bool g_prof_on = false;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_events;  // reused across sessions
static size_t g_prof_used = 0;

void note_launches(int n) { g_launches.fetch_add((unsigned long long)n); }

void prof_begin(cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return;
  if (g_prof_used == g_prof_events.size()) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) return;
    g_prof_events.push_back({a, b});
  }
  cudaEventRecord(g_prof_events[g_prof_used].first, st);
}

void prof_end(cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on || g_prof_used == g_prof_events.size()) return;
  cudaEventRecord(g_prof_events[g_prof_used].second, st);
  ++g_prof_used;
}

// ------------------------------------------------- library-managed workspace
void* managed_workspace(size_t bytes, cudaStream_t st) {
  // One buffer per (device, stream): calls queued on one stream run in order
  // and can share it; calls on different streams may overlap on the GPU and
  // must not.
  static std::mutex mu;
  static std::map<std::pair<int, cudaStream_t>, std::pair<void*, size_t>> slots;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = slots[{dev, st}];
  if (slot.second < bytes) {
    // Allocating (and the synchronisation before freeing) would break a
    // stream capture: refuse instead.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return nullptr;
    if (slot.first) {
      cudaStreamSynchronize(st);  // the old buffer may still be in use by queued work
      cudaFree(slot.first);
      slot = {nullptr, 0};
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    slot = {p, bytes};
  }
  return slot.first;
}

}  // namespace cucosma

// ===================================================================== C ABI
using namespace cucosma;

extern "C" void cucosma_gemm_desc_init(cucosma_gemm_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->dtype = CUCOSMA_R_32F;
  d->precision = CUCOSMA_PRECISION_NATIVE;
  d->epilogue = CUCOSMA_EPILOGUE_NONE;
  d->alpha = 1.0;
  d->beta = 0.0;
}

extern "C" cucosma_status cucosma_gemm_workspace_size(const cucosma_gemm_desc* d, size_t* bytes) {
  if (!bytes) return CUCOSMA_STATUS_INVALID_VALUE;
  *bytes = 0;
  cucosma_status s = validate(d, nullptr, nullptr, nullptr);
  // validate() with null pointers reports INVALID_VALUE for missing operands;
  // only the descriptor itself matters here.
  if (s != CUCOSMA_STATUS_SUCCESS && s != CUCOSMA_STATUS_INVALID_VALUE) return s;
  if (!d || d->m < 0 || d->n < 0 || d->k < 0) return CUCOSMA_STATUS_INVALID_VALUE;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  cucosma_gemm_desc tuned;
  return workspace_size(apply_tuning(d, &tuned, di), bytes, di);
}

extern "C" cucosma_status cucosma_gemm_get_plan(const cucosma_gemm_desc* d, cucosma_plan_info* info) {
  if (!d || !info) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->m < 0 || d->n < 0 || d->k < 0) return CUCOSMA_STATUS_INVALID_VALUE;
  std::memset(info, 0, sizeof(*info));
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  cucosma_gemm_desc tuned;
  d = apply_tuning(d, &tuned, di);
  if (d->precision == CUCOSMA_PRECISION_NATIVE && plan_skinny_for(d, di->sms).kind) {
    const SkinnyPlan sp = plan_skinny_for(d, di->sms);
    info->path = 0;
    info->tile_m = sp.tile_m;
    info->tile_n = sp.tile_n;
    info->tile_k = sp.kind == 1 ? (int32_t)d->k : 256;
    info->splits = sp.splits;
    info->band = 1;
    info->slices = 1;
    info->launches = sp.splits > 1 ? 2 : 1;
    info->kchunk = sp.kind == 1 ? d->k : sp.kchunk;
    info->kpad = d->k;
    info->workspace_bytes = sp.ws_bytes;
    return CUCOSMA_STATUS_SUCCESS;
  }
  if (d->precision == CUCOSMA_PRECISION_NATIVE) {
    const NativePlan pl = plan_native(d, di->sms);
    info->path = 0;
    info->tile_m = pl.bm;
    info->tile_n = simt::BN;
    info->tile_k = simt_bk(d->dtype);
    info->splits = pl.splits;
    info->band = pl.swizzle;
    info->slices = 1;
    info->launches = pl.splits > 1 ? 2 : 1;
    info->kchunk = pl.kchunk;
    info->kpad = d->k;
    info->workspace_bytes = pl.ws_bytes;
    return CUCOSMA_STATUS_SUCCESS;
  }
  tc_plan_info(d, di, info);
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_gemm(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                       void* workspace, size_t workspace_bytes, void* stream) {
  return gemm(d, A, B, C, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

extern "C" cucosma_status cucosma_gemm_managed(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                               void* stream) {
  cucosma_status s = validate(d, A, B, C);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  size_t need = 0;
  s = cucosma_gemm_workspace_size(d, &need);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  void* ws = nullptr;
  if (need) {
    ws = managed_workspace(need, static_cast<cudaStream_t>(stream));
    if (!ws) return CUCOSMA_STATUS_ALLOC_FAILED;
  }
  return gemm(d, A, B, C, ws, need, static_cast<cudaStream_t>(stream));
}

template <typename T>
static cucosma_status plain_gemm(int dtype, int m, int n, int k, T alpha, const T* A, int lda, const T* B, int ldb,
                                 T beta, T* C, int ldc, void* stream) {
  cucosma_gemm_desc d;
  cucosma_gemm_desc_init(&d);
  d.m = m;
  d.n = n;
  d.k = k;
  d.lda = lda;
  d.ldb = ldb;
  d.ldc = ldc;
  d.dtype = dtype;
  d.alpha = alpha;
  d.beta = beta;
  return cucosma_gemm_managed(&d, A, B, C, stream);
}

extern "C" cucosma_status cucosma_sgemm(int m, int n, int k, float alpha, const float* A, int lda, const float* B,
                                        int ldb, float beta, float* C, int ldc, void* stream) {
  return plain_gemm<float>(CUCOSMA_R_32F, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}
extern "C" cucosma_status cucosma_dgemm(int m, int n, int k, double alpha, const double* A, int lda, const double* B,
                                        int ldb, double beta, double* C, int ldc, void* stream) {
  return plain_gemm<double>(CUCOSMA_R_64F, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}

extern "C" cucosma_status cucosma_device_status(int* detail) {
  if (cudaDeviceSynchronize() != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  int code = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&code, g_device_status, sizeof(int)) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (cudaMemcpyToSymbol(g_device_status, &zero, sizeof(int)) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (detail) *detail = code;
  if (code == 0) return CUCOSMA_STATUS_SUCCESS;
  return (code & 0xF00) == 0x100 ? CUCOSMA_STATUS_TIMEOUT : CUCOSMA_STATUS_INTERNAL_ERROR;
}

extern "C" cucosma_status cucosma_set_wait_timeout_ns(uint64_t ns) {
  if (ns == 0) return CUCOSMA_STATUS_INVALID_VALUE;
  g_wait_timeout_ns.store(ns);
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" const char* cucosma_get_error_string(cucosma_status s) {
  switch (s) {
    case CUCOSMA_STATUS_SUCCESS: return "success";
    case CUCOSMA_STATUS_INVALID_VALUE: return "invalid value";
    case CUCOSMA_STATUS_MISALIGNED: return "pointer or row stride not 16-byte aligned";
    case CUCOSMA_STATUS_NOT_SUPPORTED: return "not supported";
    case CUCOSMA_STATUS_WORKSPACE_TOO_SMALL: return "workspace too small";
    case CUCOSMA_STATUS_LAUNCH_FAILED: return "CUDA launch or API call failed";
    case CUCOSMA_STATUS_TIMEOUT: return "device-side wait timed out";
    case CUCOSMA_STATUS_ARCH_MISMATCH: return "device is not sm_100";
    case CUCOSMA_STATUS_ALLOC_FAILED: return "workspace allocation failed";
    case CUCOSMA_STATUS_INTERNAL_ERROR: return "internal error";
  }
  return "unknown status";
}

extern "C" int cucosma_get_version(void) { return CUCOSMA_VERSION; }

extern "C" unsigned long long cucosma_launch_count(void) { return g_launches.load(); }

extern "C" cucosma_status cucosma_profile_start(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = true;
  g_prof_used = 0;
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_profile_stop(double* total_ms, int64_t* launches) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = false;
  double tot = 0.0;
  for (size_t i = 0; i < g_prof_used; ++i) {
    if (cudaEventSynchronize(g_prof_events[i].second) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g_prof_events[i].first, g_prof_events[i].second) != cudaSuccess)
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    tot += ms;
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = (int64_t)g_prof_used;
  g_prof_used = 0;
  return CUCOSMA_STATUS_SUCCESS;
}
