// simt_gemm.cu -- native FP32 (FFMA) and FP64 (DFMA) GEMM for sm_100a.
//
// Replaces the reference kernel cosmaSgemm_kernel (cuCOSMAV100.cuh:2505-2756)
// and its split-K reduction (cosmaSplitKReduce.cuh:20-58) with a B200 design:
//   * thread 0 streams A and B tiles with TMA into a 4-stage shared memory
//     ring guarded by mbarriers (the reference double-buffers with
//     __syncthreads and register-staged loads that transpose A on the way);
//   * A tiles land row-major with the 64-byte TMA swizzle (conflict-free
//     16-byte reads of any row);
//   * FP64 (simt_gemm_kernel<double>) reads 2 k-values of 8 rows per step
//     straight from the swizzled tile; FP32 (simt_sgemm_kernel) first
//     transposes each A stage into a k-major buffer, so a k-step is 4 LDS.128
//     feeding 32 two-lane FFMA2 (sm_100's packed FP32 FMA, each lane an
//     fmaf), and runs two CTAs per SM at 128 registers;
//   * 8 compute warps hold a 128x128 CTA tile, 8x8 outputs per thread;
//   * split-K writes raw partial tiles to a caller-provided workspace and a
//     separate kernel reduces them in ascending split order (deterministic),
//     then applies alpha/beta and the epilogue, like cosmaSplitKReduce;
//   * the block-index swizzle follows the reference's remap
//     (cuCOSMAV100.cuh:2586-2603).
#include <type_traits>

#include "simt_gemm.cuh"

namespace cucosma {

template <typename T>
__device__ __forceinline__ void simt_store(const T (&acc)[8][8], const SimtParams& p, const int (&rows)[8], int c0);

template <typename T>
__global__ void __launch_bounds__(simt::kThreads, simt::Cfg<T>::MIN_BLOCKS)
    simt_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const SimtParams p) {
  using namespace simt;
  constexpr int BK = Cfg<T>::BK;
  constexpr int VEC = Vec<T>::n;
  using V = typename Vec<T>::type;
  // A fragments cover KV = 2 consecutive k per row (an 8-byte load for FP32,
  // 16-byte for FP64): 2 * (8 + 8) fragment registers, so FP32 fits 128
  // registers and two CTAs per SM.
  constexpr int KV = 2;
  using AV = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  constexpr int A_STAGE = BM * BK * (int)sizeof(T);
  constexpr int B_STAGE = BK * BN * (int)sizeof(T);
  constexpr int KG = BK / KV;  // k-groups per stage
  static_assert(BK * sizeof(T) == 64, "A rows are 64 bytes (64-byte swizzle span)");

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* As = smem;
  uint8_t* Bs = smem + STAGES * A_STAGE;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * (A_STAGE + B_STAGE));
  uint64_t* empty = full + STAGES;

  // Block-index remap (reference semantics, cuCOSMAV100.cuh:2586-2603).
  int tile_n, tile_m;
  if (p.swizzle > 1) {
    tile_n = blockIdx.x / p.swizzle;
    tile_m = blockIdx.y * p.swizzle + blockIdx.x % p.swizzle;
    if (tile_m >= p.tiles_m) return;
  } else {
    tile_n = blockIdx.x;
    tile_m = blockIdx.y;
  }
  const int m0 = tile_m * BM, n0 = tile_n * BN;
  const int64_t kbeg = (int64_t)blockIdx.z * p.kchunk;
  const int64_t kend = min((int64_t)p.k, kbeg + p.kchunk);
  const int nkb = kend > kbeg ? (int)ceil_div(kend - kbeg, BK) : 0;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kComputeWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();

  // Producer role (thread 0): load k-block kb into stage kb % STAGES once all
  // warps released that stage.  Returns false if the wait for it expired.
  int issued = 0;
  auto produce = [&](int kb) -> bool {
    const int s = kb % STAGES;
    const uint32_t ph = (kb / STAGES) & 1;
    if (!mbar_wait(&empty[s], ph ^ 1, kErrTimeoutEmpty, p.ctl)) return false;
    mbar_arrive_expect_tx(&full[s], A_STAGE + B_STAGE);
    const int kx = (int)(kbeg + (int64_t)kb * BK);
    tma_load_2d(As + s * A_STAGE, &tmA, kx, m0, &full[s]);
    tma_load_2d(Bs + s * B_STAGE, &tmB, n0, kx, &full[s]);
    issued = kb + 1;
    return true;
  };
  bool ok = true;
  if (threadIdx.x == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
    for (int kb = 0; kb < min(nkb, STAGES - 1) && ok; ++kb) ok = produce(kb);
  }

  // ---------------------------------------------------------------- compute
  const int wm = warp >> 1, wn = warp & 1;  // 4 x 2 warps, warp tile 32 x 64
  const int tx = lane & 7, ty = lane >> 3;  // 8 x 4 threads
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = T(0);

  // This thread's A rows are r_i = wm*32 + ty + 4i (64-byte rows, byte
  // offset a_base + 256 i); the 64-byte swizzle XORs the 16-byte chunk index
  // with (r_i >> 1) & 3, which is sw0 for even i and sw0 ^ 2 for odd i.
  const int a_base = (wm * 32 + ty) * 64;
  const int sw0 = (ty >> 1) & 3;
  constexpr int NJ = 8 / VEC;  // vectors per thread along N
  const int b_col = wn * 64 + tx * VEC;

  for (int kb = 0; kb < nkb && ok; ++kb) {
    if (threadIdx.x == 0 && kb + STAGES - 1 < nkb) ok = produce(kb + STAGES - 1);
    const int s = kb % STAGES;
    if (!mbar_wait(&full[s], (kb / STAGES) & 1, kErrTimeoutFull, p.ctl)) {
      ok = false;
      break;
    }
    const uint8_t* as = As + s * A_STAGE;
    const T* bs = reinterpret_cast<const T*>(Bs + s * B_STAGE);
#pragma unroll
    for (int kg = 0; kg < KG; ++kg) {
      // KV consecutive k of 8 A rows (one 8- or 16-byte load each) and the
      // 8 B columns of those k: KV * 64 FMAs.
      const int kb_off = kg * KV * (int)sizeof(T);  // byte offset of k-group kg inside a 64-byte row
      T a[8][KV];
      T b[KV][8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int sw = (i & 1) ? (sw0 ^ 2) : sw0;
        const AV v = *reinterpret_cast<const AV*>(as + a_base + 256 * i + ((((kb_off >> 4) ^ sw) << 4) | (kb_off & 15)));
        const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int e = 0; e < KV; ++e) a[i][e] = pv[e];
      }
#pragma unroll
      for (int kk = 0; kk < KV; ++kk) {
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const V v = *reinterpret_cast<const V*>(bs + (kg * KV + kk) * BN + b_col + j * 8 * VEC);
          const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
          for (int e = 0; e < VEC; ++e) b[kk][j * VEC + e] = pv[e];
        }
      }
#pragma unroll
      for (int kk = 0; kk < KV; ++kk)
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i][kk], b[kk][j], acc[i][j]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok) {
    // A wait expired.  Thread 0 drains (bounded) every load it issued that
    // may still be in flight, so no copy targets this CTA after it exits.
    if (threadIdx.x == 0)
      for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
        mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, kErrTimeoutDrain, p.ctl);
    return;
  }

  int rows[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) rows[i] = m0 + wm * 32 + ty + 4 * i;
  simt_store<T>(acc, p, rows, n0 + b_col);
}

// Epilogue of the SIMT kernels: this thread's 8 x 8 accumulators, rows
// rows[i], columns c0 + j*8*VEC + [0, VEC) for j < 8/VEC; either raw partial
// sums into the split-K workspace or epi(alpha*acc + beta*C) into C.
template <typename T>
__device__ __forceinline__ void simt_store(const T (&acc)[8][8], const SimtParams& p, const int (&rows)[8], int c0) {
  constexpr int VEC = Vec<T>::n;
  constexpr int NJ = 8 / VEC;
  using V = typename Vec<T>::type;
  const T alpha = (T)p.alpha, beta = (T)p.beta;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = rows[i];
    if (r >= p.m) continue;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int c = c0 + j * 8 * VEC;
      if (c >= p.n) continue;
      if (p.partial) {
        T* w = reinterpret_cast<T*>(p.out) + (int64_t)blockIdx.z * p.ws_split_stride + (int64_t)r * p.ldo + c;
        if (c + VEC <= p.n) {
          V v;
          T* pv = reinterpret_cast<T*>(&v);
#pragma unroll
          for (int e = 0; e < VEC; ++e) pv[e] = acc[i][j * VEC + e];
          *reinterpret_cast<V*>(w) = v;
        } else {
#pragma unroll
          for (int e = 0; e < VEC; ++e)
            if (c + e < p.n) w[e] = acc[i][j * VEC + e];
        }
      } else {
        T* o = reinterpret_cast<T*>(p.out) + (int64_t)r * p.ldo + c;
        if (c + VEC <= p.n) {
          V cv;
          if (beta != T(0)) cv = *reinterpret_cast<const V*>(o);
          const T* pc = reinterpret_cast<const T*>(&cv);
          V v;
          T* pv = reinterpret_cast<T*>(&v);
#pragma unroll
          for (int e = 0; e < VEC; ++e) pv[e] = apply_epi(combine(acc[i][j * VEC + e], alpha, beta, pc + e), p.epilogue);
          *reinterpret_cast<V*>(o) = v;
        } else {
#pragma unroll
          for (int e = 0; e < VEC; ++e)
            if (c + e < p.n) o[e] = apply_epi(combine(acc[i][j * VEC + e], alpha, beta, o + e), p.epilogue);
        }
      }
    }
  }
}

// FP32 kernel.  Same TMA ring as simt_gemm_kernel, but every A stage is
// transposed once in shared memory into a k-major buffer (double buffered),
// so each k costs 2 LDS.128 for the 8 A values and 2 for the 8 B values of a
// thread's 8x8 tile (thread rows are two groups of 4 consecutive rows).  The
// one CTA barrier per stage that publishes the transposed tile also proves
// that every warp finished the previous stage, so thread 0 refills that
// stage right after it: no empty barriers, no producer wait on the critical
// path.  128 registers: two CTAs per SM.
namespace simt {
constexpr int kLdT = BM + 4;  // k-major A row pitch (floats): 16-byte aligned rows
}

__global__ void __launch_bounds__(simt::kThreads, 2)
    simt_sgemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const SimtParams p) {
  using namespace simt;
  constexpr int BK = Cfg<float>::BK;  // 16
  constexpr int A_STAGE = BM * BK * 4, B_STAGE = BK * BN * 4;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* As = smem;
  uint8_t* Bs = smem + STAGES * A_STAGE;
  float* AsT = reinterpret_cast<float*>(smem + STAGES * (A_STAGE + B_STAGE));  // [2][BK][kLdT]
  uint64_t* full = reinterpret_cast<uint64_t*>(AsT + 2 * BK * kLdT);

  int tile_n, tile_m;  // block-index remap, cuCOSMAV100.cuh:2586-2603
  if (p.swizzle > 1) {
    tile_n = blockIdx.x / p.swizzle;
    tile_m = blockIdx.y * p.swizzle + blockIdx.x % p.swizzle;
    if (tile_m >= p.tiles_m) return;
  } else {
    tile_n = blockIdx.x;
    tile_m = blockIdx.y;
  }
  const int m0 = tile_m * BM, n0 = tile_n * BN;
  const int64_t kbeg = (int64_t)blockIdx.z * p.kchunk;
  const int64_t kend = min((int64_t)p.k, kbeg + p.kchunk);
  const int nkb = kend > kbeg ? (int)ceil_div(kend - kbeg, BK) : 0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Stage kb % STAGES is free: all reads of its previous use finished before
  // a CTA barrier this thread has passed.
  auto produce = [&](int kb) {
    const int s = kb % STAGES;
    mbar_arrive_expect_tx(&full[s], A_STAGE + B_STAGE);
    const int kx = (int)(kbeg + (int64_t)kb * BK);
    tma_load_2d(As + s * A_STAGE, &tmA, kx, m0, &full[s]);
    tma_load_2d(Bs + s * B_STAGE, &tmB, n0, kx, &full[s]);
  };
  if (tid == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
    for (int kb = 0; kb < min(nkb, STAGES - 1); ++kb) produce(kb);
  }
  int issued = min(nkb, STAGES - 1);  // uniform across the CTA

  const int wm = warp >> 1, wn = warp & 1;
  const int tx = lane & 7, ty = lane >> 3;
  const int a_col = wm * 32 + ty * 4;  // this thread's rows: a_col + {0..3}, a_col + 16 + {0..3}
  const int b_col = wn * 64 + tx * 4;  // columns: b_col + {0..3}, b_col + 32 + {0..3}
  // transpose role: thread handles row tr, k-half th (8 consecutive k)
  const int tr = tid & (BM - 1), th = tid >> 7;
  const int sw = (tr >> 1) & 3;  // 64-byte TMA swizzle of row tr: chunk ^ ((tr >> 1) & 3)
  const int c0 = ((2 * th) ^ sw) << 4, c1 = ((2 * th + 1) ^ sw) << 4;
  // acc[i][q]: row i, columns 2q and 2q + 1 of the thread's 8 (packed pairs
  // for the two-lane FFMA2 of sm_100: half the issue slots of scalar FFMA)
  float2 acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[i][q] = make_float2(0.f, 0.f);

  bool ok = true;
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb % STAGES;
    const bool good = mbar_wait(&full[s], (kb / STAGES) & 1, kErrTimeoutFull, p.ctl);
    float* at = AsT + (kb & 1) * BK * kLdT;
    if (good) {
      const uint8_t* arow = As + s * A_STAGE + tr * 64;
      const float4 q0 = *reinterpret_cast<const float4*>(arow + c0);
      const float4 q1 = *reinterpret_cast<const float4*>(arow + c1);
      float* col = at + th * 8 * kLdT + tr;
      col[0 * kLdT] = q0.x;
      col[1 * kLdT] = q0.y;
      col[2 * kLdT] = q0.z;
      col[3 * kLdT] = q0.w;
      col[4 * kLdT] = q1.x;
      col[5 * kLdT] = q1.y;
      col[6 * kLdT] = q1.z;
      col[7 * kLdT] = q1.w;
    }
    // Uniform across the CTA: nobody leaves the loop while others wait here.
    ok = __syncthreads_and(good);
    if (!ok) break;
    // every warp is past stage kb - 1: refill its slot
    if (kb + STAGES - 1 < nkb) {
      if (tid == 0) produce(kb + STAGES - 1);
      issued = kb + STAGES;
    }
    const float* bs = reinterpret_cast<const float*>(Bs + s * B_STAGE);
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      const float4 a0 = *reinterpret_cast<const float4*>(at + k * kLdT + a_col);
      const float4 a1 = *reinterpret_cast<const float4*>(at + k * kLdT + a_col + 16);
      const float4 b0 = *reinterpret_cast<const float4*>(bs + k * BN + b_col);
      const float4 b1 = *reinterpret_cast<const float4*>(bs + k * BN + b_col + 32);
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float2 b[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                           make_float2(b1.z, b1.w)};
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float2 ai = make_float2(a[i], a[i]);
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = __ffma2_rn(ai, b[q], acc[i][q]);  // = fmaf per lane
      }
    }
  }
  if (!ok) {
    // loads still in flight write into this CTA's shared memory: wait for them
    if (tid == 0)
      for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
        mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, kErrTimeoutDrain, p.ctl);
    return;
  }
  int rows[8];
  float out[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    rows[i] = m0 + a_col + (i & 3) + (i >> 2) * 16;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      out[i][2 * q] = acc[i][q].x;
      out[i][2 * q + 1] = acc[i][q].y;
    }
  }
  simt_store<float>(out, p, rows, n0 + b_col);
}

// Deterministic split-K reduction: C = epi(alpha * sum_z ws[z] + beta*C),
// z ascending, the sum accumulated in T (cosmaSplitKReduce.cuh:31-40).
template <typename T>
__global__ void splitk_reduce_kernel(const T* __restrict__ ws, int64_t split_stride, int64_t ldw, int splits, T* C,
                                     int64_t ldc, int m, int n, double alpha_d, double beta_d, int epi) {
  constexpr int VEC = Vec<T>::n;
  using V = typename Vec<T>::type;
  const T alpha = (T)alpha_d, beta = (T)beta_d;
  const int64_t nv = ceil_div(n, VEC);
  const int64_t total = (int64_t)m * nv;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / nv;
    const int c = (int)(idx - r * nv) * VEC;
    const T* w = ws + r * ldw + c;
    T* o = C + r * ldc + c;
    if (c + VEC <= n) {
      V s = *reinterpret_cast<const V*>(w);
      T* ps = reinterpret_cast<T*>(&s);
      for (int z = 1; z < splits; ++z) {
        const V t = *reinterpret_cast<const V*>(w + z * split_stride);
        const T* pt = reinterpret_cast<const T*>(&t);
#pragma unroll
        for (int e = 0; e < VEC; ++e) ps[e] += pt[e];
      }
      V cv;
      if (beta != T(0)) cv = *reinterpret_cast<const V*>(o);
      const T* pc = reinterpret_cast<const T*>(&cv);
#pragma unroll
      for (int e = 0; e < VEC; ++e) ps[e] = apply_epi(combine(ps[e], alpha, beta, pc + e), epi);
      *reinterpret_cast<V*>(o) = s;
    } else {
      for (int e = 0; c + e < n; ++e) {
        T s = w[e];
        for (int z = 1; z < splits; ++z) s += w[z * split_stride + e];
        o[e] = apply_epi(combine(s, alpha, beta, o + e), epi);
      }
    }
  }
}

// C = epi(beta*C) on an m x n region (alpha == 0 or k == 0: no product term).
template <typename T>
__global__ void scale_kernel(T* C, int64_t ldc, int m, int n, double beta_d, int epi) {
  const T beta = (T)beta_d;
  const int64_t total = (int64_t)m * n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / n, c = idx - r * n;
    T* o = C + r * ldc + c;
    const T v = beta != T(0) ? beta * *o : T(0);
    *o = apply_epi(v, epi);
  }
}

// ------------------------------------------------------------------- launch
namespace simt {

template <typename T>
size_t smem_bytes() {
  constexpr int BK = Cfg<T>::BK;
  // FP32 adds the double-buffered k-major copy of A (and needs no empty barriers)
  constexpr size_t transposed = std::is_same<T, float>::value ? 2 * BK * kLdT * sizeof(float) : 0;
  return 1024 + STAGES * (BM * BK + BK * BN) * sizeof(T) + transposed + 2 * STAGES * sizeof(uint64_t);
}

// The GEMM kernel of each arithmetic type.
using GemmKernel = void (*)(const CUtensorMap, const CUtensorMap, const SimtParams);
template <typename T>
GemmKernel gemm_kernel() {
  if constexpr (std::is_same<T, float>::value) return simt_sgemm_kernel;
  else return simt_gemm_kernel<T>;
}

template <typename T>
cudaError_t launch_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const SimtParams& p, cudaStream_t stream) {
  static bool attr_set = false;  // per process; the attribute is per function
  const size_t smem = smem_bytes<T>();
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(gemm_kernel<T>(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  dim3 grid;
  if (p.swizzle > 1) {
    grid = dim3(p.tiles_n * p.swizzle, (unsigned)ceil_div(p.tiles_m, p.swizzle), p.splits);
  } else {
    grid = dim3(p.tiles_n, p.tiles_m, p.splits);
  }
  gemm_kernel<T>()<<<grid, kThreads, smem, stream>>>(tmA, tmB, p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_reduce(const T* ws, int64_t split_stride, int64_t ldw, int splits, T* C, int64_t ldc, int m, int n,
                          double alpha, double beta, int epi, int num_sms, cudaStream_t stream) {
  const int64_t work = (int64_t)m * ceil_div(n, Vec<T>::n);
  const int threads = 256;
  int64_t blocks = ceil_div(work, threads);
  blocks = std::min<int64_t>(blocks, (int64_t)num_sms * 8);
  if (blocks < 1) blocks = 1;
  splitk_reduce_kernel<T><<<(unsigned)blocks, threads, 0, stream>>>(ws, split_stride, ldw, splits, C, ldc, m, n, alpha,
                                                                    beta, epi);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_scale(T* C, int64_t ldc, int m, int n, double beta, int epi, int num_sms, cudaStream_t stream) {
  const int64_t work = (int64_t)m * n;
  int64_t blocks = std::min<int64_t>(ceil_div(work, 256), (int64_t)num_sms * 8);
  if (blocks < 1) blocks = 1;
  scale_kernel<T><<<(unsigned)blocks, 256, 0, stream>>>(C, ldc, m, n, beta, epi);
  return cudaGetLastError();
}

template <typename T>
int occupancy() {
  const size_t smem = smem_bytes<T>();
  cudaFuncSetAttribute(gemm_kernel<T>(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, gemm_kernel<T>(), kThreads, smem) != cudaSuccess)
    return 0;
  return blocks;
}
template int occupancy<float>();
template int occupancy<double>();

template cudaError_t launch_gemm<float>(const CUtensorMap&, const CUtensorMap&, const SimtParams&, cudaStream_t);
template cudaError_t launch_gemm<double>(const CUtensorMap&, const CUtensorMap&, const SimtParams&, cudaStream_t);
template cudaError_t launch_reduce<float>(const float*, int64_t, int64_t, int, float*, int64_t, int, int, double, double,
                                          int, int, cudaStream_t);
template cudaError_t launch_reduce<double>(const double*, int64_t, int64_t, int, double*, int64_t, int, int, double,
                                           double, int, int, cudaStream_t);
template cudaError_t launch_scale<float>(float*, int64_t, int, int, double, int, int, cudaStream_t);
template cudaError_t launch_scale<double>(double*, int64_t, int, int, double, int, int, cudaStream_t);
template size_t smem_bytes<float>();
template size_t smem_bytes<double>();

}  // namespace simt
}  // namespace cucosma
