// simt_gemm.cu -- native FP32 (FFMA2) and FP64 (DMMA) GEMM for sm_100a.
//
// Replaces the reference kernel cosmaSgemm_kernel (cuCOSMAV100.cuh:2505-2756)
// and its split-K reduction (cosmaSplitKReduce.cuh:20-58) with a B200 design:
//   * thread 0 streams A and B tiles with TMA into a shared memory ring
//     guarded by mbarriers (the reference double-buffers with __syncthreads
//     and register-staged loads that transpose A on the way);
//   * A tiles land row-major with a TMA swizzle (conflict-free reads);
//   * FP32 (simt_sgemm_kernel) transposes each A stage into a k-major buffer,
//     so a k-step is 4 LDS.128 feeding 32 two-lane FFMA2 (sm_100's packed
//     FP32 FMA, each lane an fmaf), 8x8 outputs a thread, two CTAs per SM;
//   * FP64 (simt_dgemm_kernel) runs on FP64 tensor-core MMAs with a 64x32
//     warp tile;
//   * 8 warps hold a 128x128 CTA tile;
//   * split-K writes raw partial tiles to a caller-provided workspace and a
//     separate kernel reduces them in ascending split order (deterministic),
//     then applies alpha/beta and the epilogue, like cosmaSplitKReduce;
//   * the block-index swizzle follows the reference's remap
//     (cuCOSMAV100.cuh:2586-2603).
#include <type_traits>

#include "simt_gemm.cuh"

namespace cucosma {

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

// FP32 kernel, CTA tile BM_ x 128 with BM_ = 128 (8 warps, 4 stages, two
// CTAs per SM) or 64 (4 warps, 3 stages, four CTAs per SM: twice the tiles
// for shapes that leave SMs idle at 128 rows).  A TMA ring of stages; every A
// stage is transposed once in shared memory into a k-major buffer (double
// buffered), so each k costs 2 LDS.128 for the 8 A values and 2 for the 8 B
// values of a thread's 8x8 tile (thread rows are two groups of 4 consecutive
// rows).  The one CTA barrier per stage that publishes the transposed tile
// also proves that every warp finished the previous stage, so thread 0
// refills that stage right after it: no empty barriers, no producer wait on
// the critical path.  128 registers a thread either way.
template <int BM_>
__global__ void __launch_bounds__(simt::SgemmShape<BM_>::kThreads, simt::SgemmShape<BM_>::kCtasPerSm)
    simt_sgemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const SimtParams p) {
  if (p.gate != nullptr && *p.gate != p.gate_value) return;  // path not chosen on the device
  using namespace simt;
  using Shape = SgemmShape<BM_>;
  constexpr int BM = BM_, STAGES = Shape::kStages, kLdT = Shape::kLdT;
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
  // transpose role (2*BM threads): thread handles row tr, k-half th (8 consecutive k)
  const int tr = tid & (BM - 1), th = tid / BM;
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

// FP64 kernel on the FP64 tensor-core MMA (mma.sync m16n8k8 .f64, the
// DMMA path: same peak as DFMA on B200, but one instruction does 32 FMAs a
// lane, so fragment loads and issue slots stop mattering).  8 warps in a 2x4
// grid, warp tile 64x32 = 4x4 MMA tiles, 64 FP64 accumulators a thread.  A
// stages (128 rows x 16 k, 128-byte rows) land with the 128-byte TMA swizzle;
// B stages (16 k x 128 n) unswizzled.  Thread 0 refills a stage two stages
// after it was consumed, so its wait on the stage's empty barrier rarely
// blocks.
namespace simt {
constexpr int kDStages = 5;
}

__device__ __forceinline__ void dmma_m16n8k8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// out[r][c], out[r][c + 1] from the raw sums v0, v1 (partial) or
// epi(alpha * v + beta * C) (final).  c is even and rows are 16-byte aligned.
__device__ __forceinline__ void store_pair(const SimtParams& p, int r, int c, double v0, double v1) {
  if (r >= p.m || c >= p.n) return;
  const bool both = c + 1 < p.n;
  if (p.partial) {
    double* w = reinterpret_cast<double*>(p.out) + (int64_t)blockIdx.z * p.ws_split_stride + (int64_t)r * p.ldo + c;
    if (both) *reinterpret_cast<double2*>(w) = make_double2(v0, v1);
    else w[0] = v0;
    return;
  }
  double* o = reinterpret_cast<double*>(p.out) + (int64_t)r * p.ldo + c;
  if (both) {
    double2 cv = make_double2(0.0, 0.0);
    if (p.beta != 0.0) cv = *reinterpret_cast<const double2*>(o);
    *reinterpret_cast<double2*>(o) = make_double2(apply_epi(combine(v0, p.alpha, p.beta, &cv.x), p.epilogue),
                                                  apply_epi(combine(v1, p.alpha, p.beta, &cv.y), p.epilogue));
  } else {
    o[0] = apply_epi(combine(v0, p.alpha, p.beta, o), p.epilogue);
  }
}

__global__ void __launch_bounds__(simt::kThreads, 1)
    simt_dgemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const SimtParams p) {
  if (p.gate != nullptr && *p.gate != p.gate_value) return;  // path not chosen on the device
  using namespace simt;
  constexpr int BK = Cfg<double>::BK;  // 16
  constexpr int S = kDStages;
  constexpr int A_STAGE = BM * BK * 8, B_STAGE = BK * BN * 8;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* As = smem;
  uint8_t* Bs = smem + S * A_STAGE;
  uint64_t* full = reinterpret_cast<uint64_t*>(Bs + S * B_STAGE);
  uint64_t* empty = full + S;

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
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kComputeWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();

  int issued = 0;
  auto produce = [&](int kb) -> bool {
    const int s = kb % S;
    if (!mbar_wait(&empty[s], ((kb / S) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) return false;
    mbar_arrive_expect_tx(&full[s], A_STAGE + B_STAGE);
    const int kx = (int)(kbeg + (int64_t)kb * BK);
    tma_load_2d(As + s * A_STAGE, &tmA, kx, m0, &full[s]);
    tma_load_2d(Bs + s * B_STAGE, &tmB, n0, kx, &full[s]);
    issued = kb + 1;
    return true;
  };
  bool ok = true;
  if (tid == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
    for (int kb = 0; kb < min(nkb, S - 2) && ok; ++kb) ok = produce(kb);
  }

  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  // A element (r, k) of a stage sits at r * 128 + (((k >> 1) ^ (r & 7)) << 4) + (k & 1) * 8;
  // every row this thread reads has r & 7 == g.
  const uint8_t* a_rows = As + (wm * 64 + g) * 128 + (t & 1) * 8;
  int a_off[2][2];  // [k-step][k = t or t + 4]
#pragma unroll
  for (int ks = 0; ks < 2; ++ks)
#pragma unroll
    for (int h = 0; h < 2; ++h) a_off[ks][h] = ((((ks * 8 + t + 4 * h) >> 1) ^ g) << 4);
  const uint8_t* b_cols = Bs + t * BN * 8 + (wn * 32 + g) * 8;

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

  for (int kb = 0; kb < nkb && ok; ++kb) {
    if (tid == 0 && kb + S - 2 < nkb) ok = produce(kb + S - 2);
    const int s = kb % S;
    if (ok) ok = mbar_wait(&full[s], (kb / S) & 1, kErrTimeoutFull, p.ctl);
    if (!ok) break;
    const uint8_t* as = a_rows + s * A_STAGE;
    const uint8_t* bs = b_cols + s * B_STAGE;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      double af[4][4], bf[4][2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const uint8_t* r0 = as + mt * 16 * 128;
        af[mt][0] = *reinterpret_cast<const double*>(r0 + a_off[ks][0]);
        af[mt][1] = *reinterpret_cast<const double*>(r0 + 8 * 128 + a_off[ks][0]);
        af[mt][2] = *reinterpret_cast<const double*>(r0 + a_off[ks][1]);
        af[mt][3] = *reinterpret_cast<const double*>(r0 + 8 * 128 + a_off[ks][1]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const uint8_t* c0 = bs + (ks * 8) * BN * 8 + nt * 64;
        bf[nt][0] = *reinterpret_cast<const double*>(c0);
        bf[nt][1] = *reinterpret_cast<const double*>(c0 + 4 * BN * 8);
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma_m16n8k8(acc[mt][nt], af[mt], bf[nt]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok) {
    // One warp's failure does not stop the others (no CTA barrier in the
    // loop); each returns after its own failed wait, thread 0 after draining.
    if (tid == 0)
      for (int kb = max(0, issued - S); kb < issued; ++kb)
        mbar_wait(&full[kb % S], (kb / S) & 1, kErrTimeoutDrain, p.ctl);
    return;
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h)
        store_pair(p, m0 + wm * 64 + mt * 16 + g + 8 * h, n0 + wn * 32 + nt * 8 + 2 * t, acc[mt][nt][2 * h],
                   acc[mt][nt][2 * h + 1]);
}

// Deterministic split-K reduction: C = epi(alpha * sum_z ws[z] + beta*C),
// z ascending, the sum accumulated in T (cosmaSplitKReduce.cuh:31-40).
template <typename T>
__global__ void splitk_reduce_kernel(const T* __restrict__ ws, int64_t split_stride, int64_t ldw, int splits, T* C,
                                     int64_t ldc, int m, int n, double alpha_d, double beta_d, int epi,
                                     const int* gate, int gate_value) {
  if (gate != nullptr && *gate != gate_value) return;  // path not chosen on the device
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
      // Splits are added in ascending order; the loads of a batch of 8 are
      // issued before its adds so that many splits do not serialise on load
      // latency.
      int z = 1;
      for (; z + 8 <= splits; z += 8) {
        V t[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) t[j] = *reinterpret_cast<const V*>(w + (int64_t)(z + j) * split_stride);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const T* pt = reinterpret_cast<const T*>(&t[j]);
#pragma unroll
          for (int e = 0; e < VEC; ++e) ps[e] += pt[e];
        }
      }
      for (; z < splits; ++z) {
        const V t = *reinterpret_cast<const V*>(w + (int64_t)z * split_stride);
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
size_t smem_bytes(int bm) {
  constexpr int BK = Cfg<T>::BK;
  if constexpr (std::is_same<T, float>::value) {
    // stages of A and B, the double-buffered k-major copy of A, full barriers
    const int stages = bm == 64 ? SgemmShape<64>::kStages : SgemmShape<128>::kStages;
    return 1024 + (size_t)stages * (bm * BK + BK * BN) * sizeof(float) + 2 * BK * (bm + 4) * sizeof(float) +
           2 * stages * sizeof(uint64_t);
  } else {
    return 1024 + kDStages * (BM * BK + BK * BN) * sizeof(T) + 2 * kDStages * sizeof(uint64_t);
  }
}

// The GEMM kernel of each arithmetic type and CTA tile height.
using GemmKernel = void (*)(const CUtensorMap, const CUtensorMap, const SimtParams);
template <typename T>
GemmKernel gemm_kernel(int bm) {
  if constexpr (std::is_same<T, float>::value) return bm == 64 ? simt_sgemm_kernel<64> : simt_sgemm_kernel<128>;
  else return simt_dgemm_kernel;
}
template <typename T>
int threads_of(int bm) {
  return std::is_same<T, float>::value ? 2 * bm : kThreads;
}

template <typename T>
cudaError_t launch_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const SimtParams& p, int bm,
                        cudaStream_t stream) {
  if (!tile_rows_supported<T>(bm)) return cudaErrorInvalidValue;
  static std::atomic<uint64_t> attr_set[2];  // devices done, per tile height (one kernel each)
  const size_t smem = smem_bytes<T>(bm);
  cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(gemm_kernel<T>(bm)), (int)smem,
                                   attr_set[bm == 64 ? 1 : 0]);
  if (e != cudaSuccess) return e;
  dim3 grid;
  if (p.swizzle > 1) {
    grid = dim3(p.tiles_n * p.swizzle, (unsigned)ceil_div(p.tiles_m, p.swizzle), p.splits);
  } else {
    grid = dim3(p.tiles_n, p.tiles_m, p.splits);
  }
  gemm_kernel<T>(bm)<<<grid, threads_of<T>(bm), smem, stream>>>(tmA, tmB, p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_reduce(const T* ws, int64_t split_stride, int64_t ldw, int splits, T* C, int64_t ldc, int m, int n,
                          double alpha, double beta, int epi, int num_sms, cudaStream_t stream, const int* gate,
                          int gate_value) {
  const int64_t work = (int64_t)m * ceil_div(n, Vec<T>::n);
  const int threads = 256;
  int64_t blocks = ceil_div(work, threads);
  blocks = std::min<int64_t>(blocks, (int64_t)num_sms * 8);
  if (blocks < 1) blocks = 1;
  splitk_reduce_kernel<T><<<(unsigned)blocks, threads, 0, stream>>>(ws, split_stride, ldw, splits, C, ldc, m, n, alpha,
                                                                    beta, epi, gate, gate_value);
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
int occupancy(int bm) {
  if (!tile_rows_supported<T>(bm)) return 0;
  const size_t smem = smem_bytes<T>(bm);
  cudaFuncSetAttribute(gemm_kernel<T>(bm), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, gemm_kernel<T>(bm), threads_of<T>(bm), smem) !=
      cudaSuccess)
    return 0;
  return blocks;
}
template int occupancy<float>(int);
template int occupancy<double>(int);

template cudaError_t launch_gemm<float>(const CUtensorMap&, const CUtensorMap&, const SimtParams&, int, cudaStream_t);
template cudaError_t launch_gemm<double>(const CUtensorMap&, const CUtensorMap&, const SimtParams&, int, cudaStream_t);
template cudaError_t launch_reduce<float>(const float*, int64_t, int64_t, int, float*, int64_t, int, int, double, double,
                                          int, int, cudaStream_t, const int*, int);
template cudaError_t launch_reduce<double>(const double*, int64_t, int64_t, int, double*, int64_t, int, int, double,
                                           double, int, int, cudaStream_t, const int*, int);
template cudaError_t launch_scale<float>(float*, int64_t, int, int, double, int, int, cudaStream_t);
template cudaError_t launch_scale<double>(double*, int64_t, int, int, double, int, int, cudaStream_t);
template size_t smem_bytes<float>(int);
template size_t smem_bytes<double>(int);

}  // namespace simt
}  // namespace cucosma
