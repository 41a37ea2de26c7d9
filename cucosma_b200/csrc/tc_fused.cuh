// tc_fused.cuh -- the tcgen05 BF16-split kernel with the split fused in.
//
// On shapes whose operands are read only a few times (large K with a small
// output, like the reference's LargeK family 256 x 256 x 1,048,576) the
// separate split pre-pass costs more than the GEMM: it reads the FP32
// operands and writes their BF16 planes, which the GEMM then reads again --
// three crossings of HBM for one.  Here the producer brings the FP32 tiles in
// with TMA and eight converter warps cut them into the BF16 planes, writing
// them straight into the shared-memory stages the MMAs read, in the swizzled
// layout TMA would have produced; the operands cross HBM once.  The planes
// are bit-identical to the pre-pass's (same split_bf16_n), and the MMA issue
// order, promotion and epilogue are those of tc_gemm_kernel, so the results
// equal the unfused kernel's bit for bit.
//
// Roles (320 threads, CTA pair): warp 0 lane 0 streams FP32 tiles into a raw
// ring (TMA, this CTA's barriers); warp 1 lane 0 of rank 0 issues the MMAs
// of both CTAs; warps 2-9 convert raw tiles into plane stages (signalling
// rank 0's full barrier, remotely from rank 1) and, between k-blocks,
// promote finished accumulator chunks into registers and run the epilogue.
// Double-buffered accumulators (NBUF >= 2) let chunk c's promotion wait until
// LAG k-blocks of chunk c+1 are converted, so the MMAs never wait for it.
// The tiles are 256 x 128 (64 promoted columns a thread beside the
// conversion's registers); the shapes this kernel is for read each operand
// about once either way.
#pragma once
#include "split_device.cuh"
#include "tc_kernel.cuh"

namespace cucosma {
namespace tc {

template <class Tr>
struct FusedCfg {
  static_assert(Tr::PAIR && !Tr::PACKED && !Tr::SPLIT && Tr::NBUF >= 2 && Tr::SWZ == 64 && Tr::EPI_WARPS == 8,
                "fused split: BF16 CTA-pair tiles with at least double-buffered accumulators");
  static constexpr int NT = Tr::NA;         // BF16 planes per operand (2 or 3)
  static constexpr int BNL = Tr::BN_LOCAL;  // B columns this CTA holds
  static_assert(BNL == 128 || BNL == 64, "B tile of 64 or 128 columns per CTA");
  static constexpr int RAW_A = 128 * 32 * 4;  // [128 rows][32 K] FP32, 128-byte swizzle
  static constexpr int RAW_B = 32 * BNL * 4;  // [32 K][BNL columns] FP32, row-major
  static constexpr int RAW_BYTES = RAW_A + RAW_B;
  static constexpr int PLANE_BYTES = Tr::STAGE_BYTES;
  static constexpr int PS = 3;  // plane stages
  static constexpr int FIXED = 1024 + Tr::STAGING_BYTES + 512;
  static constexpr int RS_FIT = (kSmemBudget - FIXED - PS * PLANE_BYTES) / RAW_BYTES;
  static constexpr int RS = RS_FIT > 4 ? 4 : RS_FIT;  // raw stages
  static_assert(RS >= 2, "raw ring");
  static constexpr int SMEM = FIXED + PS * PLANE_BYTES + RS * RAW_BYTES;
  static constexpr int LAG = PS - 1;  // k-blocks of the next chunk converted before a promotion
  static constexpr int CONV_WARPS = Tr::EPI_WARPS;
};

// One k-block: raw FP32 tiles -> NT BF16 planes of A [128][32] and of B
// [BNL][32] (K-major), in the 64-byte-swizzled layout of the MMA stages
// (16-byte chunk c of row r at c ^ ((r >> 1) & 3)).  tc = converter thread
// 0..255.  Raw A is 128-byte swizzled (chunk c of row r at c ^ (r & 7)).
template <class Tr>
__device__ __forceinline__ void convert_kblock(const uint8_t* raw, uint8_t* st, int tc) {
  using F = FusedCfg<Tr>;
  constexpr int NT = F::NT, BNL = F::BNL;
  {
    // A: row r, K half h (16 values = 4 raw chunks -> 2 plane chunks per plane)
    const int r = tc & 127, h = tc >> 7;
    const float4* src = reinterpret_cast<const float4*>(raw + r * 128);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float v[8];  // 8 values at a time: the promoted accumulators hold most registers
      const float4 q0 = src[(4 * h + 2 * half) ^ (r & 7)], q1 = src[(4 * h + 2 * half + 1) ^ (r & 7)];
      v[0] = q0.x, v[1] = q0.y, v[2] = q0.z, v[3] = q0.w, v[4] = q1.x, v[5] = q1.y, v[6] = q1.z, v[7] = q1.w;
      uint32_t pk[NT][4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        __nv_bfloat16 t0[NT], t1[NT];
        split_bf16_n<NT>(v[2 * e], t0);
        split_bf16_n<NT>(v[2 * e + 1], t1);
#pragma unroll
        for (int p = 0; p < NT; ++p) pk[p][e] = pack_bf16x2(t0[p], t1[p]);
      }
      const int chunk = (2 * h + half) ^ ((r >> 1) & 3);
#pragma unroll
      for (int p = 0; p < NT; ++p)
        *reinterpret_cast<uint4*>(st + p * Tr::A_TILE + r * 64 + chunk * 16) =
            make_uint4(pk[p][0], pk[p][1], pk[p][2], pk[p][3]);
    }
  }
  {
    // B: column c, K range (BNL = 128: 16 values, 2 chunks; 64: 8 values, 1 chunk)
    constexpr int KPER = BNL == 128 ? 16 : 8;
    const int c = tc % BNL, q = tc / BNL;
    const float* src = reinterpret_cast<const float*>(raw + F::RAW_A);
    uint8_t* bst = st + Tr::A_REGION;
#pragma unroll
    for (int half = 0; half < KPER / 8; ++half) {
      const int k0 = q * KPER + half * 8;
      uint32_t pk[NT][4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        __nv_bfloat16 t0[NT], t1[NT];
        split_bf16_n<NT>(src[(k0 + 2 * e) * BNL + c], t0);
        split_bf16_n<NT>(src[(k0 + 2 * e + 1) * BNL + c], t1);
#pragma unroll
        for (int p = 0; p < NT; ++p) pk[p][e] = pack_bf16x2(t0[p], t1[p]);
      }
      const int chunk = (k0 / 8) ^ ((c >> 1) & 3);
#pragma unroll
      for (int p = 0; p < NT; ++p)
        *reinterpret_cast<uint4*>(bst + p * Tr::B_TILE + c * 64 + chunk * 16) =
            make_uint4(pk[p][0], pk[p][1], pk[p][2], pk[p][3]);
    }
  }
}

template <class Tr>
__global__ void __maxnreg__(Tr::MAX_REGS)
    tc_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const TcParams p) {
  using F = FusedCfg<Tr>;
  constexpr int BN = Tr::BN, NACC = Tr::NACC, PS = F::PS, RS = F::RS, NBUF = Tr::NBUF, TILE_M = Tr::TILE_M;
  constexpr int A_REGION = Tr::A_REGION;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* planes = smem;
  uint8_t* raws = planes + PS * F::PLANE_BYTES;
  uint8_t* staging = raws + RS * F::RAW_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(staging + Tr::STAGING_BYTES);
  uint64_t* full = bars;             // plane stage converted (rank 0: both CTAs' converters)
  uint64_t* empty = full + PS;       // plane stage read by the MMAs (commit, both CTAs)
  uint64_t* raw_full = empty + PS;   // raw tile landed (TMA bytes)
  uint64_t* raw_empty = raw_full + RS;  // raw tile converted
  uint64_t* tfull = raw_empty + RS;
  uint64_t* tempty = tfull + 4;
  uint64_t* drain = tempty + 4;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int units = p.tiles_m * p.tiles_n * p.splits;
  const uint32_t rank = cluster_ctarank();
  const int unit0 = (int)cluster_id_x(), unit_step = (int)nclusters_x();
  const int chunk = Tr::CHUNK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < PS; ++s) {
      mbar_init(&full[s], 2 * F::CONV_WARPS);
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < RS; ++s) {
      mbar_init(&raw_full[s], 1);
      mbar_init(&raw_empty[s], F::CONV_WARPS);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 2 * Tr::EPI_WARPS);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_holder, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    // -------------------------------------------------- FP32 tile producer
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      int it = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        for (int kb = u.kb0; kb < u.kb1; ++kb, ++it) {
          const int rs = it % RS;
          if (!mbar_wait(&raw_empty[rs], ((it / RS) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) {
            ok = false;
            break;
          }
          uint8_t* r = raws + rs * F::RAW_BYTES;
          mbar_arrive_expect_tx(&raw_full[rs], F::RAW_BYTES);
          tma_load_2d(r, &tmA, kb * 32, u.tm * TILE_M + (int)rank * 128, &raw_full[rs]);
          tma_load_2d(r + F::RAW_A, &tmB, u.tn * BN + (int)rank * F::BNL, kb * 32, &raw_full[rs]);
        }
      }
      if (!ok)
        for (int j = max(0, it - RS); j < it; ++j)
          mbar_wait(&raw_full[j % RS], (j / RS) & 1, kErrTimeoutDrain, p.ctl);
    }
  } else if (warp == 1) {
    // -------------------------------------------------------- MMA issuer
    if (lane == 0 && rank == 0) {
      int it = 0, ci = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        for (int cs = u.kb0; cs < u.kb1 && ok; cs += chunk, ++ci) {
          const int ce = min(u.kb1, cs + chunk);
          const int buf = ci % NBUF;
          if (!mbar_wait(&tempty[buf], ((ci / NBUF) & 1) ^ 1, kErrTimeoutAccumFree, p.ctl)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t acc0 = tmem_base + (uint32_t)(buf * NACC * BN);
          for (int kb = cs; kb < ce; ++kb, ++it) {
            const int s = it % PS;
            if (!mbar_wait(&full[s], (it / PS) & 1, kErrTimeoutFull, p.ctl)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_base = smem_u32(planes + s * F::PLANE_BYTES);
            issue_terms<Tr>(std::make_integer_sequence<int, Tr::NT>{}, sdesc<64>(a_base), sdesc<64>(a_base + A_REGION),
                            acc0, kb != cs);
            commit_both<true>(&empty[s]);
          }
          if (!ok) break;
          commit_both<true>(&tfull[buf]);
        }
      }
      if (!ok) {
        commit_self<true>(drain);
        mbar_wait(drain, 0, kErrTimeoutDrain, p.ctl);
      }
    }
  } else {
    // ------------------------------------------ converters + epilogue
    const int tc = threadIdx.x - 64;  // 0 .. 255
    const int q = warp & 3;
    constexpr int W = Tr::COLS_PER_EW;
    const int colsub = ((warp - 2) / 4) * W;
    const uint32_t lane_base = tmem_base + ((uint32_t)(32 * q) << 16);
    uint8_t* stg = staging + (warp - 2) * Tr::STAGING_PER_WARP;
    int it = 0, ci = 0;
    bool ok = true;
    for (int unit = unit0; unit < units && ok; unit += unit_step) {
      Unit u;
      resolve_unit(p, &tmA, &tmB, unit, u);
      const int row0 = u.tm * TILE_M + (int)rank * 128 + 32 * q;
      const int col0 = u.tn * BN;
      prefetch_c_block(out_ctx(p, u), row0, col0 + colsub, W, 4, lane);
      const int kb0 = u.kb0, kb1 = u.kb1, uz = u.z;
      const int nchunks = (kb1 - kb0 + chunk - 1) / chunk;
      float master[W];
#pragma unroll
      for (int j = 0; j < W; ++j) master[j] = 0.f;
      int next = 0;  // next chunk of this unit to promote
      auto promote = [&](int c) -> bool {
        const int g = ci + c, buf = g % NBUF;
        if (!__all_sync(0xffffffffu, mbar_wait(&tfull[buf], (g / NBUF) & 1, kErrTimeoutAccum, p.ctl))) return false;
        tc_fence_after();
        Tr::accumulate(lane_base + (uint32_t)(buf * NACC * BN + colsub), master);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&tempty[buf]), 0));
        return true;
      };
      for (int kb = kb0; kb < kb1 && ok; ++kb, ++it) {
        const int local = kb - kb0;
        // chunk `next` is fully converted and LAG k-blocks of the following one too
        while (ok && next < nchunks - 1 && local >= (next + 1) * chunk + F::LAG) ok = promote(next++);
        if (!ok) break;
        const int s = it % PS, rs = it % RS;
        ok = __all_sync(0xffffffffu, mbar_wait(&empty[s], ((it / PS) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) &&
             __all_sync(0xffffffffu, mbar_wait(&raw_full[rs], (it / RS) & 1, kErrTimeoutFull, p.ctl));
        if (!ok) break;
        convert_kblock<Tr>(raws + rs * F::RAW_BYTES, planes + s * F::PLANE_BYTES, tc);
        fence_proxy_async_smem();  // the planes are read by the tensor cores (async proxy)
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&raw_empty[rs]);
          mbar_arrive_cluster(mapa_shared(smem_u32(&full[s]), 0));
        }
      }
      while (ok && next < nchunks) ok = promote(next++);
      if (!ok) break;
      resolve_unit(p, &tmA, &tmB, unit, u);  // (recomputed: fewer registers held across the k-loop)
      Tr::finish(out_ctx(p, u), master, stg, lane, row0, col0 + colsub, uz);
      ci += nchunks;
    }
  }

  tc_fence_before();
  __syncwarp();
  cluster_sync_all();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 512);
  }
}

template <class Tr>
static cudaError_t launch_fused(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p, int sms,
                                cudaStream_t st) {
  using F = FusedCfg<Tr>;
  static std::atomic<uint64_t> attr_set{0};
  cudaError_t e = debug_cuda("fused smem attribute",
                             ensure_smem_attr(reinterpret_cast<const void*>(tc_fused_kernel<Tr>), F::SMEM, attr_set));
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3(Tr::THREADS, 1, 1);
  cfg.dynamicSmemBytes = F::SMEM;
  cfg.stream = st;
  static std::atomic<int> clusters_cached[64];
  int dev = 0;
  cudaGetDevice(&dev);
  int clusters = (dev >= 0 && dev < 64) ? clusters_cached[dev].load() : 0;
  if (clusters <= 0) {
    cfg.gridDim = dim3((unsigned)(sms & ~1), 1, 1);
    if (cudaOccupancyMaxActiveClusters(&clusters, reinterpret_cast<const void*>(tc_fused_kernel<Tr>), &cfg) !=
            cudaSuccess ||
        clusters <= 0) {
      cudaGetLastError();
      clusters = sms / 2;
    }
    if (dev >= 0 && dev < 64) clusters_cached[dev].store(clusters);
  }
  const int units = p.tiles_m * p.tiles_n * p.splits;
  cfg.gridDim = dim3((unsigned)(2 * std::max(1, std::min(units, clusters))), 1, 1);
  e = debug_cuda("fused kernel launch", cudaLaunchKernelEx(&cfg, tc_fused_kernel<Tr>, a, b, p));
  if (e != cudaSuccess) return e;
  return debug_cuda("fused kernel launch (last error)", cudaGetLastError());
}

}  // namespace tc
}  // namespace cucosma
