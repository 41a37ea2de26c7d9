// tc_fused.cuh -- the tcgen05 BF16-split kernel with the split fused in.
//
// On shapes whose operands are read only a few times (large K with a small
// output, like the reference's LargeK family 256 x 256 x 1,048,576) the
// separate split pre-pass costs more than the GEMM: it reads the FP32
// operands and writes their BF16 planes, which the GEMM then reads again --
// three crossings of HBM for one.  Here the producer brings the FP32 tiles in
// with TMA and six converter warps cut them into the BF16 planes, writing
// them straight into the shared-memory stages the MMAs read, in the swizzled
// layout TMA would have produced; the operands cross HBM once.  The planes
// are bit-identical to the pre-pass's (same split_bf16_n), and the MMA issue
// order, promotion and epilogue are those of tc_gemm_kernel, so the results
// equal the unfused kernel's bit for bit.
//
// Two kernels, both CTA pairs of 512 threads with 256 x 128 tiles (the
// shapes they are for read each operand about once either way):
//   warp 0 lane 0 streams FP32 tiles in with TMA (this CTA's barriers);
//   warp 1 lane 0 of rank 0 issues the MMAs of both CTAs;
//   warps 2-9 promote finished accumulator chunks into FP32 registers and
//     run the epilogue (two per TMEM lane quadrant, 64 columns each);
//   warps 10-15 cut the FP32 tiles into planes (4 warps A's 128 rows, 2
//     warps B's 64 columns) and nothing else, so the conversion never waits
//     for a promotion or an epilogue.
// tc_fused_inplace_kernel (BF16x3): 48 KB stages of two k-blocks converted
// in place; rank 1's completions reach rank 0 through warp 1 lane 0 of rank
// 1 (forward_planes).  tc_fused_kernel (BF16x6, whose three planes do not
// fit in the FP32 tile): separate raw and plane rings of one k-block each;
// with G = 2 converter groups (warps 10, 11, 14 and 12, 13, 15) each group
// converts every other k-block, so two are in conversion at once and each
// warp's fixed cost per k-block (barrier waits, the async-proxy fence, the
// arrivals) covers twice the data.
#pragma once
#include "split_device.cuh"
#include "tc_kernel.cuh"

namespace cucosma {
namespace tc {

template <class Tr, int G>
struct FusedCfg {
  static_assert(Tr::PAIR && !Tr::PACKED && !Tr::SPLIT && Tr::NBUF >= 2 && Tr::SWZ == 64 && Tr::EPI_WARPS == 8 &&
                    Tr::BN_LOCAL == 64 && Tr::COLS_PER_EW == 64,
                "fused split: 256 x 128 BF16 CTA-pair tiles with at least double-buffered accumulators");
  static_assert(G == 1 || G == 2, "one or two converter groups");
  static constexpr int NT = Tr::NA;  // BF16 planes per operand (2 or 3)
  static constexpr int BNL = 64;     // B columns this CTA holds
  static constexpr int RAW_A = 128 * 32 * 4;  // [128 rows][32 K] FP32, 128-byte swizzle
  static constexpr int RAW_B = 32 * BNL * 4;  // [32 K][64 columns] FP32, row-major
  static constexpr int RAW_BYTES = RAW_A + RAW_B;
  static constexpr int PLANE_BYTES = Tr::STAGE_BYTES;
  static constexpr int ACC_WARPS = 8, CONV_WARPS = 6, CONV_WARP0 = 2 + ACC_WARPS;
  static constexpr int GROUP_WARPS = CONV_WARPS / G;
  static constexpr int A_THREADS = 128 / G, B_THREADS = 64 / G;  // per group; each thread G rows / columns
  static constexpr int THREADS = (CONV_WARP0 + CONV_WARPS) * 32;
  static constexpr int MAX_REGS = 16384 / (32 * ((THREADS / 32 + 3) / 4)) / 8 * 8;
  // Plane stages: three for two planes; two for three planes, which leaves
  // room for five raw stages (a stage is refilled as soon as the MMAs that
  // read it complete, a fraction of a k-block's conversion time).
  static constexpr int PS = NT == 2 ? 3 : 2;
  static constexpr int STAGING_PER_WARP = 32 * 32 * 4;  // one FP32 epilogue block per warp
  static constexpr int STAGING_BYTES = ACC_WARPS * STAGING_PER_WARP;
  static constexpr int FIXED = 1024 + STAGING_BYTES + 512;
  static constexpr int RS_FIT = (kSmemBudget - FIXED - PS * PLANE_BYTES) / RAW_BYTES;
  static constexpr int RS = RS_FIT > 6 ? 6 : RS_FIT;  // raw stages
  static_assert(RS >= 2 + G, "raw ring: loads in flight beside the tiles in conversion");
  static constexpr int SMEM = FIXED + PS * PLANE_BYTES + RS * RAW_BYTES;
};

// A rows of one k-block: raw [128][32] FP32 (128-byte swizzle: 16-byte chunk
// c of row r at c ^ (r & 7)) -> NT BF16 planes [128][32] in the 64-byte
// swizzle of the MMA stages (chunk c of row r at c ^ ((r >> 1) & 3)).
template <class Tr, int NT>
__device__ __forceinline__ void convert_a_row(const uint8_t* raw, uint8_t* st, int r) {
  const float4* src = reinterpret_cast<const float4*>(raw + r * 128);
#pragma unroll
  for (int pc = 0; pc < 4; ++pc) {
    const float4 q0 = src[(2 * pc) ^ (r & 7)], q1 = src[(2 * pc + 1) ^ (r & 7)];
    const float v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
    uint32_t pk[NT][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      __nv_bfloat16 t0[NT], t1[NT];
      split_bf16_n<NT>(v[2 * e], t0);
      split_bf16_n<NT>(v[2 * e + 1], t1);
#pragma unroll
      for (int p = 0; p < NT; ++p) pk[p][e] = pack_bf16x2(t0[p], t1[p]);
    }
    const int chunk = pc ^ ((r >> 1) & 3);
#pragma unroll
    for (int p = 0; p < NT; ++p)
      *reinterpret_cast<uint4*>(st + p * Tr::A_TILE + r * 64 + chunk * 16) =
          make_uint4(pk[p][0], pk[p][1], pk[p][2], pk[p][3]);
  }
}

// B column c of one k-block: raw [32 K][64] FP32 -> NT K-major BF16 planes
// [64][32], same 64-byte swizzle.
template <class Tr, int NT>
__device__ __forceinline__ void convert_b_col(const uint8_t* raw, uint8_t* st, int c) {
  const float* src = reinterpret_cast<const float*>(raw);
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    uint32_t pk[NT][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      __nv_bfloat16 t0[NT], t1[NT];
      split_bf16_n<NT>(src[(8 * kc + 2 * e) * 64 + c], t0);
      split_bf16_n<NT>(src[(8 * kc + 2 * e + 1) * 64 + c], t1);
#pragma unroll
      for (int p = 0; p < NT; ++p) pk[p][e] = pack_bf16x2(t0[p], t1[p]);
    }
    const int chunk = kc ^ ((c >> 1) & 3);
#pragma unroll
    for (int p = 0; p < NT; ++p)
      *reinterpret_cast<uint4*>(st + p * Tr::B_TILE + c * 64 + chunk * 16) =
          make_uint4(pk[p][0], pk[p][1], pk[p][2], pk[p][3]);
  }
}

// Rank 1 of a pair hands its converters' "planes written" to rank 0's full
// barrier through one thread: the converter warps arrive on a local barrier
// (release at CTA scope) and this otherwise idle thread waits for it and
// makes a single cluster-scope arrival per stage.  A release at cluster scope
// issued by a converter warp right after its plane stores measured about
// 1700 cycles on B200 -- as long as converting a whole stage -- so paying it
// in every converter warp of rank 1 made that CTA the pair's bottleneck.
__device__ __forceinline__ bool forward_planes(uint64_t* local_bar, uint32_t parity, uint32_t rank0_full,
                                               const WaitCtl& ctl) {
  if (!mbar_wait(local_bar, parity, kErrTimeoutFull, ctl)) return false;
  mbar_arrive_cluster(rank0_full);
  return true;
}

template <class Tr, int G>
__global__ void __maxnreg__((FusedCfg<Tr, G>::MAX_REGS))
    tc_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ TcParams p) {
  using F = FusedCfg<Tr, G>;
  constexpr int BN = Tr::BN, NACC = Tr::NACC, PS = F::PS, RS = F::RS, NBUF = Tr::NBUF, TILE_M = Tr::TILE_M;
  constexpr int A_REGION = Tr::A_REGION;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* planes = smem;
  uint8_t* raws = planes + PS * F::PLANE_BYTES;
  uint8_t* staging = raws + RS * F::RAW_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(staging + F::STAGING_BYTES);
  uint64_t* full = bars;                // plane stage converted (rank 0: both CTAs' converters)
  uint64_t* empty = full + PS;          // plane stage read by the MMAs (commit, both CTAs)
  uint64_t* raw_full = empty + PS;      // raw tile landed (TMA bytes)
  uint64_t* raw_empty = raw_full + RS;  // raw tile converted
  uint64_t* tfull = raw_empty + RS;
  uint64_t* tempty = tfull + 4;
  uint64_t* drain = tempty + 4;
  uint64_t* ebar = drain + 1;  // one per promotion/epilogue warp: its TMA loads of C
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(ebar + F::ACC_WARPS);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int units = p.tiles_m * p.tiles_n * p.splits;
  const uint32_t rank = cluster_ctarank();
  const int unit0 = (int)cluster_id_x(), unit_step = (int)nclusters_x();
  const int chunk = Tr::CHUNK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < PS; ++s) {
      mbar_init(&full[s], 2 * F::GROUP_WARPS);
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < RS; ++s) {
      mbar_init(&raw_full[s], 1);
      mbar_init(&raw_empty[s], F::GROUP_WARPS);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 2 * F::ACC_WARPS);
    }
    mbar_init(drain, 1);
    for (int w = 0; w < F::ACC_WARPS; ++w) mbar_init(&ebar[w], 1);
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
          if (!mbar_wait<true>(&tempty[buf], ((ci / NBUF) & 1) ^ 1, kErrTimeoutAccumFree, p.ctl)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t acc0 = tmem_base + (uint32_t)(buf * NACC * BN);
          for (int kb = cs; kb < ce; ++kb, ++it) {
            const int s = it % PS;
            if (!mbar_wait<true>(&full[s], (it / PS) & 1, kErrTimeoutFull, p.ctl)) {
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
  } else if (warp < F::CONV_WARP0) {
    // ------------------------------------------------ promotion + epilogue
    const int q = warp & 3;
    constexpr int W = Tr::COLS_PER_EW;
    const int colsub = ((warp - 2) / 4) * W;
    const uint32_t lane_base = tmem_base + ((uint32_t)(32 * q) << 16);
    uint8_t* stg = staging + (warp - 2) * F::STAGING_PER_WARP;
    const uint32_t tempty_rank0 = mapa_shared(smem_u32(&tempty[0]), 0);
    int ci = 0;
    for (int unit = unit0; unit < units; unit += unit_step) {
      Unit u;
      resolve_unit(p, &tmA, &tmB, unit, u);
      const int row0 = u.tm * TILE_M + (int)rank * 128 + 32 * q;
      const int col0 = u.tn * BN;
      // C prefetched into L2 one unit ahead (this unit's only for the first)
      auto prefetch_unit = [&](int un) {
        if (un >= units) return;
        Unit v;
        resolve_unit(p, &tmA, &tmB, un, v);
        prefetch_c_block(out_ctx(p, v), v.tm * TILE_M + (int)rank * 128 + 32 * q, v.tn * BN + colsub, W, 4, lane);
      };
      if (unit == unit0) prefetch_unit(unit);
      const int nchunks = (u.kb1 - u.kb0 + chunk - 1) / chunk;
      float master[W];
#pragma unroll
      for (int j = 0; j < W; ++j) master[j] = 0.f;
      bool ok = true;
      for (int c = 0; c < nchunks; ++c) {
        const int g = ci + c, buf = g % NBUF;
        if (!__all_sync(0xffffffffu, mbar_wait(&tfull[buf], (g / NBUF) & 1, kErrTimeoutAccum, p.ctl))) {
          ok = false;
          break;
        }
        tc_fence_after();
        Tr::accumulate(lane_base + (uint32_t)(buf * NACC * BN + colsub), master);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(tempty_rank0 + (uint32_t)(buf * sizeof(uint64_t)));
      }
      if (!ok) break;
      prefetch_unit(unit + unit_step);
      OutCtx o = out_ctx(p, u);
      o.tbar = &ebar[warp - 2];
      Tr::template finish<1>(o, master, stg, lane, row0, col0 + colsub, u.z);
      ci += nchunks;
    }
    if (lane == 0) bulk_wait_all();  // this warp's TMA stores of C have completed
  } else {
    // --------------------------------------------------------- converters
    const int cw = warp - F::CONV_WARP0;  // 0..5: A warps 0-3, B warps 4-5
    const bool is_a = cw < 4;
    const int grp = is_a ? cw / (4 / G) : (cw - 4) / (2 / G);
    const int ti = (is_a ? cw % (4 / G) : (cw - 4) % (2 / G)) * 32 + lane;  // thread within the group's A or B part
    const uint32_t full_rank0 = mapa_shared(smem_u32(&full[0]), 0);
    int it = 0;
    bool ok = true;
    for (int unit = unit0; unit < units && ok; unit += unit_step) {
      Unit u;
      resolve_unit(p, &tmA, &tmB, unit, u);
      for (int kb = u.kb0; kb < u.kb1; ++kb, ++it) {
        if (it % G != grp) continue;
        const int s = it % PS, rs = it % RS;
        ok = __all_sync(0xffffffffu, mbar_wait(&empty[s], ((it / PS) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) &&
             __all_sync(0xffffffffu, mbar_wait(&raw_full[rs], (it / RS) & 1, kErrTimeoutFull, p.ctl));
        if (!ok) break;
        const uint8_t* raw = raws + rs * F::RAW_BYTES;
        uint8_t* st = planes + s * F::PLANE_BYTES;
        if (is_a) {
#pragma unroll 1
          for (int j = 0; j < G; ++j) convert_a_row<Tr, F::NT>(raw, st, ti + j * F::A_THREADS);
        } else {
#pragma unroll 1
          for (int j = 0; j < G; ++j) convert_b_col<Tr, F::NT>(raw + F::RAW_A, st + A_REGION, ti + j * F::B_THREADS);
        }
        fence_proxy_async_smem();  // the planes are read by the tensor cores (async proxy)
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&raw_empty[rs]);
          if (rank == 0)
            mbar_arrive(&full[s]);
          else
            mbar_arrive_cluster(full_rank0 + (uint32_t)(s * sizeof(uint64_t)));
        }
      }
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

// ---------------------------------------------------------------------------
// BF16x3 with the split done in place.  Each 48 KB stage receives two
// k-blocks of FP32 tiles -- A [128 rows][64 K] and B [64 K][64 columns], so
// every row request TMA makes is 256 contiguous bytes (128-byte requests cap
// the large-K stream at about 4.6 TB/s on B200, 256-byte ones reach the
// copy peak) -- and the converters overwrite it with the two k-blocks' BF16
// planes (two planes of FP32 occupy exactly the FP32 tile's bytes): first
// every converter thread loads its 64 values, then -- once all six warps
// have arrived on a read-done barrier -- all store.  A stage is reloaded once the MMAs that read its planes complete,
// so four stages give two in flight, one in conversion and one in the MMAs.
// Roles as in tc_fused_kernel (producer, MMA issuer, 8 promotion/epilogue
// warps, 6 converter warps: 4 for A, 2 for B).
// STG: 32 x 32 FP32 staging blocks per epilogue warp.  1: four stages (the
// large-K shapes, whose small C leaves once); 2: three stages and the
// unfused kernels' 64-column C boxes (the C-heavy large-N shapes).
template <class Tr, int STG = 1>
struct FusedInplaceCfg {
  static_assert(Tr::PAIR && !Tr::PACKED && !Tr::SPLIT && Tr::NBUF >= 2 && Tr::SWZ == 64 && Tr::EPI_WARPS == 8 &&
                    Tr::BN_LOCAL == 64 && Tr::COLS_PER_EW == 64 && Tr::NA == 2 && Tr::CHUNK % 2 == 0,
                "in-place split: two-plane 256 x 128 BF16 CTA-pair tiles");
  static constexpr int PLANE_BYTES = Tr::STAGE_BYTES;  // one k-block's planes (A 2 x 8 KB, B 2 x 4 KB)
  static constexpr int RAW_A = 128 * 64 * 4;           // [128 rows][64 K] FP32, row-major
  static constexpr int RAW_B = 64 * 64 * 4;            // [64 K][64 columns] FP32, row-major
  static constexpr int STAGE = RAW_A + RAW_B;          // = 2 * PLANE_BYTES
  static_assert(STAGE == 2 * PLANE_BYTES, "two k-blocks of planes fill the FP32 stage exactly");
  static constexpr int ACC_WARPS = 8, CONV_WARPS = 6, CONV_WARP0 = 2 + ACC_WARPS;
  static constexpr int THREADS = (CONV_WARP0 + CONV_WARPS) * 32;
  static constexpr int MAX_REGS = 16384 / (32 * ((THREADS / 32 + 3) / 4)) / 8 * 8;
  static constexpr int STAGING_PER_WARP = STG * 32 * 32 * 4;
  static constexpr int STAGING_BYTES = ACC_WARPS * STAGING_PER_WARP;
  static constexpr int FIXED = 1024 + STAGING_BYTES + 512;
  static constexpr int NS_FIT = (kSmemBudget - FIXED) / STAGE;
  static constexpr int NS = NS_FIT > 6 ? 6 : NS_FIT;
  static_assert(NS >= 3, "stage ring");
  static constexpr int SMEM = FIXED + NS * STAGE;
};

// A: warp aw (0..3) converts rows 32 aw .. 32 aw + 31, two rows per step; in
// step i lane l takes row 2 (16 aw + i) + ((l >> 3) & 1), k-block l >> 4,
// FP32 chunk l & 7 (4 values): loads of 128 contiguous bytes per 8 lanes,
// 8-byte plane stores covering 128 contiguous bytes per 16 lanes -- free of
// bank conflicts both ways.
// read_done() is called between the loads and the stores (every converter
// warp's FP32 values must be read before any plane overwrites them); it
// returns false when its bounded wait gave up, and nothing is stored then.
template <class Tr, class Sync>
__device__ __forceinline__ bool inplace_convert_a(uint8_t* stage, int aw, int lane, Sync&& read_done) {
  using F = FusedInplaceCfg<Tr>;
  const int sub = lane >> 3, cj = lane & 7, h = sub >> 1;
  float4 v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int row = 2 * (16 * aw + i) + (sub & 1);
    v[i] = *reinterpret_cast<const float4*>(stage + row * 256 + (h * 8 + cj) * 16);
  }
  if (!read_done()) return false;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int row = 2 * (16 * aw + i) + (sub & 1);
    uint32_t w0[2], w1[2];
    split_bf16x2_n<2>(v[i].x, v[i].y, w0);
    split_bf16x2_n<2>(v[i].z, v[i].w, w1);
    uint8_t* dst = stage + h * F::PLANE_BYTES + row * 64 + (((cj >> 1) ^ ((row >> 1) & 3)) * 16) + (cj & 1) * 8;
#pragma unroll
    for (int p = 0; p < 2; ++p) *reinterpret_cast<uint2*>(dst + p * Tr::A_TILE) = make_uint2(w0[p], w1[p]);
  }
  return true;
}

// B: thread c (0..63) converts column c, all 64 K values (lanes read
// consecutive columns of a K row; 16-byte plane stores as in the pre-pass
// layout).
template <class Tr, class Sync>
__device__ __forceinline__ bool inplace_convert_b(uint8_t* stage, int c, Sync&& read_done) {
  using F = FusedInplaceCfg<Tr>;
  const float* src = reinterpret_cast<const float*>(stage + F::RAW_A);
  float v[64];
#pragma unroll
  for (int k = 0; k < 64; ++k) v[k] = src[k * 64 + c];
  if (!read_done()) return false;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t w[4][2];
#pragma unroll
      for (int e = 0; e < 4; ++e) split_bf16x2_n<2>(v[32 * h + 8 * kc + 2 * e], v[32 * h + 8 * kc + 2 * e + 1], w[e]);
      uint8_t* dst = stage + h * F::PLANE_BYTES + Tr::A_REGION + c * 64 + ((kc ^ ((c >> 1) & 3)) * 16);
#pragma unroll
      for (int p = 0; p < 2; ++p)
        *reinterpret_cast<uint4*>(dst + p * Tr::B_TILE) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
    }
  }
  return true;
}

template <class Tr, int STG>
__global__ void __maxnreg__((FusedInplaceCfg<Tr, STG>::MAX_REGS))
    tc_fused_inplace_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                            const __grid_constant__ TcParams p) {
  using F = FusedInplaceCfg<Tr, STG>;
  constexpr int BN = Tr::BN, NACC = Tr::NACC, NS = F::NS, NBUF = Tr::NBUF, TILE_M = Tr::TILE_M;
  constexpr int A_REGION = Tr::A_REGION;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* stages = smem;
  uint8_t* staging = stages + NS * F::STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(staging + F::STAGING_BYTES);
  uint64_t* raw_full = bars;       // FP32 tiles landed (TMA bytes)
  uint64_t* full = raw_full + NS;  // planes written (rank 0: both CTAs' converters)
  uint64_t* empty = full + NS;     // planes read by the MMAs (commit, both CTAs)
  uint64_t* tfull = empty + NS;
  uint64_t* tempty = tfull + 4;
  uint64_t* drain = tempty + 4;
  uint64_t* conv_rd = drain + 1;  // this CTA's converters have read the stage's FP32 values
  uint64_t* fwd = conv_rd + 1;    // rank 1: this CTA's converters wrote the stage (forwarded to rank 0)
  uint64_t* ebar = fwd + NS;      // STG per promotion/epilogue warp: its TMA loads of C (one per staging block)
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(ebar + STG * F::ACC_WARPS);
  static_assert((4 * NS + 10 + STG * F::ACC_WARPS) * 8 + 4 <= 512, "barrier area");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int units = p.tiles_m * p.tiles_n * p.splits;
  const uint32_t rank = cluster_ctarank();
  const int unit0 = (int)cluster_id_x(), unit_step = (int)nclusters_x();
  const int chunk = Tr::CHUNK;

  if (threadIdx.x == 0) {
    mbar_init(conv_rd, F::CONV_WARPS);
    for (int s = 0; s < NS; ++s) {
      mbar_init(&raw_full[s], 1);
      mbar_init(&full[s], F::CONV_WARPS + 1);  // rank 0's converters and rank 1's forwarder
      mbar_init(&empty[s], 1);
      mbar_init(&fwd[s], F::CONV_WARPS);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 2 * F::ACC_WARPS);
    }
    mbar_init(drain, 1);
    for (int w = 0; w < STG * F::ACC_WARPS; ++w) mbar_init(&ebar[w], 1);
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
      int sj = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        for (int kb = u.kb0; kb < u.kb1; kb += 2, ++sj) {
          const int st = sj % NS;
          if (!mbar_wait(&empty[st], ((sj / NS) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) {
            ok = false;
            break;
          }
          uint8_t* dst = stages + st * F::STAGE;
          mbar_arrive_expect_tx(&raw_full[st], F::STAGE);
          tma_load_2d(dst, &tmA, kb * 32, u.tm * TILE_M + (int)rank * 128, &raw_full[st]);
          tma_load_2d(dst + F::RAW_A, &tmB, u.tn * BN + (int)rank * 64, kb * 32, &raw_full[st]);
        }
      }
      if (!ok)
        for (int j = max(0, sj - NS); j < sj; ++j)
          mbar_wait(&raw_full[j % NS], (j / NS) & 1, kErrTimeoutDrain, p.ctl);
    }
  } else if (warp == 1) {
    // -------------------------------------------------------- MMA issuer
    if (lane == 0 && rank == 0) {
      int sj = 0, ci = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        for (int cs = u.kb0; cs < u.kb1 && ok; cs += chunk, ++ci) {
          const int ce = min(u.kb1, cs + chunk);
          const int buf = ci % NBUF;
          if (!mbar_wait<true>(&tempty[buf], ((ci / NBUF) & 1) ^ 1, kErrTimeoutAccumFree, p.ctl)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t acc0 = tmem_base + (uint32_t)(buf * NACC * BN);
          for (int kb = cs; kb < ce; kb += 2, ++sj) {
            const int st = sj % NS;
            if (!mbar_wait<true>(&full[st], (sj / NS) & 1, kErrTimeoutFull, p.ctl)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t base = smem_u32(stages + st * F::STAGE);
            issue_terms<Tr>(std::make_integer_sequence<int, Tr::NT>{}, sdesc<64>(base), sdesc<64>(base + A_REGION), acc0,
                            kb != cs);
            if (kb + 1 < ce)
              issue_terms<Tr>(std::make_integer_sequence<int, Tr::NT>{}, sdesc<64>(base + F::PLANE_BYTES),
                              sdesc<64>(base + F::PLANE_BYTES + A_REGION), acc0, true);
            commit_both<true>(&empty[st]);
          }
          if (!ok) break;
          commit_both<true>(&tfull[buf]);
        }
      }
      if (!ok) {
        commit_self<true>(drain);
        mbar_wait(drain, 0, kErrTimeoutDrain, p.ctl);
      }
    } else if (lane == 0) {
      // rank 1: forward each stage's conversion to rank 0
      const uint32_t full_rank0 = mapa_shared(smem_u32(&full[0]), 0);
      int sj = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        for (int kb = u.kb0; kb < u.kb1 && ok; kb += 2, ++sj) {
          const int st = sj % NS;
          ok = forward_planes(&fwd[st], (sj / NS) & 1, full_rank0 + (uint32_t)(st * sizeof(uint64_t)), p.ctl);
        }
      }
    }
  } else if (warp < F::CONV_WARP0) {
    // ------------------------------------------------ promotion + epilogue
    const int q = warp & 3;
    constexpr int W = Tr::COLS_PER_EW;
    const int colsub = ((warp - 2) / 4) * W;
    const uint32_t lane_base = tmem_base + ((uint32_t)(32 * q) << 16);
    uint8_t* stg = staging + (warp - 2) * F::STAGING_PER_WARP;
    const uint32_t tempty_rank0 = mapa_shared(smem_u32(&tempty[0]), 0);
    int ci = 0;
    for (int unit = unit0; unit < units; unit += unit_step) {
      Unit u;
      resolve_unit(p, &tmA, &tmB, unit, u);
      const int row0 = u.tm * TILE_M + (int)rank * 128 + 32 * q;
      const int col0 = u.tn * BN;
      // C prefetched into L2 one unit ahead (this unit's only for the first)
      auto prefetch_unit = [&](int un) {
        if (un >= units) return;
        Unit v;
        resolve_unit(p, &tmA, &tmB, un, v);
        prefetch_c_block(out_ctx(p, v), v.tm * TILE_M + (int)rank * 128 + 32 * q, v.tn * BN + colsub, W, 4, lane);
      };
      if (unit == unit0) prefetch_unit(unit);
      const int nchunks = (u.kb1 - u.kb0 + chunk - 1) / chunk;
      float master[W];
#pragma unroll
      for (int j = 0; j < W; ++j) master[j] = 0.f;
      bool ok = true;
      for (int c = 0; c < nchunks; ++c) {
        const int g = ci + c, buf = g % NBUF;
        if (!__all_sync(0xffffffffu, mbar_wait(&tfull[buf], (g / NBUF) & 1, kErrTimeoutAccum, p.ctl))) {
          ok = false;
          break;
        }
        tc_fence_after();
        Tr::accumulate(lane_base + (uint32_t)(buf * NACC * BN + colsub), master);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(tempty_rank0 + (uint32_t)(buf * sizeof(uint64_t)));
      }
      if (!ok) break;
      prefetch_unit(unit + unit_step);
      OutCtx o = out_ctx(p, u);
      o.tbar = &ebar[STG * (warp - 2)];  // the epilogue uses tbar[0 .. STG-1]
      Tr::template finish<STG>(o, master, stg, lane, row0, col0 + colsub, u.z);
      ci += nchunks;
    }
    if (lane == 0) bulk_wait_all();  // this warp's TMA stores of C have completed
  } else {
    // --------------------------------------------------------- converters
    // conv_rd completes once per stage, in stage order (a warp arrives for
    // stage j only after it saw the completion for stage j - 1).
    const int cw = warp - F::CONV_WARP0;
    int sj = 0;
    bool ok = true;
    for (int unit = unit0; unit < units && ok; unit += unit_step) {
      Unit u;
      resolve_unit(p, &tmA, &tmB, unit, u);
      for (int kb = u.kb0; kb < u.kb1; kb += 2, ++sj) {
        const int st = sj % NS;
        uint8_t* stage = stages + st * F::STAGE;
        ok = __all_sync(0xffffffffu, mbar_wait(&raw_full[st], (sj / NS) & 1, kErrTimeoutFull, p.ctl));
        if (!ok) break;
        const uint32_t par = (uint32_t)sj & 1;
        auto read_done = [&]() -> bool {
          __syncwarp();
          if (lane == 0) mbar_arrive(conv_rd);
          return __all_sync(0xffffffffu, mbar_wait(conv_rd, par, kErrTimeoutFull, p.ctl));
        };
        ok = cw < 4 ? inplace_convert_a<Tr>(stage, cw, lane, read_done)
                    : inplace_convert_b<Tr>(stage, (cw - 4) * 32 + lane, read_done);
        if (!ok) break;
        fence_proxy_async_smem();  // the planes are read by the tensor cores (async proxy)
        __syncwarp();
        if (lane == 0) mbar_arrive(rank == 0 ? &full[st] : &fwd[st]);
      }
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

// One persistent launch of a fused kernel: CTA pairs, as many as fit at
// once (cached per device) and no more than the units.
template <class K>
static cudaError_t launch_fused_kernel(K kernel, int threads, int smem, std::atomic<uint64_t>& attr_set,
                                       std::atomic<int>* clusters_cached, const CUtensorMap& a, const CUtensorMap& b,
                                       const TcParams& p, int sms, cudaStream_t st) {
  cudaError_t e =
      debug_cuda("fused smem attribute", ensure_smem_attr(reinterpret_cast<const void*>(kernel), smem, attr_set));
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3((unsigned)threads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  int dev = 0;
  cudaGetDevice(&dev);
  int clusters = (dev >= 0 && dev < 64) ? clusters_cached[dev].load() : 0;
  if (clusters <= 0) {
    cfg.gridDim = dim3((unsigned)(sms & ~1), 1, 1);
    if (cudaOccupancyMaxActiveClusters(&clusters, reinterpret_cast<const void*>(kernel), &cfg) != cudaSuccess ||
        clusters <= 0) {
      cudaGetLastError();
      clusters = sms / 2;
    }
    if (dev >= 0 && dev < 64) clusters_cached[dev].store(clusters);
  }
  const int units = p.tiles_m * p.tiles_n * p.splits;
  cfg.gridDim = dim3((unsigned)(2 * std::max(1, std::min(units, clusters))), 1, 1);
  e = debug_cuda("fused kernel launch", cudaLaunchKernelEx(&cfg, kernel, a, b, p));
  if (e != cudaSuccess) return e;
  return debug_cuda("fused kernel launch (last error)", cudaGetLastError());
}

// a: A [rows][32 K] boxes (128-byte swizzle), b: B [32 K][64 columns] boxes.
template <class Tr, int G = 2>
static cudaError_t launch_fused(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p, int sms,
                                cudaStream_t st) {
  using F = FusedCfg<Tr, G>;
  static std::atomic<uint64_t> attr_set{0};
  static std::atomic<int> clusters_cached[64];
  return launch_fused_kernel(tc_fused_kernel<Tr, G>, F::THREADS, F::SMEM, attr_set, clusters_cached, a, b, p, sms, st);
}

// a: A [128 rows][64 K] boxes, b: B [64 K][64 columns] boxes (no swizzle).
template <class Tr, int STG>
static cudaError_t launch_fused_inplace(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p, int sms,
                                        cudaStream_t st) {
  using F = FusedInplaceCfg<Tr, STG>;
  static std::atomic<uint64_t> attr_set{0};
  static std::atomic<int> clusters_cached[64];
  return launch_fused_kernel(tc_fused_inplace_kernel<Tr, STG>, F::THREADS, F::SMEM, attr_set, clusters_cached, a, b, p,
                             sms, st);
}

}  // namespace tc
}  // namespace cucosma
