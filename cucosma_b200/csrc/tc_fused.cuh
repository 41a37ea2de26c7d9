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
// are bit-identical to the pre-pass's (the same round-to-nearest split), and
// the MMA issue order, promotion and epilogue are those of tc_gemm_kernel, so
// the results equal the unfused kernel's bit for bit.
//
// tc_fused_inplace_kernel: a CTA pair of 512 threads with 256 x 128 tiles
// (the shapes it is for read each operand about once either way):
//   warp 0 lane 0 streams FP32 tiles in with TMA (this CTA's barriers);
//   warp 1 lane 0 of rank 0 issues the MMAs of both CTAs; in rank 1 it
//     forwards the converters' stage completions to rank 0 (forward_planes);
//   warps 2-9 promote finished accumulator chunks into FP32 registers and
//     run the epilogue (two per TMEM lane quadrant, 64 columns each);
//   warps 10-15 cut the FP32 tiles into planes (4 warps A's 128 rows, 2
//     warps B's 64 columns) and nothing else, so the conversion never waits
//     for a promotion or an epilogue.
// The planes are written over the FP32 tile they come from, in the same
// stage (details at FusedInplaceCfg).
#pragma once
#include "split_device.cuh"
#include "tc_kernel.cuh"

namespace cucosma {
namespace tc {

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

// ---------------------------------------------------------------------------
// The split done in place.  BF16x3: each 48 KB stage receives two k-blocks
// of FP32 tiles -- A [128 rows][64 K] and B [64 K][64 columns], so every row
// request TMA makes is 256 contiguous bytes (128-byte requests cap the
// large-K stream at about 4.6 TB/s on B200, 256-byte ones reach the copy
// peak) -- and the converters overwrite it with the two k-blocks' planes (two
// BF16 planes occupy exactly the FP32 tile's bytes).  BF16x6: 36 KB stages of
// one k-block (24 KB of FP32, three planes of 36 KB).  In both, every
// converter thread first loads its values, then -- once all six warps have
// arrived on a read-done barrier -- all store.  A stage is reloaded once the
// MMAs that read its planes complete.
// STG: 32 x 32 FP32 staging blocks per epilogue warp.  1: four stages (the
// large-K shapes, whose small C leaves once); 2: three stages and the
// unfused kernels' 64-column C boxes (the C-heavy large-N shapes).
template <class Tr, int STG = 1>
struct FusedInplaceCfg {
  static_assert(Tr::PAIR && !Tr::PACKED && !Tr::SPLIT && Tr::NBUF >= 2 && Tr::SWZ == 64 && Tr::EPI_WARPS == 8 &&
                    Tr::BN_LOCAL == 64 && Tr::COLS_PER_EW == 64 && (Tr::NA == 2 || Tr::NA == 3) &&
                    Tr::CHUNK % 2 == 0,
                "in-place split: two- or three-plane 256 x 128 BF16 CTA-pair tiles");
  static constexpr int NT = Tr::NA;
  // k-blocks per stage: two for two planes (A [128 rows][64 K] and B [64 K]
  // [64 columns], no swizzle: 256-byte rows; the planes fill the FP32 bytes
  // exactly); one for three planes (A [128][32 K] with the 128-byte swizzle,
  // B [32 K][64]; the planes are 1.5x the FP32 bytes and extend the stage).
  static constexpr int KB = NT == 2 ? 2 : 1;
  static constexpr int PLANE_BYTES = Tr::STAGE_BYTES;  // one k-block's planes (NT x (A 8 KB + B 4 KB))
  static constexpr int RAW_A = 128 * 32 * KB * 4;
  static constexpr int RAW_B = 32 * KB * 64 * 4;
  static constexpr int RAW_BYTES = RAW_A + RAW_B;
  static constexpr int STAGE = RAW_BYTES > KB * PLANE_BYTES ? RAW_BYTES : KB * PLANE_BYTES;
  static_assert(STAGE % 1024 == 0 && STAGE >= RAW_BYTES && STAGE >= KB * PLANE_BYTES, "stage layout");
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
__device__ __forceinline__ bool inplace_convert_a2(uint8_t* stage, int aw, int lane, Sync&& read_done) {
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
__device__ __forceinline__ bool inplace_convert_b2(uint8_t* stage, int c, Sync&& read_done) {
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

// Three planes, one k-block a stage.  A: thread r (0..127) takes row r, 32
// values as 8 chunks of the 128-byte swizzle (chunk c at c ^ (r & 7): a
// quarter-warp reads 8 different chunks), and writes its row of the three
// planes; B: thread c (0..63) takes column c, 32 values.
template <class Tr, class Sync>
__device__ __forceinline__ bool inplace_convert_a1(uint8_t* stage, int r, Sync&& read_done) {
  const float4* src = reinterpret_cast<const float4*>(stage + r * 128);
  float4 v[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) v[c] = src[c ^ (r & 7)];
  if (!read_done()) return false;
#pragma unroll
  for (int pc = 0; pc < 4; ++pc) {
    uint32_t w[4][3];
    split_bf16x2_n<3>(v[2 * pc].x, v[2 * pc].y, w[0]);
    split_bf16x2_n<3>(v[2 * pc].z, v[2 * pc].w, w[1]);
    split_bf16x2_n<3>(v[2 * pc + 1].x, v[2 * pc + 1].y, w[2]);
    split_bf16x2_n<3>(v[2 * pc + 1].z, v[2 * pc + 1].w, w[3]);
    uint8_t* dst = stage + r * 64 + ((pc ^ ((r >> 1) & 3)) * 16);
#pragma unroll
    for (int p = 0; p < 3; ++p)
      *reinterpret_cast<uint4*>(dst + p * Tr::A_TILE) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
  }
  return true;
}
template <class Tr, class Sync>
__device__ __forceinline__ bool inplace_convert_b1(uint8_t* stage, int c, Sync&& read_done) {
  using F = FusedInplaceCfg<Tr>;
  const float* src = reinterpret_cast<const float*>(stage + F::RAW_A);
  float v[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = src[k * 64 + c];
  if (!read_done()) return false;
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    uint32_t w[4][3];
#pragma unroll
    for (int e = 0; e < 4; ++e) split_bf16x2_n<3>(v[8 * kc + 2 * e], v[8 * kc + 2 * e + 1], w[e]);
    uint8_t* dst = stage + Tr::A_REGION + c * 64 + ((kc ^ ((c >> 1) & 3)) * 16);
#pragma unroll
    for (int p = 0; p < 3; ++p)
      *reinterpret_cast<uint4*>(dst + p * Tr::B_TILE) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
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
        for (int kb = u.kb0; kb < u.kb1; kb += F::KB, ++sj) {
          const int st = sj % NS;
          if (!mbar_wait(&empty[st], ((sj / NS) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) {
            ok = false;
            break;
          }
          uint8_t* dst = stages + st * F::STAGE;
          mbar_arrive_expect_tx(&raw_full[st], F::RAW_BYTES);
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
          for (int kb = cs; kb < ce; kb += F::KB, ++sj) {
            const int st = sj % NS;
            if (!mbar_wait<true>(&full[st], (sj / NS) & 1, kErrTimeoutFull, p.ctl)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t base = smem_u32(stages + st * F::STAGE);
            issue_terms<Tr>(std::make_integer_sequence<int, Tr::NT>{}, sdesc<64>(base), sdesc<64>(base + A_REGION), acc0,
                            kb != cs);
            if (F::KB == 2 && kb + 1 < ce)
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
        for (int kb = u.kb0; kb < u.kb1 && ok; kb += F::KB, ++sj) {
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
      for (int kb = u.kb0; kb < u.kb1; kb += F::KB, ++sj) {
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
        if constexpr (F::KB == 2)
          ok = cw < 4 ? inplace_convert_a2<Tr>(stage, cw, lane, read_done)
                      : inplace_convert_b2<Tr>(stage, (cw - 4) * 32 + lane, read_done);
        else
          ok = cw < 4 ? inplace_convert_a1<Tr>(stage, cw * 32 + lane, read_done)
                      : inplace_convert_b1<Tr>(stage, (cw - 4) * 32 + lane, read_done);
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

// BF16x3: a = A [128 rows][64 K] boxes, b = B [64 K][64 columns] boxes (no swizzle);
// BF16x6: a = A [128 rows][32 K] boxes (128-byte swizzle), b = B [32 K][64 columns].
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
