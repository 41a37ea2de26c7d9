// tc_kernel.cuh -- the tcgen05 kernel template, its epilogues and the
// traits of every precision path (included by tc_gemm.cu and grouped.cu).
//
//
// One persistent, warp-specialised kernel template serves both precision
// forms that have no counterpart in the reference (which is FP32 SIMT only,
// cuCOSMAV100.cuh:2505-2756):
//
//   BF16x3 / BF16x6 SGEMM   A = sum_i A_i, B = sum_j B_j (BF16 split planes);
//                           C ~= sum over the kept (i, j) of A_i * B_j, all
//                           products accumulated in one FP32 TMEM accumulator.
//   Ozaki DGEMM (INT8)      A_p, B_q signed 7-bit slices; for every diagonal
//                           d = p + q < s an exact INT32 TMEM accumulator
//                           S_d = sum_{p+q=d} A_p * B_q; the epilogue
//                           recombines sum_d S_d 2^(-7(d+2)) in FP64 (d
//                           descending) and rescales by 2^(e_row + e_col).
//
// Roles (192 threads): warp 0 lane 0 streams the slice planes of A and B
// with 3-D TMA loads (all planes of one k-block in one box) into a
// multi-stage shared-memory ring; warp 1 allocates TMEM and one lane issues
// tcgen05.mma (A and B from shared memory, K-major, swizzled) and commits to
// mbarriers; warps 2-5 drain the accumulators (tcgen05.ld), apply
// alpha/beta and the fused epilogue and store through a shared-memory
// transpose for coalesced rows.  Accumulators are double-buffered in TMEM
// when they fit, so the epilogue of one tile overlaps the next tile's MMAs.
// Work units (tile x K split) are distributed round-robin over a persistent
// grid with a banded raster (the reference's block swizzle,
// cuCOSMAV100.cuh:2586-2603, generalised).  Split-K writes raw partials to
// the workspace and a separate kernel reduces them in split order.
//
// Every mbarrier wait is bounded (ptx.cuh); on expiry the roles leave their
// loops, drain what they issued, and TMEM is released before exit.
#pragma once
#include <type_traits>
#include <cuda_bf16.h>

#include <utility>

#include "api_internal.cuh"
#include "tc_gemm.cuh"

namespace cucosma {
namespace tc {

// Shared-memory matrix descriptor, K-major operand written by TMA with a
// swizzle span of SWZ bytes per row: start >> 4 at [0,14), leading byte
// offset (unused for swizzled K-major) at [16,30), stride byte offset
// (8 rows x SWZ) >> 4 at [32,46), version 1 at [46,48), layout type at
// [61,64): 2 = 128B, 4 = 64B, 6 = 32B swizzle.
template <int SWZ>
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  constexpr uint64_t layout = SWZ == 128 ? 2 : (SWZ == 64 ? 4 : 6);
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)((8 * SWZ) >> 4) << 32) |
         ((uint64_t)1 << 46) | (layout << 61);
}

__device__ __forceinline__ void unit_coords(int unit, int tiles, int tiles_m, int tiles_n, int band, int& z, int& tm,
                                            int& tn) {
  z = unit / tiles;
  const int t = unit - z * tiles;
  const int per_band = band * tiles_n;
  const int b = t / per_band;
  const int w = t - b * per_band;
  const int rows = min(band, tiles_m - b * band);
  tm = b * band + w % rows;
  tn = w / rows;
}

// Unit -> (operand descriptors, tile, K range).  Single problem: banded
// raster over tiles x K splits.  Grouped: the problem owning the unit is
// found by binary search over the tile_start column of the problem table;
// its tiles are visited down M first, then across N.
__device__ __forceinline__ void resolve_unit(const TcParams& p, const CUtensorMap* tmA, const CUtensorMap* tmB,
                                             int unit, Unit& u) {
  if (p.ngroups == 0) {
    unit_coords(unit, p.tiles_m * p.tiles_n, p.tiles_m, p.tiles_n, p.band, u.z, u.tm, u.tn);
    u.kb0 = u.z * p.kb_per_split;
    u.kb1 = min(p.kblocks, u.kb0 + p.kb_per_split);
    u.ta = tmA;
    u.tb = tmB;
    u.group = -1;
  } else {
    int lo = 0, hi = p.ngroups - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.groups[mid].tile_start <= unit)
        lo = mid;
      else
        hi = mid - 1;
    }
    const GroupEntry& e = p.groups[lo];
    const int local = unit - e.tile_start;
    u.tm = local % e.tiles_m;
    u.tn = local / e.tiles_m;
    u.z = 0;
    u.kb0 = 0;
    u.kb1 = e.kblocks;
    u.ta = &e.tmA;
    u.tb = &e.tmB;
    u.group = lo;
  }
}

// With beta != 0: L2 prefetch of the C block an epilogue warp will read
// (rows row0 + [0, 32), columns col0 + [0, cols) of es-byte elements), issued
// before the warp waits for the tile's accumulators so that the reads find
// C in L2 instead of paying HBM latency inside the epilogue.  Every address
// stays inside the m x n region (the last line of a row is clamped to its
// last element).
__device__ __forceinline__ void prefetch_c_block(const OutCtx& o, int row0, int col0, int cols, int es, int lane) {
  if (o.partial || o.beta == 0.0 || col0 >= o.n) return;
  if (o.tmc != nullptr) {
    // the TMA epilogue's boxes, prefetched by the async proxy (the
    // epilogue's own proxy fences then have no prefetches of their own to
    // wait for)
    if (lane == 0)
      for (int c = col0; c < col0 + cols && c < o.n; c += 64) tma_prefetch_2d(o.tmc_pf, c, row0);
    return;
  }
  const int c1 = min(o.n, col0 + cols);
  const int lines = ((c1 - col0) * es + 127) / 128 + 1;  // rows need not start on a line
  const char* base = static_cast<const char*>(o.out);
  for (int i = lane; i < 32 * lines; i += 32) {
    const int r = i / lines, l = i - r * lines;
    const int row = row0 + r;
    if (row >= o.m) continue;
    const char* rowp = base + (int64_t)row * o.ldo * es;
    const int64_t off = min((int64_t)col0 * es + (int64_t)l * 128, (int64_t)(c1 - 1) * es);
    prefetch_l2(rowp + off);
  }
}

__device__ __forceinline__ OutCtx out_ctx(const TcParams& p, const Unit& u) {
  OutCtx o;
  o.epilogue = p.epilogue;
  o.alpha = p.alpha;
  o.beta = p.beta;
  o.ctl = p.ctl;
  o.tbar = nullptr;
  o.stg_blocks = 1;
  o.tmc = (u.group < 0 && p.tma_out && !p.partial) ? &p.tmc : nullptr;
  o.tmc_pf = &p.tmc_pf;
  o.tmc3 = (o.tmc != nullptr && p.tma_wide) ? &p.tmc3 : nullptr;
  if (u.group < 0) {
    o.m = p.m;
    o.n = p.n;
    o.partial = p.partial;
    o.out = p.out;
    o.ldo = p.ldo;
    o.ws_split_stride = p.ws_split_stride;
    o.ea = p.ea;
    o.eb = p.eb;
  } else {
    const GroupEntry& e = p.groups[u.group];
    o.m = e.m;
    o.n = e.n;
    o.partial = 0;
    o.out = e.C;
    o.ldo = e.ldc;
    o.ws_split_stride = 0;
    o.ea = e.ea;
    o.eb = e.eb;
  }
  return o;
}

// Issues the MMAs of term T for one stage.  Descriptor start addresses
// advance by compile-time offsets (>> 4, no carry out of the 14-bit field
// since every operand lies inside shared memory).
template <class Tr, int T>
__device__ __forceinline__ void issue_term(uint64_t ad0, uint64_t bd0, uint32_t acc0, bool not_first_kb) {
  constexpr int KSTEPS = Tr::KSTEPS;
  constexpr int PA = Tr::kTerms.a[T], PB = Tr::kTerms.b[T], D = Tr::kTerms.d[T];
  constexpr bool FIRST = Tr::kTerms.first[T];
  constexpr uint32_t IDESC = Tr::kInt8 ? idesc_s8_s32(Tr::TILE_M, Tr::BN) : idesc_bf16_f32(Tr::TILE_M, Tr::BN);
#pragma unroll
  for (int kk = 0; kk < KSTEPS; ++kk) {
    const uint64_t ad = ad0 + (uint64_t)(Tr::a_off(PA, kk) >> 4);
    const uint64_t bd = bd0 + (uint64_t)(Tr::b_off(PB, kk) >> 4);
    const bool acc = (FIRST && kk == 0) ? not_first_kb : true;
    if constexpr (Tr::kInt8) {
      if constexpr (Tr::PAIR)
        mma_i8_pair(acc0 + (uint32_t)(D * Tr::BN), ad, bd, IDESC, acc);
      else
        mma_i8(acc0 + (uint32_t)(D * Tr::BN), ad, bd, IDESC, acc);
    } else {
      if constexpr (Tr::PAIR)
        mma_bf16_pair(acc0 + (uint32_t)(D * Tr::BN), ad, bd, IDESC, acc);
      else
        mma_bf16(acc0 + (uint32_t)(D * Tr::BN), ad, bd, IDESC, acc);
    }
  }
}
template <class Tr, int... Ts>
__device__ __forceinline__ void issue_terms(std::integer_sequence<int, Ts...>, uint64_t ad0, uint64_t bd0, uint32_t acc0,
                                            bool not_first_kb) {
  (issue_term<Tr, Ts>(ad0, bd0, acc0, not_first_kb), ...);
}

// Stacked Ozaki form: for sub-tile J and A slice P, one MMA of N = (S - P) *
// SUB columns whose B operand is the stacked slices 0 .. S-1-P of the
// sub-tile (rows (q, column)), accumulating A_P * B_q into the diagonal
// block d = P + q at TMEM column (J * S + P + q) * SUB.  P = 0 spans every
// diagonal, so on a unit's first k-block it initialises the accumulators
// (accumulate = 0) before the narrower MMAs of P > 0 add to them.
template <class Tr, int J, int P>
__device__ __forceinline__ void issue_stacked_one(uint64_t ad0, uint32_t b_base, uint32_t acc0, bool not_first_kb) {
  constexpr int S = Tr::NA, SUB = Tr::SUB;
  constexpr uint32_t IDESC = idesc_s8_s32(128, (S - P) * SUB);
  const uint64_t ad = ad0 + (uint64_t)(Tr::a_off(P, 0) >> 4);
  const uint64_t bd = sdesc<32>(b_base + (uint32_t)(J * Tr::B_SUB_BYTES));
  mma_i8(acc0 + (uint32_t)((J * S + P) * SUB), ad, bd, IDESC, P > 0 || not_first_kb);
}
// Issue order: A slice major (p = 0, 1, ...), sub-tiles inner, so the two
// MMAs that read the same A slice are adjacent (measured 6 % faster than
// sub-tile major); within each sub-tile p still ascends.
template <class Tr, int... Is>
__device__ __forceinline__ void issue_stacked(std::integer_sequence<int, Is...>, uint64_t ad0, uint32_t b_base,
                                              uint32_t acc0, bool not_first_kb) {
  (issue_stacked_one<Tr, Is % Tr::NSUB, Is / Tr::NSUB>(ad0, b_base, acc0, not_first_kb), ...);
}

// Commit helpers: in a CTA pair the MMAs are issued by rank 0 for both CTAs
// and their completion is signalled on the barrier at the same offset in
// both CTAs (mask 0b11), or in rank 0 only (mask 0b01).
template <bool PAIR>
__device__ __forceinline__ void commit_both(uint64_t* bar) {
  if constexpr (PAIR)
    mma_commit_pair_mc(bar, 3);
  else
    mma_commit(bar);
}
template <bool PAIR>
__device__ __forceinline__ void commit_self(uint64_t* bar) {
  if constexpr (PAIR)
    mma_commit_pair_mc(bar, 1);
  else
    mma_commit(bar);
}

// Register cap: what one CTA per SM can give each thread (see MAX_REGS).
template <class Tr>
__global__ void __maxnreg__(Tr::MAX_REGS)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ TcParams p) {
  constexpr int BN = Tr::BN, SWZ = Tr::SWZ, NA = Tr::NA, NB = Tr::NB, NACC = Tr::NACC, ST = Tr::STAGES;
  constexpr int A_REGION = Tr::A_REGION;
  constexpr int STAGE_BYTES = Tr::STAGE_BYTES;
  constexpr int NBUF = Tr::NBUF;
  constexpr bool PAIR = Tr::PAIR;
  constexpr int TILE_M = Tr::TILE_M;

  // Not the path chosen on the device: every CTA (both of a pair) leaves
  // before touching barriers or TMEM.
  if (p.gate != nullptr && *p.gate != p.gate_value) return;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* stages = smem;
  uint8_t* staging = smem + ST * STAGE_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(staging + Tr::STAGING_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + ST;
  uint64_t* tfull = bars + 2 * ST;
  uint64_t* tempty = tfull + 4;
  uint64_t* drain = tempty + 4;
  uint64_t* ebar = drain + 1;  // two per epilogue warp: its TMA loads of C (one per staging block)
  uint64_t* tfwd = ebar + 2 * Tr::EPI_WARPS;  // pair, rank 1: its epilogue released accumulator b (forwarded)
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(tfwd + 4);
  static_assert(NBUF <= 4, "accumulator buffers");
  static_assert((2 * ST + 13 + 2 * Tr::EPI_WARPS) * 8 + 4 <= 512, "barrier area");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int units = p.ngroups > 0 ? p.total_tiles : p.tiles_m * p.tiles_n * p.splits;
  // CTA pair: rank 0 issues the MMAs of both CTAs; the pair (cluster) walks
  // the units together.  Single CTA: rank 0, one CTA per unit.
  const uint32_t rank = PAIR ? cluster_ctarank() : 0u;
  const int unit0 = PAIR ? (int)cluster_id_x() : (int)blockIdx.x;
  const int unit_step = PAIR ? (int)nclusters_x() : (int)gridDim.x;
  // K-blocks per accumulator chunk: with promotion the tensor cores
  // accumulate CHUNK k-blocks in TMEM and the epilogue warps add each chunk
  // into FP32 registers (round to nearest); otherwise one chunk per unit.
  const int chunk = Tr::PROMOTE ? Tr::CHUNK : (1 << 30);

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&tfull[b], 1);
      // rank 0's: released by its epilogue warps and, in a pair, by rank 1's forwarder
      mbar_init(&tempty[b], Tr::EPI_WARPS + (PAIR ? 1 : 0));
      mbar_init(&tfwd[b], Tr::EPI_WARPS);
    }
    mbar_init(drain, 1);
    for (int w = 0; w < 2 * Tr::EPI_WARPS; ++w) mbar_init(&ebar[w], 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    if constexpr (PAIR) {
      tmem_alloc_pair(tmem_holder, 512);
      tmem_relinquish_pair();
    } else {
      tmem_alloc(tmem_holder, 512);
      tmem_relinquish();
    }
  }
  tc_fence_before();
  if constexpr (PAIR)
    cluster_sync_all();  // both CTAs' barriers initialised before any remote arrive or load
  else
    __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      if (p.ngroups == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
      }
      int it = 0;  // global k-block counter (ring position)
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        const int tm = u.tm, tn = u.tn;
        for (int kb = u.kb0; kb < u.kb1; ++kb, ++it) {
          const int s = it % ST;
          if (!mbar_wait(&empty[s], ((it / ST) & 1) ^ 1, kErrTimeoutEmpty, p.ctl)) {
            ok = false;
            break;
          }
          uint8_t* st = stages + s * STAGE_BYTES;
          if (it == p.skip_stage) continue;  // test hook: this stage is never filled
          if constexpr (PAIR) {
            // Both CTAs' bytes complete on rank 0's full barrier; only rank 0 arrives.
            if (rank == 0) mbar_arrive_expect_tx(&full[s], 2 * STAGE_BYTES);
            const uint32_t bar0 = mapa_shared(smem_u32(&full[s]), 0);
            tma_load_3d_pair(st, u.ta, kb * Tr::BK, tm * TILE_M + (int)rank * 128, 0, bar0);
            tma_load_3d_pair(st + A_REGION, u.tb, kb * Tr::BK, tn * BN + (int)rank * Tr::BN_LOCAL, 0, bar0);
            continue;
          }
          mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
          if constexpr (Tr::PACKED) {
            // boxes of [rows][128 B]: slices 4j..4j+3 of k-block kb
#pragma unroll
            for (int j = 0; j < Tr::TILES_A; ++j) tma_load_3d(st + j * Tr::A_TILE, u.ta, j * 128, kb, tm * 128, &full[s]);
            if constexpr (Tr::STACKED) {
              // per sub-tile one box [slices][SUB columns][32 B] of k-block kb
              const int zs = p.b_layout_slices > 0 ? p.b_layout_slices : NB;  // slices per k-block in memory
#pragma unroll
              for (int j = 0; j < Tr::NSUB; ++j)
                tma_load_3d(st + A_REGION + j * Tr::B_SUB_BYTES, u.tb, 0, tn * BN + j * Tr::SUB, kb * zs, &full[s]);
            } else {
#pragma unroll
              for (int j = 0; j < Tr::TILES_B; ++j)
                tma_load_3d(st + A_REGION + j * Tr::B_TILE, u.tb, j * 128, kb, tn * BN, &full[s]);
            }
          } else {
            // one box of [planes][rows][BK] per operand
            tma_load_3d(st, u.ta, kb * Tr::BK, tm * 128, 0, &full[s]);
            tma_load_3d(st + A_REGION, u.tb, kb * Tr::BK, tn * BN, 0, &full[s]);
          }
        }
      }
      // Drain loads that may still be in flight (bounded).  In a pair, rank
      // 0's full barriers count both CTAs' bytes.
      if (!ok && rank == 0)
        for (int j = max(0, it - ST); j < it; ++j) mbar_wait(&full[j % ST], (j / ST) & 1, kErrTimeoutDrain, p.ctl);
    }
  } else if (warp == 1) {
    // -------------------------------------------------------- MMA issuer
    if (lane == 0 && rank == 0) {
      int it = 0, ci = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        const int kb1 = u.kb1;
        for (int cs = u.kb0; cs < kb1 && ok; cs += chunk, ++ci) {
          const int ce = min(kb1, cs + chunk);
          const int buf = ci % NBUF;
          if (!Tr::SPLIT && !mbar_wait<PAIR>(&tempty[buf], ((ci / NBUF) & 1) ^ 1, kErrTimeoutAccumFree, p.ctl)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t acc0 = tmem_base + (uint32_t)(buf * NACC * BN);
          for (int kb = cs; kb < ce; ++kb, ++it) {
            const int s = it % ST;
            if (!mbar_wait(&full[s], (it / ST) & 1, kErrTimeoutFull, p.ctl)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_base = smem_u32(stages + s * STAGE_BYTES);
            const uint64_t ad0 = sdesc<SWZ>(a_base);
            if constexpr (Tr::SPLIT) {
              // corrections (terms 0 .. NT-2, accumulator 1) once that
              // accumulator is drained, then the main term (accumulator 0)
              const uint64_t bd0 = sdesc<SWZ>(a_base + A_REGION);
              if (kb == cs && !mbar_wait<PAIR>(&tempty[1], (ci & 1) ^ 1, kErrTimeoutAccumFree, p.ctl)) {
                ok = false;
                break;
              }
              tc_fence_after();
              issue_terms<Tr>(std::make_integer_sequence<int, Tr::NT - 1>{}, ad0, bd0, acc0, kb != cs);
              if (kb == cs && !mbar_wait<PAIR>(&tempty[0], (ci & 1) ^ 1, kErrTimeoutAccumFree, p.ctl)) {
                ok = false;
                break;
              }
              tc_fence_after();
              issue_term<Tr, Tr::NT - 1>(ad0, bd0, acc0, kb != cs);
            } else if constexpr (Tr::STACKED) {
              issue_stacked<Tr>(std::make_integer_sequence<int, Tr::NSUB * NA>{}, ad0, a_base + A_REGION, acc0,
                                kb != cs);
            } else {
              const uint64_t bd0 = sdesc<SWZ>(a_base + A_REGION);
              issue_terms<Tr>(std::make_integer_sequence<int, Tr::NT>{}, ad0, bd0, acc0, kb != cs);
            }
            commit_both<PAIR>(&empty[s]);  // stage free (in both CTAs) once these MMAs have read it
          }
          if (!ok) break;
          commit_both<PAIR>(&tfull[buf]);  // accumulator ready once every MMA above completes
        }
      }
      if (!ok) {
        commit_self<PAIR>(drain);  // wait (bounded) for every MMA issued so far
        mbar_wait(drain, 0, kErrTimeoutDrain, p.ctl);
      }
    } else if (PAIR && lane == 0) {
      // Rank 1: forward each accumulator release of this CTA's epilogue
      // warps to rank 0 with one cluster-scope arrival (a release at cluster
      // scope costs a warp about 1700 cycles on B200; paid here, once, off
      // the epilogue warps' path).  Same release sequence as the epilogue.
      const uint32_t tempty0 = mapa_shared(smem_u32(&tempty[0]), 0);
      auto forward = [&](int idx, uint32_t parity) {
        if (!mbar_wait(&tfwd[idx], parity, kErrTimeoutAccum, p.ctl)) return false;
        mbar_arrive_cluster(tempty0 + (uint32_t)(idx * sizeof(uint64_t)));
        return true;
      };
      int ci = 0;
      bool ok = true;
      for (int unit = unit0; unit < units && ok; unit += unit_step) {
        Unit u;
        resolve_unit(p, &tmA, &tmB, unit, u);
        if constexpr (Tr::PROMOTE) {
          for (int cs = u.kb0; cs < u.kb1 && ok; cs += chunk, ++ci) {
            if constexpr (Tr::SPLIT)
              ok = forward(1, ci & 1) && forward(0, ci & 1);
            else
              ok = forward(ci % NBUF, (ci / NBUF) & 1);
          }
        } else {
          ok = forward(ci % NBUF, (ci / NBUF) & 1);
          ++ci;
        }
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    // Epilogue warp ew: TMEM lane quadrant warp % 4 (the only lanes a warp may
    // access) and, with 8 epilogue warps, one half of the tile's columns.
    // In a pair each CTA drains its own 128 rows of the 256-row tile.
    const int q = warp & 3;
    constexpr int W = Tr::COLS_PER_EW;
    const int colsub = ((warp - 2) / 4) * W;
    const uint32_t lane_base = tmem_base + ((uint32_t)(32 * q) << 16);
    uint8_t* stg = staging + (warp - 2) * Tr::STAGING_PER_WARP;
    // Releasing an accumulator: arrive on tempty[idx] (rank 0), or on the
    // local tfwd[idx] that rank 1's forwarder hands on to rank 0.
    auto release = [&](int idx) {
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(rank == 0 ? &tempty[idx] : &tfwd[idx]);
    };
    int ci = 0;
    bool ok = true;
    for (int unit = unit0; unit < units && ok; unit += unit_step) {
      Unit u;
      resolve_unit(p, &tmA, &tmB, unit, u);
      const int z = u.z;
      const int row0 = u.tm * TILE_M + (int)rank * 128 + 32 * q;
      const int col0 = u.tn * BN;
      // C blocks are prefetched into L2 one unit ahead: this unit's (first
      // unit only) and, before this unit's epilogue reads its C, the next's.
      auto prefetch_unit = [&](int un) {
        if (un >= units) return;
        Unit v;
        resolve_unit(p, &tmA, &tmB, un, v);
        prefetch_c_block(out_ctx(p, v), v.tm * TILE_M + (int)rank * 128 + 32 * q,
                         v.tn * BN + (Tr::PROMOTE ? colsub : 0), Tr::PROMOTE ? W : BN, Tr::kInt8 ? 8 : 4, lane);
      };
      if (unit == unit0) prefetch_unit(unit);
      // the output context is built where it is used (fewer registers held across the chunk loop)
      auto octx = [&]() {
        OutCtx o = out_ctx(p, u);
        o.tbar = &ebar[2 * (warp - 2)];
        o.stg_blocks = Tr::STAGING_PER_WARP / (32 * 32 * 4);
        return o;
      };
      if constexpr (Tr::PROMOTE) {
        float master[W];
#pragma unroll
        for (int j = 0; j < W; ++j) master[j] = 0.f;
        for (int cs = u.kb0; cs < u.kb1; cs += chunk, ++ci) {
          const int buf = ci % NBUF;
          ok = __all_sync(0xffffffffu, mbar_wait(&tfull[buf], (ci / NBUF) & 1, kErrTimeoutAccum, p.ctl));
          if (!ok) break;
          tc_fence_after();
          if constexpr (Tr::SPLIT) {
            const uint32_t t = lane_base + (uint32_t)colsub;
            Tr::accumulate_one(t, 1, master);  // corrections first: their MMAs resume first
            release(1);
            Tr::accumulate_one(t, 0, master);
            release(0);
          } else {
            Tr::accumulate(lane_base + (uint32_t)(buf * NACC * BN + colsub), master);
            release(buf);
          }
        }
        if (!ok) break;
        prefetch_unit(unit + unit_step);
        Tr::finish(octx(), master, stg, lane, row0, col0 + colsub, z);
      } else {
        const int buf = ci % NBUF;
        ok = __all_sync(0xffffffffu, mbar_wait(&tfull[buf], (ci / NBUF) & 1, kErrTimeoutAccum, p.ctl));
        if (!ok) break;
        tc_fence_after();
        prefetch_unit(unit + unit_step);
        if constexpr (Tr::kDrain) {
          Tr::drain(lane_base + (uint32_t)(buf * NACC * BN), stg, lane);
          release(buf);  // the next unit's MMAs run during the stores below
          Tr::store(octx(), stg, lane, row0, col0, z);
        } else {
          Tr::epilogue(octx(), lane_base + (uint32_t)(buf * NACC * BN), stg, lane, row0, col0, z);
          release(buf);
        }
        ++ci;
      }
    }
    if (lane == 0) bulk_wait_all();  // this warp's TMA stores of C have completed
  }

  tc_fence_before();
  __syncwarp();
  if constexpr (PAIR)
    cluster_sync_all();  // neither CTA leaves while the other may still signal its barriers
  else
    __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    if constexpr (PAIR)
      tmem_dealloc_pair(tmem_base, 512);
    else
      tmem_dealloc(tmem_base, 512);
  }
}

// ------------------------------------------------------------ epilogues
// FP32 result (BF16 split paths).  Each warp owns 32 rows; chunks of 32
// columns go TMEM -> registers -> padded shared tile -> coalesced rows.
struct EpiF32 {
  static constexpr bool kDrain = false;
  // A 32 x 32 FP32 block per warp: row r's 16-byte chunk c at c ^ (r & 7)
  // (the 128-byte swizzle TMA uses; the buffer is 1024-byte aligned).  Rows
  // are read and written as float4 chunks by the lane owning the row, and
  // columns one float per lane -- both free of bank conflicts.
  static constexpr int STAGING_PER_WARP = 2 * 32 * 32 * 4;  // two blocks: C loads overlap the previous block
  // Columns c0 .. c0 + 31 of a register accumulator row, as a 32-array (c0
  // is a compile-time constant at every use, so no copy is made).
  template <int BN>
  static __device__ __forceinline__ const float (&cols32(const float (&m)[BN], int c0))[32] {
    return *reinterpret_cast<const float(*)[32]>(&m[c0]);
  }
  static __device__ __forceinline__ int sw(int r, int c) { return r * 32 + ((((c >> 2) ^ (r & 7))) << 2) + (c & 3); }

  // This lane's row of the block: epi(alpha * acc + beta * C) with C read
  // from (and the result written back to) the swizzled staging row s4.
  template <int EPI>
  static __device__ __forceinline__ void combine_row_t(float4* s4, const float (&acc)[32], float alpha, float beta,
                                                       int lane) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int pos = c ^ (lane & 7);
      const float4 cv = beta != 0.f ? s4[pos] : make_float4(0.f, 0.f, 0.f, 0.f);
      float4 r;
      r.x = epi_t<EPI>(combine(acc[4 * c], alpha, beta, &cv.x));
      r.y = epi_t<EPI>(combine(acc[4 * c + 1], alpha, beta, &cv.y));
      r.z = epi_t<EPI>(combine(acc[4 * c + 2], alpha, beta, &cv.z));
      r.w = epi_t<EPI>(combine(acc[4 * c + 3], alpha, beta, &cv.w));
      s4[pos] = r;
    }
  }
  static __device__ __forceinline__ void combine_row(int epi, float4* s4, const float (&acc)[32], float alpha,
                                                     float beta, int lane) {
    if (epi == kEpiSigmoid)
      combine_row_t<kEpiSigmoid>(s4, acc, alpha, beta, lane);
    else if (epi == kEpiRelu)
      combine_row_t<kEpiRelu>(s4, acc, alpha, beta, lane);
    else
      combine_row_t<kEpiNone>(s4, acc, alpha, beta, lane);
  }

  // Write one 32 x 32 block of results: acc[j] is this lane's row (row0 +
  // lane) at column col + j.
  //  * store_block_tma (p.tmc set): lane 0 waits until the previous block's store has read
  //    the buffer, brings the C block in (beta != 0; out-of-range rows and
  //    columns read as zero), every lane combines its row in place, and lane
  //    0 stores the block (out-of-range parts are not written) -- a handful
  //    of instructions per element, no predicates, C moved as whole boxes.
  //  * store_block (split-K partials, grouped problems, unaligned C): C is
  //    fetched by cp.async (lanes = columns, all rows in flight; C was
  //    prefetched into L2), combined per row, and stored as 128-byte rows;
  //    partials are stored raw.
  static __device__ __forceinline__ void store_block_tma(const OutCtx& p, const float (&acc)[32], float* stg, int lane,
                                                         int row0, int col) {
    if (col >= p.n) return;  // the whole block lies right of C (col is the block's first column)
    const float alpha = (float)p.alpha, beta = (float)p.beta;
    float4* s4 = reinterpret_cast<float4*>(stg) + lane * 8;  // this lane's row
    {
      if (lane == 0) bulk_wait_read_all();
      __syncwarp();
      if (beta != 0.f) {
        if (lane == 0) {
          const uint64_t token = mbar_arrive_expect_tx_token(p.tbar, 32 * 32 * 4);
          tma_load_2d(stg, p.tmc, col, row0, p.tbar);
          if (!mbar_wait_token(p.tbar, token, kErrTimeoutOutput, p.ctl))
            mbar_wait_token(p.tbar, token, kErrTimeoutDrain, p.ctl);  // once more before the buffer is reused
        }
        __syncwarp();
      }
      combine_row(p.epilogue, s4, acc, alpha, beta, lane);
      fence_proxy_async_smem();  // the block is read by TMA (async proxy)
      __syncwarp();
      if (lane == 0) {
        tma_store_2d(p.tmc, stg, col, row0);
        bulk_commit();
      }
    }
  }

  static __device__ __forceinline__ void store_block(const OutCtx& p, float* o, const float (&acc)[32], float* stg,
                                                     int lane, int row0, int col) {
    if (col >= p.n) return;  // the whole block lies right of C (col is the block's first column)
    const float alpha = (float)p.alpha, beta = (float)p.beta;
    float4* s4 = reinterpret_cast<float4*>(stg) + lane * 8;  // this lane's row
    const int cl = col + lane;  // this lane's column in the store pass
    if (p.partial) {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        s4[c ^ (lane & 7)] = make_float4(acc[4 * c], acc[4 * c + 1], acc[4 * c + 2], acc[4 * c + 3]);
    } else {
      if (beta != 0.f) {
#pragma unroll 4
        for (int r = 0; r < 32; ++r) {
          const int row = row0 + r;
          if (row < p.m && cl < p.n)
            cp_async4(&stg[sw(r, lane)], o + (int64_t)row * p.ldo + cl);
          else
            stg[sw(r, lane)] = 0.f;
        }
        cp_async_wait_all();
        __syncwarp();
      }
      combine_row(p.epilogue, s4, acc, alpha, beta, lane);
    }
    __syncwarp();
    if (cl < p.n) {
      float* w = o + cl;
      const int64_t ld = p.ldo;
#pragma unroll 4
      for (int r = 0; r < 32; ++r) {
        const int row = row0 + r;
        if (row < p.m) w[(int64_t)row * ld] = stg[sw(r, lane)];
      }
    }
    __syncwarp();
  }

  template <int BN>
  static __device__ __forceinline__ void run(const OutCtx& p, uint32_t tacc, uint8_t* stg_raw, int lane, int row0,
                                             int col0, int z) {
    float* stg = reinterpret_cast<float*>(stg_raw);
    float* o = reinterpret_cast<float*>(p.out) + (p.partial ? (int64_t)z * p.ws_split_stride : 0);
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v0[16], v1[16];
      tmem_ld16(tacc + c0, v0);
      tmem_ld16(tacc + c0 + 16, v1);
      tmem_ld_wait();
      float acc[32];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        acc[j] = __uint_as_float(v0[j]);
        acc[16 + j] = __uint_as_float(v1[j]);
      }
      if (p.tmc != nullptr)
        store_block_tma(p, acc, stg, lane, row0, col0 + c0);
      else
        store_block(p, o, acc, stg, lane, row0, col0 + c0);
    }
  }

  // Promotion: add one chunk's TMEM accumulators (this thread's row, BN
  // columns each; the correction products' accumulator NACC-1 first, the
  // main product's accumulator 0 last) into the FP32 register accumulator,
  // rounding to nearest.
  // W columns of this warp (from tacc); accumulators STRIDE columns apart.
  // With 128 register accumulators a thread loads 16 columns at a time (the
  // loads of one chunk are off the MMA's critical path), otherwise 32.
  template <int W, int STRIDE, int NACC>
  static __device__ __forceinline__ void accumulate(uint32_t tacc, float (&master)[W]) {
#pragma unroll
    for (int d = NACC - 1; d >= 0; --d) {
      if constexpr (W > 64) {
#pragma unroll
        for (int c0 = 0; c0 < W; c0 += 16) {
          uint32_t v0[16];
          tmem_ld16(tacc + d * STRIDE + c0, v0);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 16; ++j) master[c0 + j] = __fadd_rn(master[c0 + j], __uint_as_float(v0[j]));
        }
      } else {
#pragma unroll
        for (int c0 = 0; c0 < W; c0 += 32) {
          uint32_t v0[16], v1[16];
          tmem_ld16(tacc + d * STRIDE + c0, v0);
          tmem_ld16(tacc + d * STRIDE + c0 + 16, v1);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            master[c0 + j] = __fadd_rn(master[c0 + j], __uint_as_float(v0[j]));
            master[c0 + 16 + j] = __fadd_rn(master[c0 + 16 + j], __uint_as_float(v1[j]));
          }
        }
      }
    }
  }

  // TMA path with two staging blocks: block i + 1's C load is in flight
  // while block i is combined and stored (each buffer is reloaded once the
  // store issued from it two blocks earlier has read it).
  template <int BN>
  static __device__ __forceinline__ void finish_tma2(const OutCtx& p, const float (&master)[BN], float* stg, int lane,
                                                     int row0, int col0) {
    const float alpha = (float)p.alpha, beta = (float)p.beta;
    const bool ld = beta != 0.f;
    if (lane == 0) bulk_wait_read_all();  // the previous tile's stores have read both blocks
    __syncwarp();
    uint64_t tok[2] = {0, 0};
    if (ld && lane == 0 && col0 < p.n) {
      tok[0] = mbar_arrive_expect_tx_token(&p.tbar[0], 32 * 32 * 4);
      tma_load_2d(stg, p.tmc, col0, row0, &p.tbar[0]);
    }
#pragma unroll
    for (int i = 0; i < BN / 32; ++i) {
      const int col = col0 + 32 * i;
      if (col >= p.n) break;
      float* b = stg + (i & 1) * (32 * 32);
      if (ld) {
        if (lane == 0 && !mbar_wait_token(&p.tbar[i & 1], tok[i & 1], kErrTimeoutOutput, p.ctl))
          mbar_wait_token(&p.tbar[i & 1], tok[i & 1], kErrTimeoutDrain, p.ctl);
        __syncwarp();
      } else if (i >= 2) {
        if (lane == 0) bulk_wait_read_but_last();  // the store from this block two steps ago has read it
        __syncwarp();
      }
      combine_row(p.epilogue, reinterpret_cast<float4*>(b) + lane * 8, cols32(master, 32 * i), alpha, beta, lane);
      fence_proxy_async_smem();  // the block is read by TMA (async proxy)
      __syncwarp();
      if (lane == 0) {
        tma_store_2d(p.tmc, b, col, row0);
        bulk_commit();
        if (ld && i + 1 < BN / 32 && col + 32 < p.n) {
          bulk_wait_read_but_last();  // the other block's previous store has read it
          float* nb = stg + ((i + 1) & 1) * (32 * 32);
          tok[(i + 1) & 1] = mbar_arrive_expect_tx_token(&p.tbar[(i + 1) & 1], 32 * 32 * 4);
          tma_load_2d(nb, p.tmc, col + 32, row0, &p.tbar[(i + 1) & 1]);
        }
      }
    }
  }

  // 64-column blocks through the 3-D map: one 8 KB staging block [32 rows]
  // [2 chunks][32] (line 2r + h of row r, chunk h, 128-byte swizzle), one box
  // load of C (beta != 0) and one box store per block, 256-byte rows each.
  template <int BN>
  static __device__ __forceinline__ void finish_tma_wide(const OutCtx& p, const float (&master)[BN], float* stg,
                                                         int lane, int row0, int col0) {
    const float alpha = (float)p.alpha, beta = (float)p.beta;
    float4* s4 = reinterpret_cast<float4*>(stg);
    const uint64_t pol = l2_evict_first_policy();
#pragma unroll
    for (int i = 0; i < BN / 64; ++i) {
      const int col = col0 + 64 * i;
      if (col >= p.n) break;
      if (lane == 0) bulk_wait_read_all();  // the previous block's store has read the buffer
      __syncwarp();
      if (beta != 0.f) {
        if (lane == 0) {
          const uint64_t token = mbar_arrive_expect_tx_token(&p.tbar[0], 2 * 32 * 32 * 4);
          tma_load_3d_hint(stg, p.tmc3, 0, col / 32, row0, &p.tbar[0], pol);
          if (!mbar_wait_token(&p.tbar[0], token, kErrTimeoutOutput, p.ctl))
            mbar_wait_token(&p.tbar[0], token, kErrTimeoutDrain, p.ctl);
        }
        __syncwarp();
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int line = 2 * lane + h;
        combine_row(p.epilogue, s4 + line * 8, cols32(master, 64 * i + 32 * h), alpha, beta, line);
      }
      fence_proxy_async_smem();  // the block is read by TMA (async proxy)
      __syncwarp();
      if (lane == 0) {
        tma_store_3d_hint(p.tmc3, stg, 0, col / 32, row0, pol);
        bulk_commit();
      }
    }
  }

  // STG: 32 x 32 staging blocks the warp has (2 in tc_gemm_kernel, 1 in the
  // fused kernels), fixed at compile time so only the matching paths exist.
  template <int BN, int STG>
  static __device__ __forceinline__ void finish(const OutCtx& p, const float (&master)[BN], uint8_t* stg_raw,
                                                int lane, int row0, int col0, int z) {
    float* stg = reinterpret_cast<float*>(stg_raw);
    if (p.tmc != nullptr) {
      if constexpr (STG >= 2) {
        if (p.tmc3 != nullptr && BN % 64 == 0)
          finish_tma_wide<BN>(p, master, stg, lane, row0, col0);
        else
          finish_tma2<BN>(p, master, stg, lane, row0, col0);
        return;
      }
#pragma unroll
      for (int c0 = 0; c0 < BN; c0 += 32) {
        float acc[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = master[c0 + j];
        store_block_tma(p, acc, stg, lane, row0, col0 + c0);
      }
      return;
    }
    float* o = reinterpret_cast<float*>(p.out) + (p.partial ? (int64_t)z * p.ws_split_stride : 0);
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float acc[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] = master[c0 + j];
      store_block(p, o, acc, stg, lane, row0, col0 + c0);
    }
  }
};

// FP64 result (Ozaki).  Chunks of 16 columns: part = sum_{d = S-1..0}
// S_d * 2^(-7(d+2)) (FP64, d descending), then 2^(e_row + e_col) and
// alpha/beta; or the raw part into the split-K workspace.  Accumulator
// layout: sub-tiles of SUB columns, each S diagonal blocks of SUB columns.
template <int S, int SUB>
struct EpiOzaki {
  // Two-phase form (kDrain): the warp first drains its 32 rows x BN of the
  // accumulator into a padded shared tile (LD doubles a row) and releases
  // TMEM, so that the next unit's MMAs overlap the C combine and stores.  The
  // accumulator fills all 512 TMEM columns (one buffer), so without this the
  // MMA warp waits for the whole epilogue.  S = 5 and 9 keep the one-phase
  // form: their stages are larger and the tile would leave two ring stages.
  static constexpr bool kDrain = S != 5 && S != 9;
  static constexpr int LD = ozaki_bn(S) + 1;  // (LD * 2) % 32 == 2: conflict-free row writes
  static constexpr int STAGING_PER_WARP = kDrain ? 32 * LD * 8 : 32 * 17 * 8;

  // part[j] = sum_d S_d 2^(-7(d+2)) for this lane's row at column c0 + j of
  // the tile, d descending; two diagonals' TMEM loads share one wait.
  static __device__ __forceinline__ void recombine(uint32_t tacc, int c0, double (&part)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j) part[j] = 0.0;
    const uint32_t base = tacc + (uint32_t)((c0 / SUB) * S * SUB + c0 % SUB);
#pragma unroll
    for (int d = S - 1; d >= 0; d -= 2) {
      uint32_t v[16], u[16];
      tmem_ld16(base + (uint32_t)(d * SUB), v);
      if (d >= 1) tmem_ld16(base + (uint32_t)((d - 1) * SUB), u);
      tmem_ld_wait();
      const double w = ldexp(1.0, -7 * (d + 2));
#pragma unroll
      for (int j = 0; j < 16; ++j) part[j] = part[j] + (double)(int32_t)v[j] * w;
      if (d >= 1) {
        const double w1 = ldexp(1.0, -7 * (d + 1));
#pragma unroll
        for (int j = 0; j < 16; ++j) part[j] = part[j] + (double)(int32_t)u[j] * w1;
      }
    }
  }

  // One 16-column block of results: lane (cl = lane % 16, rows (lane >> 4) + 2h)
  // takes its 16 values from the shared tile at stg[r * ld + cl] and writes
  // them (scaled by 2^(e_row + e_col), alpha / beta, activation) or, for a
  // split-K unit, the raw parts into the workspace.
  static __device__ __forceinline__ void store_block(const OutCtx& p, const double* stg, int ld, int lane, int row0,
                                                     int col, int z) {
    if (col >= p.n) return;
    const int ecol = p.partial ? 0 : p.eb[col];
    // This lane's row exponents and, when beta != 0, its C values, read
    // together up front (the stores below may alias them, so they are not
    // reordered otherwise): one read latency a block instead of one a row.
    int erow[16];
    double cv[16];
#pragma unroll
    for (int h = 0; h < 16; ++h) {
      const int row = row0 + (lane >> 4) + 2 * h;
      const bool in = !p.partial && row < p.m;
      erow[h] = in ? p.ea[row] : 0;
      cv[h] = in && p.beta != 0.0 ? reinterpret_cast<const double*>(p.out)[(int64_t)row * p.ldo + col] : 0.0;
    }
#pragma unroll
    for (int h = 0; h < 16; ++h) {
      const int r = (lane >> 4) + 2 * h;
      const int row = row0 + r;
      if (row >= p.m) continue;
      const double v = stg[r * ld + (lane & 15)];
      if (p.partial) {
        reinterpret_cast<double*>(p.out)[(int64_t)z * p.ws_split_stride + (int64_t)row * p.ldo + col] = v;
      } else {
        double* po = reinterpret_cast<double*>(p.out) + (int64_t)row * p.ldo + col;
        const double r_ = ldexp(v, erow[h] + ecol);
        const double o = p.beta == 0.0 ? p.alpha * r_ : fma(p.alpha, r_, p.beta * cv[h]);
        *po = apply_epi(o, p.epilogue);
      }
    }
  }

  // Phase 1 of the two-phase form: TMEM -> shared tile (row lane, LD doubles a row).
  template <int BN>
  static __device__ __forceinline__ void drain(uint32_t tacc, uint8_t* stg_raw, int lane) {
    static_assert(!kDrain || BN + 1 == LD, "tile width");
    double* row = reinterpret_cast<double*>(stg_raw) + lane * LD;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      double part[16];
      recombine(tacc, c0, part);
#pragma unroll
      for (int j = 0; j < 16; ++j) row[c0 + j] = part[j];
    }
    __syncwarp();
  }

  // Phase 2: shared tile -> C (or the split-K workspace).
  template <int BN>
  static __device__ __forceinline__ void store(const OutCtx& p, const uint8_t* stg_raw, int lane, int row0, int col0,
                                               int z) {
    const double* stg = reinterpret_cast<const double*>(stg_raw);
#pragma unroll 1
    for (int c0 = 0; c0 < BN && col0 + c0 < p.n; c0 += 16)
      store_block(p, stg + c0, LD, lane, row0, col0 + c0 + (lane & 15), z);
    __syncwarp();  // the next unit's drain overwrites the tile
  }

  // One-phase form: per 16-column block, TMEM -> padded 32 x 17 block -> C.
  template <int BN>
  static __device__ __forceinline__ void run(const OutCtx& p, uint32_t tacc, uint8_t* stg_raw, int lane, int row0,
                                             int col0, int z) {
    double* stg = reinterpret_cast<double*>(stg_raw);
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      double part[16];
      recombine(tacc, c0, part);
#pragma unroll
      for (int j = 0; j < 16; ++j) stg[lane * 17 + j] = part[j];
      __syncwarp();
      store_block(p, stg, 17, lane, row0, col0 + c0 + (lane & 15), z);
      __syncwarp();
    }
  }
};

// ------------------------------------------------------------- traits
constexpr int kSmemBudget = 227 * 1024;

// Stage layout.  Unpacked (BF16 planes): one tile of rows x SWZ bytes per
// plane, KSTEPS MMAs of 32 bytes of K each per plane pair.  Packed (Ozaki
// INT8 slices): one stage is one 32-wide k-block; four slices share each
// 128-byte swizzled row, so slice p sits in tile p / 4 at byte offset
// (p % 4) * 32 -- selected like a K offset inside the swizzle atom.
template <int NT_, int BN_, int SWZ_, int NA_, int NB_, int NACC_, bool INT8_, class Epi, bool PROMOTE_ = false,
          int CHUNK_ = 0, int EPI_WARPS_ = 4, int SUB_ = 0, bool PAIR_ = false, bool SPLIT_ = false>
struct TraitsBase {
  static constexpr int NT = NT_, BN = BN_, SWZ = SWZ_, NA = NA_, NB = NB_, NACC = NACC_;
  static constexpr bool kInt8 = INT8_;
  // PAIR: a CTA pair (cluster of 2) computes a 256 x BN tile with
  // cta_group::2 MMAs (M = 256); each CTA loads its 128 rows of A and BN / 2
  // columns of B and holds its 128 rows x BN of the accumulator in its TMEM.
  static constexpr bool PAIR = PAIR_;
  static constexpr int TILE_M = PAIR_ ? 256 : 128;
  static constexpr int BN_LOCAL = PAIR_ ? BN_ / 2 : BN_;
  // SUB > 0: stacked Ozaki form -- B slices of each SUB-column sub-tile
  // stacked along N (one [NB][SUB][32 B] box, 32-byte swizzle), NSUB
  // sub-tiles per tile, NACC = NB diagonal blocks per sub-tile.
  static constexpr int SUB = SUB_;
  static constexpr bool STACKED = SUB_ > 0;
  static constexpr int NSUB = STACKED ? BN_ / SUB_ : 1;
  static constexpr int B_SUB_BYTES = STACKED ? NB_ * SUB_ * 32 : 0;
  static constexpr bool PROMOTE = PROMOTE_;
  static constexpr int CHUNK = CHUNK_;
  // SPLIT: two promoted accumulators (corrections NACC-1 = 1, main 0) in one
  // TMEM buffer, released separately: the epilogue drains the corrections
  // first and frees them, so the next chunk's correction MMAs (issued first
  // in every k-block) overlap the drain of the main accumulator.
  static constexpr bool SPLIT = SPLIT_;
  // 4 epilogue warps (one per TMEM lane quadrant) or 8 (each quadrant
  // split into two column halves, so promoted register accumulators fit).
  static constexpr int EPI_WARPS = EPI_WARPS_;
  static constexpr int THREADS = (2 + EPI_WARPS) * 32;
  // Registers a thread may hold: each of the SM's four sub-partitions has
  // 16384 registers for the warps placed on it (ceil(warps / 4) of them).
  static constexpr int WARPS_PER_SMSP = (THREADS / 32 + 3) / 4;
  static constexpr int MAX_REGS = (16384 / (32 * WARPS_PER_SMSP)) / 8 * 8 > 255 ? 255
                                                                               : (16384 / (32 * WARPS_PER_SMSP)) / 8 * 8;
  static constexpr int COLS_PER_EW = BN / (EPI_WARPS / 4);
  static_assert(EPI_WARPS == 4 || (EPI_WARPS == 8 && PROMOTE_), "8 epilogue warps only for promotion");
  static constexpr bool PACKED = INT8_;
  static constexpr int BK = PACKED ? 32 : SWZ / 2;  // K elements per stage
  static constexpr int KSTEPS = PACKED ? 1 : SWZ / 32;
  static constexpr int TILES_A = PACKED ? (NA + 3) / 4 : NA;  // TMA boxes per operand per stage
  static constexpr int TILES_B = PACKED ? (NB + 3) / 4 : NB;
  static constexpr int A_TILE = 128 * SWZ, B_TILE = BN_LOCAL * SWZ;
  static constexpr int A_REGION = TILES_A * A_TILE;
  static constexpr __host__ __device__ int a_off(int p, int kk) {
    return PACKED ? (p / 4) * A_TILE + (p % 4) * 32 : p * A_TILE + kk * 32;
  }
  static constexpr __host__ __device__ int b_off(int q, int kk) {
    return PACKED ? (q / 4) * B_TILE + (q % 4) * 32 : q * B_TILE + kk * 32;
  }
  static constexpr int NBUF =
      PROMOTE ? (512 / (NACC * BN) > 4 ? 4 : 512 / (NACC * BN)) : ((2 * NACC * BN <= 512) ? 2 : 1);
  static constexpr int STAGING_PER_WARP = Epi::STAGING_PER_WARP;
  static constexpr int STAGING_BYTES = EPI_WARPS * STAGING_PER_WARP;
  static constexpr int STAGE_BYTES = TILES_A * A_TILE + (STACKED ? NSUB * B_SUB_BYTES : TILES_B * B_TILE);
  static_assert(!STACKED || (INT8_ && NSUB * SUB_ == BN_ && NB_ * SUB_ <= 256 && SUB_ % 16 == 0 &&
                             B_SUB_BYTES % 256 == 0 && NACC_ == NB_),
                "stacked form: INT8, whole sub-tiles, MMA N <= 256");
  static_assert(!PAIR_ || (!PACKED && BN_ % 32 == 0 && BN_ <= 256), "pair tiles: BF16 planes, MMA N <= 256");
  static constexpr int FIXED = 1024 + STAGING_BYTES + 512;
  static constexpr int STAGES_FIT = (kSmemBudget - FIXED) / STAGE_BYTES;
  static constexpr int STAGES = STAGES_FIT > 6 ? 6 : STAGES_FIT;
  static constexpr int SMEM = FIXED + STAGES * STAGE_BYTES;
  static_assert(STAGES >= 2, "at least a double-buffered ring");
  static_assert(NACC * BN * NBUF <= 512, "accumulators exceed TMEM");
  static_assert(SMEM > 116 * 1024, "one CTA per SM keeps the 512-column TMEM allocation uncontended");
  static_assert(!std::is_same<Epi, EpiF32>::value || STAGE_BYTES % 1024 == 0,
                "the FP32 epilogue's swizzled staging starts 1024-byte aligned");
  static_assert(!PROMOTE || (CHUNK > 0 && (NBUF >= 2 || SPLIT_)), "promotion needs chunk buffers");
  static_assert(!SPLIT_ || (PROMOTE_ && NACC_ == 2 && NBUF == 1), "split release: two accumulators, one buffer");
  static __device__ __forceinline__ void epilogue(const OutCtx& p, uint32_t tacc, uint8_t* stg, int lane, int row0,
                                                  int col0, int z) {
    Epi::template run<BN>(p, tacc, stg, lane, row0, col0, z);
  }
  static constexpr bool kDrain = Epi::kDrain;
  static __device__ __forceinline__ void drain(uint32_t tacc, uint8_t* stg, int lane) {
    Epi::template drain<BN>(tacc, stg, lane);
  }
  static __device__ __forceinline__ void store(const OutCtx& p, const uint8_t* stg, int lane, int row0, int col0,
                                               int z) {
    Epi::template store<BN>(p, stg, lane, row0, col0, z);
  }
  static __device__ __forceinline__ void accumulate(uint32_t tacc, float (&master)[COLS_PER_EW]) {
    if constexpr (PROMOTE) Epi::template accumulate<COLS_PER_EW, BN, NACC>(tacc, master);
  }
  // Accumulator d alone (split release).
  static __device__ __forceinline__ void accumulate_one(uint32_t tacc, int d, float (&master)[COLS_PER_EW]) {
    if constexpr (PROMOTE) Epi::template accumulate<COLS_PER_EW, BN, 1>(tacc + (uint32_t)(d * BN), master);
  }
  template <int STG = STAGING_PER_WARP / 4096>
  static __device__ __forceinline__ void finish(const OutCtx& p, const float (&master)[COLS_PER_EW], uint8_t* stg,
                                                int lane, int row0, int col0, int z) {
    if constexpr (PROMOTE) Epi::template finish<COLS_PER_EW, STG>(p, master, stg, lane, row0, col0, z);
  }
};

// K-blocks (32 wide) the tensor cores accumulate before the epilogue adds
// the chunk into its FP32 registers (8: measured 4.7 % faster than 4 on
// BF16x3 at 8192^3 for a 1.6 % larger normwise error).
constexpr int kPromoteChunk = 8;

// BF16x3: (lo,hi), (hi,lo), (hi,hi) -- small terms first -- one accumulator.
// Term tables: for term t, the A plane a[t], the B plane b[t], the
// accumulator d[t], and whether t is the first term of the k-block order to
// write accumulator d[t] (that MMA overwrites instead of accumulating on the
// first k-block of a unit).  Built at compile time.
template <int NT>
struct TermTable {
  int a[NT], b[NT], d[NT];
  bool first[NT];
};

// BF16x3: (lo,hi), (hi,lo), (hi,hi) -- small terms first -- one accumulator.
// Default (tile id 0): 128 x 256 tiles, one TMEM accumulator promoted into
// FP32 registers every kPromoteChunk k-blocks by 8 epilogue warps (two per
// lane quadrant, 128 columns each): without promotion the truncating
// accumulation grows its error linearly in K.  Tile id 1: the same tile
// without promotion (whole K in TMEM).  Tile id 2: 128 x 128 tiles with
// promotion and the correction products in their own accumulator.
struct Bf16x3 : TraitsBase<3, 256, 64, 2, 2, 1, false, EpiF32, true, kPromoteChunk, 8> {
  static constexpr TermTable<3> kTerms{{1, 0, 0}, {0, 1, 0}, {0, 0, 0}, {true, false, false}};
};
struct Bf16x3Wide : TraitsBase<3, 256, 64, 2, 2, 1, false, EpiF32> {
  static constexpr TermTable<3> kTerms{{1, 0, 0}, {0, 1, 0}, {0, 0, 0}, {true, false, false}};
};
struct Bf16x3Promoted : TraitsBase<3, 128, 64, 2, 2, 2, false, EpiF32, true, kPromoteChunk> {
  static constexpr TermTable<3> kTerms{{1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {true, false, true}};
};

// BF16x6: 3-way split, the six products with i + j <= 2; the five
// correction products accumulate in TMEM accumulator 1, the main product
// hi*hi in accumulator 0, so the main accumulator is rounded only by its own
// MMAs; both are promoted into FP32 registers every kPromoteChunk k-blocks.
// Order: smallest first, MMAs that read the same A plane adjacent.
struct Bf16x6 : TraitsBase<6, 128, 64, 3, 3, 2, false, EpiF32, true, kPromoteChunk> {
  static constexpr TermTable<6> kTerms{
      {2, 1, 1, 0, 0, 0}, {0, 1, 0, 2, 1, 0}, {1, 1, 1, 1, 1, 0}, {true, false, false, false, false, true}};
};

// CTA-pair tiles (256 rows): half the shared-memory operand reads and L2
// traffic per output of the 128-row tiles at the same MMA N.
//   Bf16x3Pair  256 x 256, one accumulator promoted every kPromoteChunk k-blocks
//               (Bf16x3Pair128: the 256 x 128 form, used with the fused split).
//   Bf16x6Pair  256 x 128, main and correction accumulators (as Bf16x6),
//               double-buffered.
//   Bf16x6PairWide 256 x 256, main and correction accumulators filling TMEM
//               (one buffer, split release); the 256 x 128 tiles need about
//               1.5x the L2-to-shared-memory bandwidth per flop.
struct Bf16x3Pair : TraitsBase<3, 256, 64, 2, 2, 1, false, EpiF32, true, kPromoteChunk, 8, 0, true> {
  static constexpr TermTable<3> kTerms{{1, 0, 0}, {0, 1, 0}, {0, 0, 0}, {true, false, false}};
};
struct Bf16x3Pair128 : TraitsBase<3, 128, 64, 2, 2, 1, false, EpiF32, true, kPromoteChunk, 8, 0, true> {
  static constexpr TermTable<3> kTerms{{1, 0, 0}, {0, 1, 0}, {0, 0, 0}, {true, false, false}};
};
struct Bf16x6Pair : TraitsBase<6, 128, 64, 3, 3, 2, false, EpiF32, true, kPromoteChunk, 8, 0, true> {
  static constexpr TermTable<6> kTerms{
      {2, 1, 1, 0, 0, 0}, {0, 1, 0, 2, 1, 0}, {1, 1, 1, 1, 1, 0}, {true, false, false, false, false, true}};
};
struct Bf16x6PairWide : TraitsBase<6, 256, 64, 3, 3, 2, false, EpiF32, true, kPromoteChunk, 8, 0, true, true> {
  static constexpr TermTable<6> kTerms{
      {2, 1, 1, 0, 0, 0}, {0, 1, 0, 2, 1, 0}, {1, 1, 1, 1, 1, 0}, {true, false, false, false, false, true}};
};

// Ozaki with S slices: all pairs (p, q) with p + q < S, accumulated into
// diagonal d = p + q.  Stacked form: S MMAs per sub-tile and k-block (one
// per A slice, N shrinking with p) instead of S(S+1)/2 narrow ones -- an MMA
// instruction has a fixed cost in the tensor pipe's front end and reads its
// whole A operand, so few wide MMAs keep the tensor cores busy.  (The term
// table below describes the pairs; the stacked issue order is p ascending
// within each sub-tile.)
template <int S>
struct OzakiBN {
  static constexpr int value = ozaki_bn(S);
};
template <int S>
constexpr TermTable<S*(S + 1) / 2> ozaki_terms() {
  TermTable<S*(S + 1) / 2> t{};
  int i = 0;
  for (int p = 0; p < S; ++p)
    for (int q = 0; p + q < S; ++q) {
      t.a[i] = p;
      t.b[i] = q;
      t.d[i] = p + q;
      t.first[i] = p == 0;
      ++i;
    }
  return t;
}
template <int S>
struct Ozaki : TraitsBase<S*(S + 1) / 2, OzakiBN<S>::value, 128, S, S, S, true, EpiOzaki<S, ozaki_sub(S)>, false, 0,
                          4, ozaki_sub(S)> {
  static constexpr TermTable<S*(S + 1) / 2> kTerms = ozaki_terms<S>();
};

// Launch on `grid` CTAs (pair kernels: grid / 2 clusters of two CTAs; grid even).
template <class Tr>
static cudaError_t launch(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p, int grid, cudaStream_t st) {
  static std::atomic<uint64_t> attr_set{0};  // devices whose context has the limit raised
  cudaError_t e = debug_cuda("smem attribute",
                             ensure_smem_attr(reinterpret_cast<const void*>(tc_gemm_kernel<Tr>), Tr::SMEM, attr_set));
  if (e != cudaSuccess) return e;
  if constexpr (Tr::PAIR) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(Tr::THREADS, 1, 1);
    cfg.dynamicSmemBytes = Tr::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = debug_cuda("pair kernel launch", cudaLaunchKernelEx(&cfg, tc_gemm_kernel<Tr>, a, b, p));
    if (e != cudaSuccess) return e;
    return debug_cuda("pair kernel launch (last error)", cudaGetLastError());
  }
  tc_gemm_kernel<Tr><<<grid, Tr::THREADS, Tr::SMEM, st>>>(a, b, p);
  return debug_cuda("kernel launch", cudaGetLastError());
}

// Clusters of two CTAs of a pair kernel that can be resident at once on the
// current device (one CTA per SM; a GPC with an odd SM count leaves one idle).
template <class Tr>
static int max_pair_clusters(int sms) {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return sms / 2;
  int v = cached[dev].load(std::memory_order_relaxed);
  if (v > 0) return v;
  static std::atomic<uint64_t> attr_set{0};
  if (ensure_smem_attr(reinterpret_cast<const void*>(tc_gemm_kernel<Tr>), Tr::SMEM, attr_set) != cudaSuccess)
    return sms / 2;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(sms & ~1), 1, 1);
  cfg.blockDim = dim3(Tr::THREADS, 1, 1);
  cfg.dynamicSmemBytes = Tr::SMEM;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (debug_cuda("cluster occupancy",
                 cudaOccupancyMaxActiveClusters(&n, reinterpret_cast<const void*>(tc_gemm_kernel<Tr>), &cfg)) !=
          cudaSuccess ||
      n <= 0) {
    cudaGetLastError();
    n = sms / 2;
  }
  cached[dev].store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace tc
}  // namespace cucosma
