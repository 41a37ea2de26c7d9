// tc_gemm.cuh -- parameters of the tcgen05 precision-path kernel.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace cucosma {

constexpr int kOzakiDefaultSlices = 8;

// Ozaki tile geometry for S slices (stacked form, see tc_kernel.cuh): the B
// slices of a sub-tile of ozaki_sub(S) output columns are stacked along N, so
// one MMA of N = (S - p) * sub columns covers every diagonal that A slice p
// feeds; S * sub <= 256 (the largest MMA N).  ozaki_nsub(S) sub-tiles fill
// the 512 TMEM columns; the tile is 128 x ozaki_bn(S).
constexpr int ozaki_sub(int s) { return s <= 4 ? 64 : (s == 5 ? 48 : (s <= 8 ? 32 : 16)); }
constexpr int ozaki_nsub(int s) { return 512 / (s * ozaki_sub(s)); }
constexpr int ozaki_bn(int s) { return ozaki_nsub(s) * ozaki_sub(s); }

namespace tc {

// One problem of a grouped launch, stored in the workspace.  The tensor maps
// describe this problem's operand planes (they live in global memory; the
// TMA unit reads them there).  Tiles of all problems are numbered
// consecutively: this problem owns [tile_start, tile_start + tiles_m*tiles_n).
struct alignas(64) GroupEntry {
  CUtensorMap tmA, tmB;
  void* C;
  int64_t ldc;
  const int32_t* ea;  // Ozaki exponents of this problem (null for BF16)
  const int32_t* eb;
  int m, n, k, kblocks;
  int tiles_m, tiles_n, tile_start, pad0;
  // operand pre-pass: sources, destination planes, first pre-pass block of
  // this problem for the A rows / B tiles / exponent passes
  const void* A;
  const void* B;
  int64_t lda, ldb, kpad;
  void* planes_a;
  void* planes_b;
  int pre_a_start, pre_b_start, exp_a_start, exp_b_start;
};

struct TcParams {
  // FP32 output C through TMA (tma_out = 1): 32 x 32 boxes, 128-byte
  // swizzle; used by the epilogue for whole-problem outputs (not split-K
  // partials, not grouped launches).
  CUtensorMap tmc;
  // The same C with 64-column boxes (no swizzle), for L2 prefetches only:
  // 256-byte row requests (128-byte ones cap a stream near 4.6 TB/s on B200).
  CUtensorMap tmc_pf;
  // With N a multiple of 32: C as {32 columns, N / 32 column chunks, M rows}
  // with [32 rows][2 chunks][32] boxes (128-byte swizzle per 128-byte line),
  // so the epilogue's loads and stores are 256-byte row requests.
  CUtensorMap tmc3;
  int tma_out, tma_wide;
  int m, n, k;
  int tiles_m, tiles_n;
  int kblocks;       // k-blocks of the whole K
  int kb_per_split;  // k-blocks per split-K unit
  int splits;
  int band;          // raster band height (tiles of M visited together)
  int epilogue;
  int partial;       // 1: raw partial sums into the workspace (split-K)
  double alpha, beta;
  void* out;
  int64_t ldo;
  int64_t ws_split_stride;
  const int32_t* ea;  // Ozaki row exponents of A
  const int32_t* eb;  // Ozaki column exponents of B
  WaitCtl ctl;
  int skip_stage;  // test hook: ring position whose loads the producer omits (-1: none)
  // Grouped launch: when ngroups > 0 the problems come from groups[] (all
  // other per-problem fields above are ignored) and units = total_tiles.
  const GroupEntry* groups;
  int ngroups, total_tiles;
  // Optional device-side gate: the kernel runs only if *gate == gate_value
  // (the adaptive Ozaki call's slice count, chosen on the device).
  const int* gate;
  int gate_value;
  // Ozaki: slices per k-block in the stacked B layout (0: the kernel's own count).
  int b_layout_slices;
};

// Where a work unit's result goes (from TcParams, or from a GroupEntry).
struct OutCtx {
  int m, n, epilogue, partial;
  double alpha, beta;
  void* out;
  int64_t ldo, ws_split_stride;
  const int32_t* ea;
  const int32_t* eb;
  const CUtensorMap* tmc;     // non-null: the FP32 epilogue moves C by TMA
  const CUtensorMap* tmc_pf;  // its 64-column prefetch boxes
  const CUtensorMap* tmc3;    // non-null: 64-column 3-D boxes (needs two staging blocks)
  uint64_t* tbar;          // this epilogue warp's barriers for its C loads (one per staging block)
  int stg_blocks;          // 32 x 32 staging blocks this warp has (1 or 2)
  WaitCtl ctl;
};

// A resolved work unit: operand descriptors, tile coordinates, K range.
struct Unit {
  const CUtensorMap* ta;
  const CUtensorMap* tb;
  int tm, tn, z, kb0, kb1;
  int group;  // -1 when not grouped
};

}  // namespace tc
}  // namespace cucosma
