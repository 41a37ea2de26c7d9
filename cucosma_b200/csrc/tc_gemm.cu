// tc_gemm.cu -- planning and host entry points of the tensor-core precision
// paths (BF16x3, BF16x6, Ozaki); the kernel template is in tc_kernel.cuh.
#include "simt_gemm.cuh"
#include "split.cuh"
#include "tc_fused.cuh"
#include <cstdlib>
#include "tc_kernel.cuh"

namespace cucosma {
namespace tc {

// Split-K reduction of the Ozaki path: tot = sum_z ws[z] (z ascending),
// C = epi(alpha * ldexp(tot, ea + eb) + beta * C).  With a gate it runs only
// for the slice count chosen on the device.
__global__ void ozaki_reduce_kernel(const double* __restrict__ ws, int64_t split_stride, int64_t ldw, int splits,
                                    double* C, int64_t ldc, int m, int n, const int32_t* __restrict__ ea,
                                    const int32_t* __restrict__ eb, double alpha, double beta, int epi,
                                    const int* gate, int gate_value) {
  if (gate != nullptr && *gate != gate_value) return;
  const int64_t total = (int64_t)m * n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / n;
    const int c = (int)(idx - r * n);
    const double* w = ws + r * ldw + c;
    double tot = w[0];
    for (int zz = 1; zz < splits; ++zz) tot = tot + w[zz * split_stride];
    const double v = ldexp(tot, ea[r] + eb[c]);
    double* po = C + r * ldc + c;
    const double o = beta == 0.0 ? alpha * v : fma(alpha, v, beta * *po);
    *po = apply_epi(o, epi);
  }
}

// ------------------------------------------------------------ planning
// BF16 kernel variants (the descriptor's tile id selects one; 0 = auto).
enum Variant : int {
  kV3Promoted = 0,   // BF16x3 128 x 256, promoted (tile id 3)
  kV3Wide = 1,       // BF16x3 128 x 256, whole K in TMEM (tile id 1)
  kV3Small = 2,      // BF16x3 128 x 128, promoted, two accumulators (tile id 2)
  kV3Pair = 3,       // BF16x3 256 x 256 CTA pair (tile id 4)
  kV6Single = 4,     // BF16x6 128 x 128 (tile id 1)
  kV6Pair = 5,       // BF16x6 256 x 128 CTA pair, two double-buffered accumulators (tile id 2)
  kV6PairWide = 6,   // BF16x6 256 x 256 CTA pair, two accumulators, split release (tile id 3)
  kVOzaki = 7,
  kV3Fused = 10,     // BF16x3 256 x 128 pair, split fused into the kernel (tile id 5)
  kV6Fused = 11,     // BF16x6 256 x 128 pair, split fused into the kernel (tile id 4)
};

// Tiling of one kernel: tiles, K blocks and splits, raster band.
struct Tiling {
  int slices, bn, tiles_m, tiles_n, kblocks, kb_per_split, splits, band;
};

struct Plan {
  int kind;  // 0 bf16x3, 1 bf16x6, 2 ozaki
  int variant, pair, tile_m, bn_local, bk;
  int fused;         // BF16 split done inside the GEMM kernel (no planes in the workspace)
  Tiling t;          // the kernel (Ozaki adaptive: the 8-slice candidate)
  int adaptive;      // Ozaki with the slice count chosen on the device
  int layout_slices; // Ozaki slices per k-block in the workspace
  Tiling t9;         // adaptive Ozaki: the 9-slice candidate
  NativePlan native; // adaptive Ozaki: the native FP64 fallback
  int64_t kpad;
  // Workspace: operand B first (its planes / slices, exponents and
  // magnitude sums depend on N and K only, so row blocks of one problem can
  // share them), then A, then the split-K partials of whichever kernel runs.
  size_t off_b, off_eb, off_colsum, off_stats, off_a, off_ea, off_rowsum, off_part, bytes;
  int64_t ldw;
};

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

static Tiling make_tiling(const Plan& pl, int slices, int bn, const cucosma_gemm_desc* d, const DeviceInfo* di) {
  Tiling t{};
  const int64_t M = d->m, N = d->n, K = d->k;
  t.slices = slices;
  t.bn = bn;
  t.tiles_m = (int)ceil_div(M, pl.tile_m);
  t.tiles_n = (int)ceil_div(N, bn);
  t.kblocks = (int)ceil_div(K, pl.bk);
  const int64_t tiles = (int64_t)t.tiles_m * t.tiles_n;
  // Work slots: one per SM, or one per SM pair for pair tiles.
  const int slots = pl.pair ? di->sms / 2 : di->sms;
  int64_t min_splits = 1, kbmax = INT32_MAX;
  if (pl.kind == 2) {
    // Exact INT32 diagonals: slices * kchunk * 127^2 < 2^31.
    kbmax = ((int64_t)2147483647 / ((int64_t)slices * 127 * 127)) / pl.bk;
    min_splits = ceil_div(t.kblocks, kbmax);
  }
  int64_t splits = d->split_k > 0 ? d->split_k : 1;
  if (d->split_k <= 0 && tiles < slots) splits = std::max<int64_t>(1, std::min<int64_t>(slots / tiles, t.kblocks / 16));
  splits = std::max(splits, min_splits);
  // More splits than one wave of units (the Ozaki exactness bound on long
  // K): as many splits as the same number of waves holds, so that the last
  // wave is full and every unit is shorter (256 x 256 x 1,048,576 at 8
  // slices: 64 splits x 8 tiles = 3.5 waves of 148; 74 splits fill 4).
  if (d->split_k <= 0 && splits > 1 && tiles * splits > slots) {
    const int64_t waves = ceil_div(tiles * splits, (int64_t)slots);
    splits = std::max(splits, waves * slots / tiles);
  }
  splits = std::min<int64_t>(splits, t.kblocks);
  t.kb_per_split = (int)std::min<int64_t>(ceil_div(t.kblocks, splits), kbmax);
  t.splits = (int)ceil_div(t.kblocks, t.kb_per_split);
  // Raster band (tiles of M visited together): measured best at 8192^3 and
  // 16384^3 -- 16 for the BF16 paths (128 x 256 tiles), 4 for Ozaki; pair
  // tiles keep the same band height in rows (8 tiles of 256).
  t.band = d->swizzle > 0 ? d->swizzle : (pl.kind == 2 ? 4 : (pl.pair ? 8 : 16));
  return t;
}

// The fused split pays off when the separate pre-pass (read the FP32
// operands, write nt BF16 planes) would take more than a quarter of the
// GEMM's own bound (tensor time at nt products of BF16, or the HBM time of
// reading the planes and writing -- with beta, also reading -- C): operands
// read only a few times, as in the large-K and large-N families (measured on
// B200, beta 0.5, BF16x3 / BF16x6: 256 x 256 x 1,048,576 0.58 / 0.88 ms fused
// against about 1.2 / 2.6 ms; 256 x 1,048,576 x 256 0.85 / 1.06 against 1.23
// / 1.19 ms), and not where small operands are re-read by many tiles (16384 x
// 16384 x 256, BF16x6: 1.01 fused against 0.70 ms with the pre-pass, whose
// cost there is negligible).
static bool fused_pays(const cucosma_gemm_desc* d, int nt) {
  const double M = (double)d->m, N = (double)d->n, K = (double)d->k;
  const double hbm = 6.5e12, bf16 = 1.6e15;
  const double products = nt == 2 ? 3.0 : 6.0;
  const double c_bytes = M * N * 4.0 * (d->beta != 0.0 ? 2.0 : 1.0), ab_bytes = (M * K + K * N) * 4.0;
  if (ab_bytes < 32.0 * (1 << 20)) return false;  // small operands: the pre-pass costs microseconds
  const double t_pre = (M * K + K * N) * (4.0 + 2.0 * nt) / hbm;
  const double t_mma = 2.0 * M * N * K * products / bf16;
  const double t_mem = ((M * K + K * N) * 2.0 * nt + c_bytes) / hbm;
  return t_pre > 0.25 * std::max(t_mma, t_mem);
}

static Plan make_plan(const cucosma_gemm_desc* d, const DeviceInfo* di, bool allow_fused = true) {
  Plan pl{};
  allow_fused = allow_fused && d->flags == 0;  // the test hooks run the pre-pass path (as does its workspace query)
  const int64_t M = d->m, N = d->n, K = d->k;
  int slices = 0, bn = 0;
  pl.bk = 32;
  if (d->precision == CUCOSMA_PRECISION_OZAKI) {
    pl.kind = 2;
    pl.variant = kVOzaki;
    pl.adaptive = d->slices == 0;
    slices = pl.adaptive ? 8 : d->slices;
    pl.layout_slices = pl.adaptive ? kOzakiLayoutAdaptive : slices;
    bn = ozaki_bn(slices);
    pl.kpad = round_up(K, 32);
  } else {
    pl.kind = d->precision == CUCOSMA_PRECISION_BF16X6 ? 1 : 0;
    slices = pl.kind == 1 ? 3 : 2;
    pl.layout_slices = slices;
    // Auto: CTA-pair tiles unless the problem has a single 128-row block.
    const bool pair_ok = M > 128;
    if (pl.kind == 0) {
      switch (d->tile) {
        case 1: pl.variant = kV3Wide; break;
        case 2: pl.variant = kV3Small; break;
        case 3: pl.variant = kV3Promoted; break;
        case 4: pl.variant = kV3Pair; break;
        case 5: pl.variant = allow_fused ? kV3Fused : kV3Pair; break;
        default:
          pl.variant = !pair_ok ? kV3Promoted : (allow_fused && fused_pays(d, 2)) ? kV3Fused : kV3Pair;
      }
    } else {
      switch (d->tile) {
        case 1: pl.variant = kV6Single; break;
        case 2: pl.variant = kV6Pair; break;
        case 3: pl.variant = kV6PairWide; break;
        case 4: pl.variant = allow_fused ? kV6Fused : kV6Pair; break;
        default:
          pl.variant = !pair_ok ? kV6Single : (allow_fused && fused_pays(d, 3)) ? kV6Fused : kV6PairWide;
      }
    }
    bn = (pl.variant == kV3Small || pl.variant == kV6Single || pl.variant == kV6Pair || pl.variant == kV6Fused ||
          pl.variant == kV3Fused)
             ? 128
             : 256;
    pl.fused = pl.variant == kV3Fused || pl.variant == kV6Fused;
    pl.kpad = round_up(K, 8);
  }
  pl.pair = (pl.variant == kV3Pair || pl.variant == kV6Pair || pl.variant == kV6PairWide || pl.fused) ? 1 : 0;
  pl.tile_m = pl.pair ? 256 : 128;
  pl.bn_local = pl.pair ? bn / 2 : bn;
  pl.t = make_tiling(pl, slices, bn, d, di);
  if (pl.adaptive) {
    pl.t9 = make_tiling(pl, 9, ozaki_bn(9), d, di);
    cucosma_gemm_desc nd = *d;
    nd.precision = CUCOSMA_PRECISION_NATIVE;
    nd.slices = 0;
    nd.tile = 0;
    pl.native = plan_native(&nd, di->sms);
  }
  const int es_in = pl.kind == 2 ? 1 : 2;
  const int es_out = pl.kind == 2 ? 8 : 4;
  const size_t ls = pl.fused ? 0 : (size_t)pl.layout_slices;  // the fused kernel keeps no planes
  size_t off = 0;
  pl.off_b = off;
  off = al256(off + ls * N * pl.kpad * es_in);
  pl.off_eb = pl.off_colsum = pl.off_stats = off;
  if (pl.kind == 2) {
    off = al256(off + (size_t)N * 4);
    pl.off_colsum = pl.off_stats = off;
    if (pl.adaptive) {
      off = al256(off + (size_t)N * 8);
      pl.off_stats = off;
      off = al256(off + sizeof(OzakiStats));
    }
  }
  pl.off_a = off;
  off = al256(off + ls * M * pl.kpad * es_in);
  pl.off_ea = pl.off_rowsum = off;
  if (pl.kind == 2) {
    off = al256(off + (size_t)M * 4);
    pl.off_rowsum = off;
    if (pl.adaptive) off = al256(off + (size_t)M * 8);
  }
  pl.ldw = round_up(N, 4);
  pl.off_part = off;
  size_t part = pl.t.splits > 1 ? (size_t)pl.t.splits * M * pl.ldw * es_out : 0;
  if (pl.adaptive) {
    if (pl.t9.splits > 1) part = std::max(part, (size_t)pl.t9.splits * M * pl.ldw * es_out);
    part = std::max(part, pl.native.ws_bytes);
  }
  if (part) off = al256(off + part);
  pl.bytes = off;
  return pl;
}

static int plan_launches(const Plan& pl) {
  if (pl.fused) return 1 + (pl.t.splits > 1 ? 1 : 0);
  if (pl.kind != 2) return 3 + (pl.t.splits > 1 ? 1 : 0);
  if (!pl.adaptive) return 4 + (pl.t.splits > 1 ? 1 : 0);
  // prep B (2), prep A, decision, the three gated kernels and their reductions
  return 7 + (pl.t.splits > 1) + (pl.t9.splits > 1) + (pl.native.splits > 1);
}

}  // namespace tc

// ------------------------------------------------------------ host API
using namespace tc;

cucosma_status tc_workspace_size(const cucosma_gemm_desc* d, size_t* bytes, const DeviceInfo* di) {
  *bytes = make_plan(d, di).bytes;
  return CUCOSMA_STATUS_SUCCESS;
}

bool tc_plan_is_fused(const cucosma_gemm_desc* d, const DeviceInfo* di) { return make_plan(d, di).fused != 0; }

void tc_plan_info(const cucosma_gemm_desc* d, const DeviceInfo* di, cucosma_plan_info* info, bool allow_fused) {
  const Plan pl = make_plan(d, di, allow_fused);
  info->path = pl.kind + 1;
  info->tile_m = pl.tile_m;
  info->tile_n = pl.t.bn;
  info->tile_k = pl.bk;
  info->splits = pl.t.splits;
  info->band = pl.t.band;
  info->slices = pl.adaptive ? 0 : pl.t.slices;
  info->launches = plan_launches(pl);
  info->kchunk = (int64_t)pl.t.kb_per_split * pl.bk;
  info->kpad = pl.kpad;
  info->workspace_bytes = pl.bytes;
  info->off_a = pl.off_a;
  info->off_b = pl.off_b;
  info->off_ea = pl.off_ea;
  info->off_eb = pl.off_eb;
  info->off_part = pl.off_part;
  info->off_choice = pl.adaptive ? pl.off_stats + offsetof(OzakiStats, choice) : 0;
  info->layout_slices = pl.layout_slices;
  info->fused = pl.fused;
}

namespace {

// Kernel parameters of one tiling (shared fields of every precision path).
TcParams tc_params(const cucosma_gemm_desc* d, const Tiling& t, const Plan& pl, void* C, uint8_t* w,
                   const DeviceInfo* di) {
  TcParams p{};
  p.m = (int)d->m;
  p.n = (int)d->n;
  p.k = (int)d->k;
  p.tiles_m = t.tiles_m;
  p.tiles_n = t.tiles_n;
  p.kblocks = t.kblocks;
  p.kb_per_split = t.kb_per_split;
  p.splits = t.splits;
  p.band = t.band;
  p.epilogue = d->epilogue;
  p.alpha = d->alpha;
  p.beta = d->beta;
  wait_ctl(di, &p.ctl.status, &p.ctl.timeout_ns);
  p.skip_stage = (d->flags & CUCOSMA_FLAG_TEST_SKIP_STAGE) ? 0 : -1;
  if (t.splits > 1) {
    p.partial = 1;
    p.out = w + pl.off_part;
    p.ldo = pl.ldw;
    p.ws_split_stride = (int64_t)d->m * pl.ldw;
  } else {
    p.partial = 0;
    p.out = C;
    p.ldo = d->ldc;
    // FP32 results leave through TMA when C allows a tensor map (16-byte
    // aligned base and rows) and its rows end on a 16-byte boundary (a box
    // store clips the columns past N only to the 16-byte granule: on B200 it
    // wrote the rest of the last granule); otherwise the epilogue stores rows
    // itself.  CUCOSMA_TMA_EPILOGUE=0 turns the TMA path off.
    static const bool tma_epilogue = [] {
      const char* e = std::getenv("CUCOSMA_TMA_EPILOGUE");
      return !(e && e[0] == '0');
    }();
    if (tma_epilogue && pl.kind != 2 && C != nullptr && (reinterpret_cast<uintptr_t>(C) & 15) == 0 &&
        (d->ldc * 4) % 16 == 0 && d->n % 4 == 0)
      p.tma_out = encode_2d(&p.tmc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, (uint64_t)d->n, (uint64_t)d->m,
                            (uint64_t)d->ldc, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B) &&
                          encode_2d(&p.tmc_pf, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, (uint64_t)d->n,
                                    (uint64_t)d->m, (uint64_t)d->ldc, 64, 32, CU_TENSOR_MAP_SWIZZLE_NONE)
                      ? 1
                      : 0;
    static const bool tma_wide = [] {
      const char* e = std::getenv("CUCOSMA_TMA_WIDE");
      return !(e && e[0] == '0');
    }();
    if (p.tma_out && tma_wide && d->n % 32 == 0)
      p.tma_wide = encode_3d(&p.tmc3, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, 32, (uint64_t)d->n / 32, (uint64_t)d->m,
                             32, (uint64_t)d->ldc, 32, 2, 32, CU_TENSOR_MAP_SWIZZLE_128B)
                       ? 1
                       : 0;
  }
  return p;
}

// One Ozaki GEMM (+ its split-K reduction) with t.slices slices read from a
// layout of pl.layout_slices slices per k-block; gated when gate != null.
cudaError_t run_ozaki(const cucosma_gemm_desc* d, const Plan& pl, const Tiling& t, void* C, uint8_t* w,
                      const DeviceInfo* di, cudaStream_t st, const int* gate, int& launches) {
  const int s = t.slices, ls = pl.layout_slices;
  const int m = (int)d->m, n = (int)d->n;
  int32_t* ea = reinterpret_cast<int32_t*>(w + pl.off_ea);
  int32_t* eb = reinterpret_cast<int32_t*>(w + pl.off_eb);
  TcParams p = tc_params(d, t, pl, C, w, di);
  p.ea = ea;
  p.eb = eb;
  p.gate = gate;
  p.gate_value = s;
  p.b_layout_slices = ls;
  // A slices (packed) as a 3-D byte tensor {32 ls (slices of one k-block), k-blocks, rows}: boxes of 128
  // bytes bring slices 4j .. 4j+3; B slices (stacked) as {32 bytes, columns, k-block * ls + slice}, one
  // box = slices 0 .. s-1 of a sub-tile.
  const uint64_t kbs = (uint64_t)pl.kpad / 32;
  CUtensorMap ta, tb;
  if (!encode_3d(&ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, w + pl.off_a, 32ull * ls, kbs, m, 32ull * ls,
                 (uint64_t)pl.kpad * ls, 128, 1, 128, CU_TENSOR_MAP_SWIZZLE_128B) ||
      !encode_3d(&tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, w + pl.off_b, 32, n, kbs * ls, 32, 32ull * n, 32, ozaki_sub(s),
                 s, CU_TENSOR_MAP_SWIZZLE_32B))
    return cudaErrorInvalidValue;
  const int grid = std::min(t.tiles_m * t.tiles_n * t.splits, di->sms);
  cudaError_t e;
  switch (s) {
    case 4: e = launch<Ozaki<4>>(ta, tb, p, grid, st); break;
    case 5: e = launch<Ozaki<5>>(ta, tb, p, grid, st); break;
    case 6: e = launch<Ozaki<6>>(ta, tb, p, grid, st); break;
    case 7: e = launch<Ozaki<7>>(ta, tb, p, grid, st); break;
    case 8: e = launch<Ozaki<8>>(ta, tb, p, grid, st); break;
    case 9: e = launch<Ozaki<9>>(ta, tb, p, grid, st); break;
    default: return cudaErrorInvalidValue;
  }
  launches += 1;
  if (e == cudaSuccess && t.splits > 1) {
    const int64_t work = (int64_t)m * n;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(work, 256), di->sms * 8));
    ozaki_reduce_kernel<<<blocks, 256, 0, st>>>((const double*)p.out, p.ws_split_stride, pl.ldw, t.splits,
                                                (double*)C, d->ldc, m, n, ea, eb, d->alpha, d->beta, d->epilogue, gate,
                                                s);
    e = cudaGetLastError();
    launches += 1;
  }
  return e;
}

}  // namespace

cucosma_status tc_gemm_ex(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws,
                          size_t ws_bytes, const DeviceInfo* di, cudaStream_t st, int prep) {
  // Callers that supply prepared planes (prep without both operands) never
  // get the fused kernel, which reads the FP32 operands themselves.
  const bool allow_fused =
      (prep & (kPrepA | kPrepB)) == (kPrepA | kPrepB) && !(prep & kNoFused) && A != nullptr && B != nullptr;
  const Plan pl = make_plan(d, di, allow_fused);
  if (pl.bytes > 0 && (ws == nullptr || ws_bytes < pl.bytes)) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  if (pl.kind == 2 && (pl.t.slices < 4 || pl.t.slices > 9)) return CUCOSMA_STATUS_NOT_SUPPORTED;
  uint8_t* w = static_cast<uint8_t*>(ws);
  const int m = (int)d->m, n = (int)d->n, k = (int)d->k;
  cudaError_t e = cudaSuccess;
  int launches = 0;
  if (pl.fused) {
    // FP32 operand tiles straight from the caller's buffers.  BF16x3 (in
    // place): A [128 rows][64 K] and B [64 K][64 columns] boxes, 256-byte
    // rows; BF16x6: A [128 rows][32 K] (128-byte swizzle) and B [32 K][64].
    const int kw = pl.kind == 0 ? 64 : 32;  // k-values per FP32 row of a stage
    CUtensorMap ta, tb;
    if (!encode_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, A, k, m, d->lda, kw, 128,
                   pl.kind == 0 ? CU_TENSOR_MAP_SWIZZLE_NONE : CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, B, n, k, d->ldb, pl.bn_local, kw,
                   CU_TENSOR_MAP_SWIZZLE_NONE))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    const TcParams p = tc_params(d, pl.t, pl, C, w, di);
    prof_begin(st);
    // C-heavy shapes (C traffic above a quarter of the operands'): the
    // variant with two staging blocks per epilogue warp and three stages
    // (256 x 1,048,576 x 256, beta 0.5: 0.85 against 0.94 ms on B200)
    const double c_bytes = (double)d->m * d->n * 4.0 * (d->beta != 0.0 ? 2.0 : 1.0);
    const double ab_bytes = ((double)d->m * d->k + (double)d->k * d->n) * 4.0;
    const bool c_heavy = c_bytes > 0.25 * ab_bytes;
    if (pl.kind == 1)
      e = c_heavy ? launch_fused_inplace<Bf16x6Pair, 2>(ta, tb, p, di->sms, st)
                  : launch_fused_inplace<Bf16x6Pair, 1>(ta, tb, p, di->sms, st);
    else
      e = c_heavy ? launch_fused_inplace<Bf16x3Pair128, 2>(ta, tb, p, di->sms, st)
                  : launch_fused_inplace<Bf16x3Pair128, 1>(ta, tb, p, di->sms, st);
    prof_end(st);
    launches += 1;
    if (e == cudaSuccess && pl.t.splits > 1) {
      e = simt::launch_reduce<float>((const float*)p.out, p.ws_split_stride, pl.ldw, pl.t.splits, (float*)C, d->ldc, m,
                                     n, d->alpha, d->beta, d->epilogue, di->sms, st);
      launches += 1;
    }
  } else if (pl.kind != 2) {
    const int nt = pl.t.slices;
    if (prep & kPrepA) {
      e = launch_split_bf16((const float*)A, d->lda, m, k, pl.kpad, nt, w + pl.off_a, false, di->sms, st);
      launches += 1;
    }
    if (e == cudaSuccess && (prep & kPrepB)) {
      e = launch_split_bf16((const float*)B, d->ldb, k, n, pl.kpad, nt, w + pl.off_b, true, di->sms, st);
      launches += 1;
    }
    if (e != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    CUtensorMap ta, tb;
    if (!encode_3d(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, w + pl.off_a, k, m, nt, pl.kpad, (uint64_t)m * pl.kpad,
                   pl.bk, 128, nt, CU_TENSOR_MAP_SWIZZLE_64B) ||
        !encode_3d(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, w + pl.off_b, k, n, nt, pl.kpad, (uint64_t)n * pl.kpad,
                   pl.bk, pl.bn_local, nt, CU_TENSOR_MAP_SWIZZLE_64B))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    const TcParams p = tc_params(d, pl.t, pl, C, w, di);
    const int units = pl.t.tiles_m * pl.t.tiles_n * pl.t.splits;
    const int grid = std::min(units, di->sms);
    auto pair_grid = [&](int clusters) { return 2 * std::max(1, std::min(units, clusters)); };
    prof_begin(st);
    switch (pl.variant) {
      case kV6Single: e = launch<Bf16x6>(ta, tb, p, grid, st); break;
      case kV6Pair: e = launch<Bf16x6Pair>(ta, tb, p, pair_grid(max_pair_clusters<Bf16x6Pair>(di->sms)), st); break;
      case kV6PairWide:
        e = launch<Bf16x6PairWide>(ta, tb, p, pair_grid(max_pair_clusters<Bf16x6PairWide>(di->sms)), st);
        break;
      case kV3Small: e = launch<Bf16x3Promoted>(ta, tb, p, grid, st); break;
      case kV3Wide: e = launch<Bf16x3Wide>(ta, tb, p, grid, st); break;
      case kV3Pair: e = launch<Bf16x3Pair>(ta, tb, p, pair_grid(max_pair_clusters<Bf16x3Pair>(di->sms)), st); break;
      default: e = launch<Bf16x3>(ta, tb, p, grid, st);
    }
    prof_end(st);
    launches += 1;
    if (e == cudaSuccess && pl.t.splits > 1) {
      e = simt::launch_reduce<float>((const float*)p.out, p.ws_split_stride, pl.ldw, pl.t.splits, (float*)C, d->ldc, m,
                                     n, d->alpha, d->beta, d->epilogue, di->sms, st);
      launches += 1;
    }
  } else {
    const int ls = pl.layout_slices;
    int32_t* ea = reinterpret_cast<int32_t*>(w + pl.off_ea);
    int32_t* eb = reinterpret_cast<int32_t*>(w + pl.off_eb);
    OzakiStats* stats = pl.adaptive ? reinterpret_cast<OzakiStats*>(w + pl.off_stats) : nullptr;
    unsigned long long* colsum = pl.adaptive ? reinterpret_cast<unsigned long long*>(w + pl.off_colsum) : nullptr;
    unsigned long long* rowsum = pl.adaptive ? reinterpret_cast<unsigned long long*>(w + pl.off_rowsum) : nullptr;
    if (prep & kPrepB) {
      e = launch_ozaki_prep_b(ls, (const double*)B, d->ldb, k, n, pl.kpad, eb, reinterpret_cast<int8_t*>(w + pl.off_b),
                              colsum, stats, di->sms, st);
      launches += 2;
    }
    if (e == cudaSuccess && (prep & kPrepA)) {
      e = launch_ozaki_prep_a(ls, (const double*)A, d->lda, m, k, pl.kpad, ea, reinterpret_cast<int8_t*>(w + pl.off_a),
                              rowsum, stats, di->sms, st);
      launches += pl.kpad > kOzakiRowChunk ? 2 : 1;  // long rows: exponent and slicing kernels
    }
    if (e == cudaSuccess && pl.adaptive) {
      e = launch_ozaki_decide(rowsum, m, colsum, n, k, stats, di->sms, st);
      launches += 1;
    }
    if (e != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    prof_begin(st);
    if (!pl.adaptive) {
      e = run_ozaki(d, pl, pl.t, C, w, di, st, nullptr, launches);
    } else {
      // Three kernels, each gated on the device's choice: 8 slices, 9
      // slices, or native FP64 (the two not chosen return at once).
      const int* gate = &stats->choice;
      e = run_ozaki(d, pl, pl.t, C, w, di, st, gate, launches);
      if (e == cudaSuccess) e = run_ozaki(d, pl, pl.t9, C, w, di, st, gate, launches);
      if (e == cudaSuccess) {
        cucosma_gemm_desc nd = *d;
        nd.precision = CUCOSMA_PRECISION_NATIVE;
        // (counts its own launches)
        if (native_gemm_gated(&nd, pl.native, A, B, C, w + pl.off_part, di, st, gate, 0) != CUCOSMA_STATUS_SUCCESS)
          e = cudaErrorLaunchFailure;
      }
    }
    prof_end(st);
  }
  note_launches(launches);
  return e == cudaSuccess ? CUCOSMA_STATUS_SUCCESS : CUCOSMA_STATUS_LAUNCH_FAILED;
}

}  // namespace cucosma
