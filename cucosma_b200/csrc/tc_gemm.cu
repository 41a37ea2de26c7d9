// tc_gemm.cu -- planning and host entry points of the tensor-core precision
// paths (BF16x3, BF16x6, Ozaki); the kernel template is in tc_kernel.cuh.
#include "simt_gemm.cuh"
#include "split.cuh"
#include "tc_kernel.cuh"

namespace cucosma {
namespace tc {

// Split-K reduction of the Ozaki path: tot = sum_z ws[z] (z ascending),
// C = epi(alpha * ldexp(tot, ea + eb) + beta * C).
__global__ void ozaki_reduce_kernel(const double* __restrict__ ws, int64_t split_stride, int64_t ldw, int splits,
                                    double* C, int64_t ldc, int m, int n, const int32_t* __restrict__ ea,
                                    const int32_t* __restrict__ eb, double alpha, double beta, int epi) {
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
struct Plan {
  int kind;  // 0 bf16x3, 1 bf16x6, 2 ozaki
  int slices, bn, bk, tiles_m, tiles_n, kblocks, kb_per_split, splits, band;
  int64_t kpad;
  size_t off_a, off_b, off_ea, off_eb, off_part, bytes;
  int64_t ldw;
};

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

static Plan make_plan(const cucosma_gemm_desc* d, const DeviceInfo* di) {
  Plan pl{};
  const int64_t M = d->m, N = d->n, K = d->k;
  if (d->precision == CUCOSMA_PRECISION_OZAKI) {
    pl.kind = 2;
    pl.slices = d->slices ? d->slices : kOzakiDefaultSlices;
    pl.bn = ozaki_bn(pl.slices);
    pl.bk = 32;
    pl.kpad = round_up(K, 32);
  } else {
    pl.kind = d->precision == CUCOSMA_PRECISION_BF16X6 ? 1 : 0;
    pl.slices = pl.kind == 1 ? 3 : 2;
    pl.bn = (pl.kind == 0 && d->tile != 2) ? 256 : 128;  // BF16x3 tile 2: promoted 128 x 128
    pl.bk = 32;
    pl.kpad = round_up(K, 8);
  }
  pl.tiles_m = (int)ceil_div(M, 128);
  pl.tiles_n = (int)ceil_div(N, pl.bn);
  pl.kblocks = (int)ceil_div(K, pl.bk);
  const int64_t tiles = (int64_t)pl.tiles_m * pl.tiles_n;
  int64_t min_splits = 1;
  if (pl.kind == 2) {
    // Exact INT32 diagonals: slices * kchunk * 127^2 < 2^31.
    const int64_t kmax = ((int64_t)2147483647 / ((int64_t)pl.slices * 127 * 127)) / pl.bk * pl.bk;
    min_splits = ceil_div(K, kmax);
  }
  int64_t splits = d->split_k > 0 ? d->split_k : 1;
  if (d->split_k <= 0 && tiles < di->sms) splits = std::max<int64_t>(1, std::min<int64_t>(di->sms / tiles, pl.kblocks / 16));
  splits = std::max(splits, min_splits);
  splits = std::min<int64_t>(splits, pl.kblocks);
  pl.kb_per_split = (int)ceil_div(pl.kblocks, splits);
  if (pl.kind == 2) {
    const int64_t kbmax = ((int64_t)2147483647 / ((int64_t)pl.slices * 127 * 127)) / pl.bk;
    pl.kb_per_split = (int)std::min<int64_t>(pl.kb_per_split, kbmax);
  }
  pl.splits = (int)ceil_div(pl.kblocks, pl.kb_per_split);
  // Raster band (tiles of M visited together): measured best at 8192^3 and
  // 16384^3 -- 16 for the BF16 paths (128 x 256 tiles), 4 for Ozaki.
  pl.band = d->swizzle > 0 ? d->swizzle : (pl.kind == 2 ? 4 : 16);
  const int es_in = pl.kind == 2 ? 1 : 2;
  const int es_out = pl.kind == 2 ? 8 : 4;
  size_t off = 0;
  pl.off_a = off;
  off = al256(off + (size_t)pl.slices * M * pl.kpad * es_in);
  pl.off_b = off;
  off = al256(off + (size_t)pl.slices * N * pl.kpad * es_in);
  pl.off_ea = off;
  if (pl.kind == 2) {
    off = al256(off + (size_t)M * 4);
    pl.off_eb = off;
    off = al256(off + (size_t)N * 4);
  }
  pl.ldw = round_up(N, 4);
  pl.off_part = off;
  if (pl.splits > 1) off = al256(off + (size_t)pl.splits * M * pl.ldw * es_out);
  pl.bytes = off;
  return pl;
}

}  // namespace tc

// ------------------------------------------------------------ host API
using namespace tc;

cucosma_status tc_workspace_size(const cucosma_gemm_desc* d, size_t* bytes, const DeviceInfo* di) {
  *bytes = make_plan(d, di).bytes;
  return CUCOSMA_STATUS_SUCCESS;
}

void tc_plan_info(const cucosma_gemm_desc* d, const DeviceInfo* di, cucosma_plan_info* info) {
  const Plan pl = make_plan(d, di);
  info->path = pl.kind + 1;
  info->tile_m = 128;
  info->tile_n = pl.bn;
  info->tile_k = pl.bk;
  info->splits = pl.splits;
  info->band = pl.band;
  info->slices = pl.slices;
  info->launches = (pl.kind == 2 ? 4 : 3) + (pl.splits > 1 ? 1 : 0);
  info->kchunk = (int64_t)pl.kb_per_split * pl.bk;
  info->kpad = pl.kpad;
  info->workspace_bytes = pl.bytes;
  info->off_a = pl.off_a;
  info->off_b = pl.off_b;
  info->off_ea = pl.off_ea;
  info->off_eb = pl.off_eb;
  info->off_part = pl.off_part;
}

cucosma_status tc_gemm(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws,
                       const DeviceInfo* di, cudaStream_t st) {
  return tc_gemm_ex(d, A, B, C, ws, di, st, false);
}

cucosma_status tc_gemm_ex(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws,
                          const DeviceInfo* di, cudaStream_t st, bool planes_ready) {
  const Plan pl = make_plan(d, di);
  if (planes_ready && pl.kind == 2) return CUCOSMA_STATUS_NOT_SUPPORTED;
  if (pl.kind == 2 && (pl.slices < 4 || pl.slices > 9)) return CUCOSMA_STATUS_NOT_SUPPORTED;
  uint8_t* w = static_cast<uint8_t*>(ws);
  const int m = (int)d->m, n = (int)d->n, k = (int)d->k;
  TcParams p{};
  p.m = m;
  p.n = n;
  p.k = k;
  p.tiles_m = pl.tiles_m;
  p.tiles_n = pl.tiles_n;
  p.kblocks = pl.kblocks;
  p.kb_per_split = pl.kb_per_split;
  p.splits = pl.splits;
  p.band = pl.band;
  p.epilogue = d->epilogue;
  p.alpha = d->alpha;
  p.beta = d->beta;
  wait_ctl(di, &p.ctl.status, &p.ctl.timeout_ns);
  p.skip_stage = (d->flags & CUCOSMA_FLAG_TEST_SKIP_STAGE) ? 0 : -1;
  if (pl.splits > 1) {
    p.partial = 1;
    p.out = w + pl.off_part;
    p.ldo = pl.ldw;
    p.ws_split_stride = (int64_t)m * pl.ldw;
  } else {
    p.partial = 0;
    p.out = C;
    p.ldo = d->ldc;
  }
  const int units = pl.tiles_m * pl.tiles_n * pl.splits;
  const int grid = std::min(units, di->sms);
  CUtensorMap ta, tb;
  cudaError_t e = cudaSuccess;
  int launches = 0;
  if (pl.kind != 2) {
    const int nt = pl.slices;
    if (!planes_ready) {
      e = launch_split_bf16((const float*)A, d->lda, m, k, pl.kpad, nt, w + pl.off_a, false, di->sms, st);
      if (e == cudaSuccess)
        e = launch_split_bf16((const float*)B, d->ldb, k, n, pl.kpad, nt, w + pl.off_b, true, di->sms, st);
      launches += 2;
      if (e != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    }
    if (!encode_3d(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, w + pl.off_a, k, m, nt, pl.kpad, (uint64_t)m * pl.kpad,
                   pl.bk, 128, nt, CU_TENSOR_MAP_SWIZZLE_64B) ||
        !encode_3d(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, w + pl.off_b, k, n, nt, pl.kpad, (uint64_t)n * pl.kpad,
                   pl.bk, pl.bn, nt, CU_TENSOR_MAP_SWIZZLE_64B))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    prof_begin(st);
    e = pl.kind == 1 ? launch<Bf16x6>(ta, tb, p, grid, st)
        : pl.bn == 128 ? launch<Bf16x3Promoted>(ta, tb, p, grid, st)
        : d->tile == 1 ? launch<Bf16x3Wide>(ta, tb, p, grid, st)
                       : launch<Bf16x3>(ta, tb, p, grid, st);
    prof_end(st);
    launches += 1;
    if (e == cudaSuccess && pl.splits > 1) {
      e = simt::launch_reduce<float>((const float*)p.out, p.ws_split_stride, pl.ldw, pl.splits, (float*)C, d->ldc, m, n,
                                     d->alpha, d->beta, d->epilogue, di->sms, st);
      launches += 1;
    }
  } else {
    const int s = pl.slices;
    int32_t* ea = reinterpret_cast<int32_t*>(w + pl.off_ea);
    int32_t* eb = reinterpret_cast<int32_t*>(w + pl.off_eb);
    e = launch_ozaki_exponents((const double*)A, d->lda, (const double*)B, d->ldb, m, n, k, ea, eb, di->sms, st);
    if (e == cudaSuccess)
      e = launch_ozaki_slices(s, (const double*)A, d->lda, (const double*)B, d->ldb, m, n, k, pl.kpad, ea, eb,
                              reinterpret_cast<int8_t*>(w + pl.off_a), reinterpret_cast<int8_t*>(w + pl.off_b),
                              di->sms, st);
    launches += 3;
    if (e != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    // A slices (packed) as a 3-D byte tensor {32 s (slices of one k-block), k-blocks, rows}; B slices
    // (stacked) as {32 bytes, columns, k-block * s + slice}, one box = all slices of a sub-tile.
    const uint64_t kbs = (uint64_t)pl.kpad / 32;
    if (!encode_3d(&ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, w + pl.off_a, 32ull * s, kbs, m, 32ull * s,
                   (uint64_t)pl.kpad * s, 128, 1, 128, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_3d(&tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, w + pl.off_b, 32, n, kbs * s, 32, 32ull * n, 32, ozaki_sub(s),
                   s, CU_TENSOR_MAP_SWIZZLE_32B))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    p.ea = ea;
    p.eb = eb;
    prof_begin(st);
    switch (s) {
      case 4: e = launch<Ozaki<4>>(ta, tb, p, grid, st); break;
      case 5: e = launch<Ozaki<5>>(ta, tb, p, grid, st); break;
      case 6: e = launch<Ozaki<6>>(ta, tb, p, grid, st); break;
      case 7: e = launch<Ozaki<7>>(ta, tb, p, grid, st); break;
      case 8: e = launch<Ozaki<8>>(ta, tb, p, grid, st); break;
      case 9: e = launch<Ozaki<9>>(ta, tb, p, grid, st); break;
      default: return CUCOSMA_STATUS_NOT_SUPPORTED;
    }
    prof_end(st);
    launches += 1;
    if (e == cudaSuccess && pl.splits > 1) {
      const int64_t work = (int64_t)m * n;
      const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(work, 256), di->sms * 8));
      ozaki_reduce_kernel<<<blocks, 256, 0, st>>>((const double*)p.out, p.ws_split_stride, pl.ldw, pl.splits,
                                                  (double*)C, d->ldc, m, n, ea, eb, d->alpha, d->beta, d->epilogue);
      e = cudaGetLastError();
      launches += 1;
    }
  }
  note_launches(launches);
  return e == cudaSuccess ? CUCOSMA_STATUS_SUCCESS : CUCOSMA_STATUS_LAUNCH_FAILED;
}

}  // namespace cucosma
