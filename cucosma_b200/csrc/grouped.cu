// grouped.cu -- many uneven GEMMs in one persistent tcgen05 launch.
//
// The reference can only run one compile-time shape per build (config.h:9-31);
// a batch of 512 shapes would be 512 builds.  Here a plan lays every
// problem's operand planes out in the workspace, encodes one pair of TMA
// descriptors per problem, and uploads a table of GroupEntry records.  A
// launch is then:
//   BF16x3 / BF16x6: one table-driven split kernel for the A rows and the B
//                    tiles of every problem + the persistent GEMM kernel;
//   Ozaki:           exponents, slices (both table-driven) + the GEMM kernel.
// The GEMM kernel numbers the tiles of all problems consecutively and each
// CTA walks them round-robin (tc_kernel.cuh, resolve_unit), so small problems
// no longer leave most of the GPU idle the way one launch per problem does.
#include <algorithm>
#include <cstring>
#include <vector>

#include "split_device.cuh"
#include "tc_kernel.cuh"

struct cucosma_grouped_plan_st {
  cucosma_gemm_desc desc;
  int count = 0, kind = 0, slices = 0, total_tiles = 0;
  int tile = 1, tile_m = 128, tile_n = 128, pair = 0, from_cache = 0;
  int pre_a_blocks = 0, pre_b_blocks = 0, exp_a_blocks = 0, exp_b_blocks = 0;
  int device = 0;
  void* workspace = nullptr;
  cucosma::tc::GroupEntry* table = nullptr;  // device copy inside the workspace
};

namespace cucosma {
namespace tc {

// Problem owning pre-pass block b: last entry whose start field is <= b.
template <int FIELD>
__device__ __forceinline__ int find_entry(const GroupEntry* g, int count, int b) {
  auto start = [&](int i) {
    return FIELD == 0 ? g[i].pre_a_start : FIELD == 1 ? g[i].pre_b_start : FIELD == 2 ? g[i].exp_a_start
                                                                                      : g[i].exp_b_start;
  };
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start(mid) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// BF16 split of every problem (NT terms).  Blocks [0, a_blocks): 8 rows of
// some A per block, one warp per row, lanes over 8-column groups (two 16-byte
// loads, one 16-byte store per plane).  Blocks after that: one 64 (k) x 64 (n)
// tile of some B, transposed: 16 lanes load 64 floats of a row; a lane then
// converts 4 consecutive k of one column (one 8-byte store per plane).
template <int NT>
__global__ void __launch_bounds__(256) grouped_split_bf16_kernel(const GroupEntry* __restrict__ g, int count,
                                                                 int a_blocks) {
  __shared__ float tile[64][65];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int b = blockIdx.x;
  if (b < a_blocks) {
    const GroupEntry& e = g[find_entry<0>(g, count, b)];
    const int r = (b - e.pre_a_start) * 8 + warp;
    if (r >= e.m) return;
    const float* src = static_cast<const float*>(e.A) + (int64_t)r * e.lda;
    __nv_bfloat16* dst = static_cast<__nv_bfloat16*>(e.planes_a) + (int64_t)r * e.kpad;
    const int64_t plane = (int64_t)e.m * e.kpad;
    const int nc8 = (int)(e.kpad / 8);
    for (int gi = lane; gi < nc8; gi += 32) {
      const int c = gi * 8;
      float v[8];
      if (c + 8 <= e.k) {
        const float4 q0 = *reinterpret_cast<const float4*>(src + c);  // 16-byte rows, c % 8 == 0
        const float4 q1 = *reinterpret_cast<const float4*>(src + c + 4);
        v[0] = q0.x, v[1] = q0.y, v[2] = q0.z, v[3] = q0.w, v[4] = q1.x, v[5] = q1.y, v[6] = q1.z, v[7] = q1.w;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = c + j < e.k ? src[c + j] : 0.f;
      }
      uint32_t pk[NT][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        __nv_bfloat16 t0[NT], t1[NT];
        split_bf16_n<NT>(v[2 * j], t0);
        split_bf16_n<NT>(v[2 * j + 1], t1);
#pragma unroll
        for (int i = 0; i < NT; ++i) pk[i][j] = pack_bf16x2(t0[i], t1[i]);
      }
#pragma unroll
      for (int i = 0; i < NT; ++i)
        *reinterpret_cast<uint4*>(dst + i * plane + c) = make_uint4(pk[i][0], pk[i][1], pk[i][2], pk[i][3]);
    }
    return;
  }
  b -= a_blocks;
  const GroupEntry& e = g[find_entry<1>(g, count, b)];
  const int t = b - e.pre_b_start;
  const int tiles_n64 = (e.n + 63) / 64;
  const int k0 = (t / tiles_n64) * 64, n0 = (t % tiles_n64) * 64;
  const float* B = static_cast<const float*>(e.B);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = p * 16 + tid / 16, c = (tid % 16) * 4;
    const int k = k0 + i, n = n0 + c;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (k < e.k) {
      const float* src = B + (int64_t)k * e.ldb + n;
      if (n + 4 <= e.n) {
        const float4 q = *reinterpret_cast<const float4*>(src);  // n % 4 == 0, 16-byte rows
        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = n + j < e.n ? src[j] : 0.f;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) tile[i][c + j] = v[j];
  }
  __syncthreads();
  const int64_t plane = (int64_t)e.n * e.kpad;
  __nv_bfloat16* out = static_cast<__nv_bfloat16*>(e.planes_b);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int item = p * 256 + tid, nl = item / 16, kq = item % 16;
    const int n = n0 + nl, k = k0 + kq * 4;
    if (n < e.n && k < e.kpad) {  // kpad % 8 == 0: k + 3 < kpad as well
      uint32_t pk[NT][2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        __nv_bfloat16 t0[NT], t1[NT];
        split_bf16_n<NT>(tile[kq * 4 + 2 * j][nl], t0);
        split_bf16_n<NT>(tile[kq * 4 + 2 * j + 1][nl], t1);
#pragma unroll
        for (int i = 0; i < NT; ++i) pk[i][j] = pack_bf16x2(t0[i], t1[i]);
      }
      __nv_bfloat16* dst = out + (int64_t)n * e.kpad + k;
#pragma unroll
      for (int i = 0; i < NT; ++i) *reinterpret_cast<uint2*>(dst + i * plane) = make_uint2(pk[i][0], pk[i][1]);
    }
  }
}

// Ozaki exponents of every problem: blocks [0, a_blocks) take 8 rows of some
// A (warp per row); the rest take 32 columns of some B (8 thread rows
// striding over K).
__global__ void __launch_bounds__(256) grouped_ozaki_exp_kernel(const GroupEntry* __restrict__ g, int count,
                                                                int a_blocks) {
  __shared__ double red[8][33];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int b = blockIdx.x;
  if (b < a_blocks) {
    const GroupEntry& e = g[find_entry<2>(g, count, b)];
    const int r = (b - e.exp_a_start) * 8 + warp;
    if (r >= e.m) return;
    const double* src = static_cast<const double*>(e.A) + (int64_t)r * e.lda;
    double m = 0.0;
    for (int c = lane; c < e.k; c += 32) m = fmax(m, fabs(src[c]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) const_cast<int32_t*>(e.ea)[r] = exp_of(m);
    return;
  }
  b -= a_blocks;
  const GroupEntry& e = g[find_entry<3>(g, count, b)];
  const int n = (b - e.exp_b_start) * 32 + lane;
  const double* B = static_cast<const double*>(e.B);
  double m = 0.0;
  if (n < e.n)
    for (int k = warp; k < e.k; k += 8) m = fmax(m, fabs(B[(int64_t)k * e.ldb + n]));
  red[warp][lane] = m;
  __syncthreads();
  if (warp == 0 && n < e.n) {
    for (int i = 1; i < 8; ++i) m = fmax(m, red[i][lane]);
    const_cast<int32_t*>(e.eb)[n] = exp_of(m);
  }
}

// Ozaki slices of every problem (A packed, B stacked): blocks [0, a_blocks) take
// 8 rows of some A (warp per row, lanes over 4-column groups); the rest take
// one 32 (k) x 64 (n) tile of some B, transposed.
template <int S>
__global__ void __launch_bounds__(256) grouped_ozaki_slice_kernel(const GroupEntry* __restrict__ g, int count,
                                                                  int a_blocks) {
  __shared__ double tile[32][65];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int b = blockIdx.x;
  if (b < a_blocks) {
    const GroupEntry& e = g[find_entry<0>(g, count, b)];
    const int r = (b - e.pre_a_start) * 8 + warp;
    if (r >= e.m) return;
    const double* src = static_cast<const double*>(e.A) + (int64_t)r * e.lda;
    int8_t* out = static_cast<int8_t*>(e.planes_a);
    const int ex = e.ea[r];
    const int nc4 = (int)(e.kpad / 4);
    for (int gi = lane; gi < nc4; gi += 32) {
      const int c = gi * 4;
      double v[4];
      if (c + 4 <= e.k) {
        const double2 v0 = *reinterpret_cast<const double2*>(src + c);  // 16-byte rows, c % 4 == 0
        const double2 v1 = *reinterpret_cast<const double2*>(src + c + 2);
        v[0] = v0.x, v[1] = v0.y, v[2] = v1.x, v[3] = v1.y;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = c + j < e.k ? src[c + j] : 0.0;
      }
      uint32_t w[S];
      slice4_packed<S>(v, ex, w);
#pragma unroll
      for (int t = 0; t < S; ++t) *reinterpret_cast<uint32_t*>(out + packed_index<S>(r, c, e.kpad, t)) = w[t];
    }
    return;
  }
  // one 32 (k) x 64 (n) tile of some B: 16 lanes load 64 doubles of a row; a
  // lane slices 4 consecutive k of one column (one 4-byte store per slice)
  b -= a_blocks;
  const GroupEntry& e = g[find_entry<1>(g, count, b)];
  const int t = b - e.pre_b_start;
  const int tiles_n64 = (e.n + 63) / 64;
  const int k0 = (t / tiles_n64) * 32, n0 = (t % tiles_n64) * 64;
  const double* B = static_cast<const double*>(e.B);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const int i = p * 16 + tid / 16, c = (tid % 16) * 4;
    const int k = k0 + i, n = n0 + c;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (k < e.k) {
      const double* src = B + (int64_t)k * e.ldb + n;
      if (n + 4 <= e.n) {
        const double2 v0 = *reinterpret_cast<const double2*>(src);
        const double2 v1 = *reinterpret_cast<const double2*>(src + 2);
        v[0] = v0.x, v[1] = v0.y, v[2] = v1.x, v[3] = v1.y;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = n + j < e.n ? src[j] : 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) tile[i][c + j] = v[j];
  }
  __syncthreads();
  int8_t* out = static_cast<int8_t*>(e.planes_b);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const int item = p * 256 + tid, nl = item / 8, kq = item % 8;
    const int n = n0 + nl, k = k0 + kq * 4;
    if (n >= e.n) continue;
    const int ex = e.eb[n];
    const double v[4] = {tile[kq * 4][nl], tile[kq * 4 + 1][nl], tile[kq * 4 + 2][nl], tile[kq * 4 + 3][nl]};
    uint32_t w[S];
    slice4_packed<S>(v, ex, w);
#pragma unroll
    for (int s_ = 0; s_ < S; ++s_) *reinterpret_cast<uint32_t*>(out + stacked_index<S>(n, k, e.n, s_)) = w[s_];
  }
}

// ----------------------------------------------------------------- host
namespace {

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Tile of a grouped launch (descriptor tile id, 0 = the tuner's cached choice
// for this batch, else 1):
//   BF16X3  1 = 128 x 128 promoted, 2 = 128 x 256 promoted, 3 = 256 x 256 CTA pair
//   BF16X6  1 = 128 x 128, 2 = 256 x 256 CTA pair (split release)
//   OZAKI   1 = 128 x ozaki_bn(slices)
struct GTile {
  int id, tile_m, bn, pair;
};
bool grouped_tile(int kind, int slices, int id, GTile& g) {
  if (id == 0) id = 1;
  if (kind == 0 && id >= 1 && id <= 3) {
    g = id == 1 ? GTile{1, 128, 128, 0} : id == 2 ? GTile{2, 128, 256, 0} : GTile{3, 256, 256, 1};
    return true;
  }
  if (kind == 1 && id >= 1 && id <= 2) {
    g = id == 1 ? GTile{1, 128, 128, 0} : GTile{2, 256, 256, 1};
    return true;
  }
  if (kind == 2 && id == 1) {
    g = GTile{1, 128, ozaki_bn(slices), 0};
    return true;
  }
  return false;
}

struct Layout {
  int kind, slices, bn, tile_m, pair, tile;
  size_t table_bytes, total_bytes;
  std::vector<GroupEntry> entries;  // pointers relative to the workspace base (offsets)
  std::vector<size_t> off_a, off_b, off_ea, off_eb;
  int total_tiles, pre_a, pre_b, exp_a, exp_b;
};

cucosma_status layout(const cucosma_gemm_desc* d, const cucosma_gemm_problem* pr, int count, Layout& L,
                      int tile = -1) {
  if (!d || !pr || count <= 0) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->flags != 0 || d->epilogue < 0 || d->epilogue > CUCOSMA_EPILOGUE_RELU) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->precision == CUCOSMA_PRECISION_OZAKI) {
    if (d->dtype != CUCOSMA_R_64F) return CUCOSMA_STATUS_NOT_SUPPORTED;
    L.kind = 2;
    L.slices = d->slices ? d->slices : kOzakiDefaultSlices;
    if (L.slices < 4 || L.slices > 9) return CUCOSMA_STATUS_NOT_SUPPORTED;
  } else if (d->precision == CUCOSMA_PRECISION_BF16X3 || d->precision == CUCOSMA_PRECISION_BF16X6) {
    if (d->dtype != CUCOSMA_R_32F) return CUCOSMA_STATUS_NOT_SUPPORTED;
    L.kind = d->precision == CUCOSMA_PRECISION_BF16X6 ? 1 : 0;
    L.slices = L.kind == 1 ? 3 : 2;
  } else {
    return CUCOSMA_STATUS_NOT_SUPPORTED;  // the grouped launch is a tensor-core path
  }
  GTile g{};
  if (!grouped_tile(L.kind, L.slices, tile >= 0 ? tile : d->tile, g)) return CUCOSMA_STATUS_NOT_SUPPORTED;
  L.bn = g.bn;
  L.tile_m = g.tile_m;
  L.pair = g.pair;
  L.tile = g.id;
  const int es_in = L.kind == 2 ? 8 : 4;
  const int es_pl = L.kind == 2 ? 1 : 2;
  const int64_t kmax_exact = ((int64_t)2147483647 / ((int64_t)L.slices * 127 * 127)) / 32 * 32;
  L.table_bytes = al256(sizeof(GroupEntry) * (size_t)count);
  size_t off = L.table_bytes;
  L.entries.assign(count, GroupEntry{});
  L.off_a.resize(count);
  L.off_b.resize(count);
  L.off_ea.resize(count);
  L.off_eb.resize(count);
  // Table order: K descending (stable).  The persistent kernel hands units out
  // round-robin in table order, so the long-K tiles are spread over the CTAs
  // first and the short ones even out the end.
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pr[a].k > pr[b].k; });
  int tiles = 0, pa = 0, pb = 0, xa = 0, xb = 0;
  for (int i = 0; i < count; ++i) {
    const cucosma_gemm_problem& q = pr[order[i]];
    if (q.m <= 0 || q.n <= 0 || q.k <= 0) return CUCOSMA_STATUS_INVALID_VALUE;
    if (q.m > INT32_MAX || q.n > INT32_MAX || q.k > INT32_MAX) return CUCOSMA_STATUS_INVALID_VALUE;
    if (q.lda < q.k || q.ldb < q.n || q.ldc < q.n || !q.A || !q.B || !q.C) return CUCOSMA_STATUS_INVALID_VALUE;
    if ((reinterpret_cast<uintptr_t>(q.A) | reinterpret_cast<uintptr_t>(q.B) | reinterpret_cast<uintptr_t>(q.C)) & 15)
      return CUCOSMA_STATUS_MISALIGNED;
    if ((q.lda * es_in) % 16 || (q.ldb * es_in) % 16 || (q.ldc * es_in) % 16) return CUCOSMA_STATUS_MISALIGNED;
    if (L.kind == 2 && q.k > kmax_exact) return CUCOSMA_STATUS_NOT_SUPPORTED;  // no split-K in grouped launches
    GroupEntry& e = L.entries[i];
    e.m = (int)q.m;
    e.n = (int)q.n;
    e.k = (int)q.k;
    e.kpad = L.kind == 2 ? round_up(q.k, 32) : round_up(q.k, 8);
    e.kblocks = (int)ceil_div(q.k, 32);
    e.tiles_m = (int)ceil_div(q.m, L.tile_m);
    e.tiles_n = (int)ceil_div(q.n, L.bn);
    e.tile_start = tiles;
    tiles += e.tiles_m * e.tiles_n;
    e.C = q.C;
    e.ldc = q.ldc;
    e.A = q.A;
    e.B = q.B;
    e.lda = q.lda;
    e.ldb = q.ldb;
    e.pre_a_start = pa;
    pa += (int)ceil_div(q.m, 8);
    e.pre_b_start = pb;
    pb += L.kind == 2 ? (int)(ceil_div(e.kpad, 32) * ceil_div(q.n, 64)) : (int)(ceil_div(e.kpad, 64) * ceil_div(q.n, 64));
    e.exp_a_start = xa;
    xa += (int)ceil_div(q.m, 8);
    e.exp_b_start = xb;
    xb += (int)ceil_div(q.n, 32);
    L.off_a[i] = off;
    off = al256(off + (size_t)L.slices * q.m * e.kpad * es_pl);
    L.off_b[i] = off;
    off = al256(off + (size_t)L.slices * q.n * e.kpad * es_pl);
    if (L.kind == 2) {
      L.off_ea[i] = off;
      off = al256(off + (size_t)q.m * 4);
      L.off_eb[i] = off;
      off = al256(off + (size_t)q.n * 4);
    }
  }
  L.total_tiles = tiles;
  L.pre_a = pa;
  L.pre_b = pb;
  L.exp_a = xa;
  L.exp_b = xb;
  L.total_bytes = off;
  return CUCOSMA_STATUS_SUCCESS;
}

}  // namespace
}  // namespace tc
}  // namespace cucosma

using namespace cucosma;
using namespace cucosma::tc;

extern "C" cucosma_status cucosma_grouped_workspace_size(const cucosma_gemm_desc* d,
                                                         const cucosma_gemm_problem* problems, int count,
                                                         size_t* bytes) {
  if (!bytes) return CUCOSMA_STATUS_INVALID_VALUE;
  Layout L;
  cucosma_status s = layout(d, problems, count, L);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  *bytes = L.total_bytes;
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_grouped_plan_create(const cucosma_gemm_desc* d,
                                                      const cucosma_gemm_problem* problems, int count,
                                                      void* workspace, size_t workspace_bytes,
                                                      cucosma_grouped_plan* plan) {
  if (!plan) return CUCOSMA_STATUS_INVALID_VALUE;
  *plan = nullptr;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (di->cc_major != 10 || di->cc_minor != 0) return CUCOSMA_STATUS_ARCH_MISMATCH;
  // tile 0: the tuner's choice for this batch of shapes, when it has one
  int tile = d ? d->tile : 0, from_cache = 0;
  if (d && tile == 0) {
    tile = grouped_tuned_tile(d, problems, count, di);
    from_cache = tile > 0;
  }
  Layout L;
  cucosma_status s = layout(d, problems, count, L, tile);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (!workspace || workspace_bytes < L.total_bytes) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  if (reinterpret_cast<uintptr_t>(workspace) & 255) return CUCOSMA_STATUS_MISALIGNED;
  uint8_t* w = static_cast<uint8_t*>(workspace);
  for (int i = 0; i < count; ++i) {
    GroupEntry& e = L.entries[i];
    e.planes_a = w + L.off_a[i];
    e.planes_b = w + L.off_b[i];
    const int s_ = L.slices;
    bool ok;
    if (L.kind == 2) {
      e.ea = reinterpret_cast<int32_t*>(w + L.off_ea[i]);
      e.eb = reinterpret_cast<int32_t*>(w + L.off_eb[i]);
      const uint64_t kbs = (uint64_t)e.kpad / 32;
      ok = encode_3d(&e.tmA, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, e.planes_a, 32ull * s_, kbs, e.m, 32ull * s_,
                     (uint64_t)e.kpad * s_, 128, 1, 128, CU_TENSOR_MAP_SWIZZLE_128B) &&
           encode_3d(&e.tmB, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, e.planes_b, 32, e.n, kbs * s_, 32, 32ull * e.n, 32,
                     ozaki_sub(s_), s_, CU_TENSOR_MAP_SWIZZLE_32B);
    } else {
      ok = encode_3d(&e.tmA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, e.planes_a, e.k, e.m, s_, e.kpad,
                     (uint64_t)e.m * e.kpad, 32, 128, s_, CU_TENSOR_MAP_SWIZZLE_64B) &&
           encode_3d(&e.tmB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, e.planes_b, e.k, e.n, s_, e.kpad,
                     (uint64_t)e.n * e.kpad, 32, L.pair ? L.bn / 2 : L.bn, s_, CU_TENSOR_MAP_SWIZZLE_64B);
    }
    if (!ok) return CUCOSMA_STATUS_LAUNCH_FAILED;
  }
  if (cudaMemcpy(workspace, L.entries.data(), sizeof(GroupEntry) * (size_t)count, cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  auto* p = new cucosma_grouped_plan_st;
  p->desc = *d;
  p->count = count;
  p->kind = L.kind;
  p->slices = L.slices;
  p->total_tiles = L.total_tiles;
  p->tile = L.tile;
  p->tile_m = L.tile_m;
  p->tile_n = L.bn;
  p->pair = L.pair;
  p->from_cache = from_cache;
  p->pre_a_blocks = L.pre_a;
  p->pre_b_blocks = L.pre_b;
  p->exp_a_blocks = L.exp_a;
  p->exp_b_blocks = L.exp_b;
  cudaGetDevice(&p->device);
  p->workspace = workspace;
  p->table = reinterpret_cast<GroupEntry*>(workspace);
  *plan = p;
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_grouped_plan_destroy(cucosma_grouped_plan plan) {
  delete plan;
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_grouped_plan_get_tile(cucosma_grouped_plan plan, int32_t* tile, int32_t* tile_m,
                                                       int32_t* tile_n, int32_t* from_cache) {
  if (!plan) return CUCOSMA_STATUS_INVALID_VALUE;
  if (tile) *tile = plan->tile;
  if (tile_m) *tile_m = plan->tile_m;
  if (tile_n) *tile_n = plan->tile_n;
  if (from_cache) *from_cache = plan->from_cache;
  return CUCOSMA_STATUS_SUCCESS;
}

template <int S>
static cudaError_t launch_ozaki_grouped(const cucosma_grouped_plan_st& pl, const TcParams& p, const CUtensorMap& dummy,
                                        int grid, cudaStream_t st) {
  grouped_ozaki_slice_kernel<S><<<pl.pre_a_blocks + pl.pre_b_blocks, 256, 0, st>>>(pl.table, pl.count,
                                                                                   pl.pre_a_blocks);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  prof_begin(st);
  e = launch<Ozaki<S>>(dummy, dummy, p, grid, st);
  prof_end(st);
  return e;
}

extern "C" cucosma_status cucosma_gemm_grouped(cucosma_grouped_plan plan, void* stream) {
  if (!plan) return CUCOSMA_STATUS_INVALID_VALUE;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  TcParams p{};
  p.skip_stage = -1;
  p.epilogue = plan->desc.epilogue;
  p.alpha = plan->desc.alpha;
  p.beta = plan->desc.beta;
  p.groups = plan->table;
  p.ngroups = plan->count;
  p.total_tiles = plan->total_tiles;
  p.splits = 1;
  wait_ctl(di, &p.ctl.status, &p.ctl.timeout_ns);
  const int grid = std::min(plan->total_tiles, di->sms);
  CUtensorMap dummy;
  std::memset(&dummy, 0, sizeof(dummy));
  cudaError_t e;
  if (plan->kind != 2) {
    const unsigned blocks = (unsigned)(plan->pre_a_blocks + plan->pre_b_blocks);
    if (plan->slices == 3)
      grouped_split_bf16_kernel<3><<<blocks, 256, 0, st>>>(plan->table, plan->count, plan->pre_a_blocks);
    else
      grouped_split_bf16_kernel<2><<<blocks, 256, 0, st>>>(plan->table, plan->count, plan->pre_a_blocks);
    e = cudaGetLastError();
    if (e != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    auto pair_grid = [&](int clusters) { return 2 * std::max(1, std::min(plan->total_tiles, clusters)); };
    prof_begin(st);
    if (plan->kind == 1)
      e = plan->tile == 2
              ? launch<Bf16x6PairWide>(dummy, dummy, p, pair_grid(max_pair_clusters<Bf16x6PairWide>(di->sms)), st)
              : launch<Bf16x6>(dummy, dummy, p, grid, st);
    else
      e = plan->tile == 3   ? launch<Bf16x3Pair>(dummy, dummy, p, pair_grid(max_pair_clusters<Bf16x3Pair>(di->sms)), st)
          : plan->tile == 2 ? launch<Bf16x3>(dummy, dummy, p, grid, st)
                            : launch<Bf16x3Promoted>(dummy, dummy, p, grid, st);
    prof_end(st);
    note_launches(2);
  } else {
    grouped_ozaki_exp_kernel<<<plan->exp_a_blocks + plan->exp_b_blocks, 256, 0, st>>>(plan->table, plan->count,
                                                                                      plan->exp_a_blocks);
    e = cudaGetLastError();
    if (e != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
    switch (plan->slices) {
      case 4: e = launch_ozaki_grouped<4>(*plan, p, dummy, grid, st); break;
      case 5: e = launch_ozaki_grouped<5>(*plan, p, dummy, grid, st); break;
      case 6: e = launch_ozaki_grouped<6>(*plan, p, dummy, grid, st); break;
      case 7: e = launch_ozaki_grouped<7>(*plan, p, dummy, grid, st); break;
      case 8: e = launch_ozaki_grouped<8>(*plan, p, dummy, grid, st); break;
      case 9: e = launch_ozaki_grouped<9>(*plan, p, dummy, grid, st); break;
      default: return CUCOSMA_STATUS_NOT_SUPPORTED;
    }
    note_launches(3);
  }
  return e == cudaSuccess ? CUCOSMA_STATUS_SUCCESS : CUCOSMA_STATUS_LAUNCH_FAILED;
}
