// skinny.cu -- native-precision GEMM for skinny shapes (see skinny.cuh).
//
// Kind 1, small K (K <= 16): the whole K fits one shared-memory tile; a CTA
// produces a 64-row x (64 * VEC)-column block of C (8 x (256 * VEC) when
// M <= 8), each thread 16 (8) rows x VEC columns with one vector store per
// row.  The kernel is bound by writing C
// (and reading it when beta != 0), the form of 38416 x 38416 x 4 and
// 4 x 3,000,000 x 4.
//
// Kind 2, thin M or N (<= 8) with K > 16: a CTA owns an 8 x 8 output block and
// one K split; its 256 threads stride over K (coalesced reads of the thin
// operand's rows and 32-byte rows of the other), each keeping the 64 partial
// products, then reduce across the CTA in a fixed order.  Splits write raw
// partials that a second kernel sums in a fixed order (the split-K reduction
// of simt_gemm.cu, or one warp per output when there are many splits and few
// outputs), so the result is deterministic.  The form of 4 x 8 x 3,000,000 (the
// reference's SPLIT_K = 320 row), HBM-bound on reading A and B once.
//
// Both accumulate each dot product with FMAs in ascending k and apply
// C = epi(alpha * acc + beta * C) like every other kernel here.
#include <algorithm>

#include "simt_gemm.cuh"
#include "skinny.cuh"

namespace cucosma {

template <typename T, int RG, int RPT>
__global__ void __launch_bounds__(256)
    smallk_kernel(const T* __restrict__ A, int64_t lda, const T* __restrict__ B, int64_t ldb, T* C, int64_t ldc,
                  int m, int n, int k, T alpha, T beta, int epi, int tiles_n, int64_t tiles) {
  // RG row groups of RPT rows x (256 / RG) column groups of VEC columns.  With
  // one row group every B element is used by one thread only, so B is read
  // straight from global memory; otherwise a K x BNS tile is shared.
  constexpr int VEC = Vec<T>::n;
  using V = typename Vec<T>::type;
  constexpr int CG = 256 / RG, BMS = RG * RPT, BNS = CG * VEC;
  constexpr bool SHARE_B = RG > 1;
  __shared__ T As[BMS][skinny::kMaxSmallK + 1];
  __shared__ __align__(16) T Bs[SHARE_B ? skinny::kMaxSmallK : 1][SHARE_B ? BNS : VEC];
  const int tid = threadIdx.x, cg = tid % CG, rg = tid / CG;
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int tm = (int)(t / tiles_n), tn = (int)(t - (int64_t)tm * tiles_n);
    const int m0 = tm * BMS, n0 = tn * BNS;
    __syncthreads();  // the previous block's reads of As / Bs are done
    for (int i = tid; i < BMS * k; i += 256) {
      const int r = i / k, kk = i - r * k;
      As[r][kk] = m0 + r < m ? A[(int64_t)(m0 + r) * lda + kk] : T(0);
    }
    if constexpr (SHARE_B) {
      for (int i = tid; i < k * CG; i += 256) {
        const int kk = i / CG, c = (i - kk * CG) * VEC, col = n0 + c;
        const T* src = B + (int64_t)kk * ldb + col;
        V v;
        T* pv = reinterpret_cast<T*>(&v);
        if (col + VEC <= n) {
          v = *reinterpret_cast<const V*>(src);  // col % VEC == 0 and 16-byte rows
        } else {
#pragma unroll
          for (int e = 0; e < VEC; ++e) pv[e] = col + e < n ? src[e] : T(0);
        }
        *reinterpret_cast<V*>(&Bs[kk][c]) = v;
      }
    }
    __syncthreads();
    const int col = n0 + cg * VEC;
    T acc[RPT][VEC];
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
      for (int e = 0; e < VEC; ++e) acc[r][e] = T(0);
    for (int kk = 0; kk < k; ++kk) {
      V bv;
      if constexpr (SHARE_B) {
        bv = *reinterpret_cast<const V*>(&Bs[kk][cg * VEC]);
      } else {
        const T* src = B + (int64_t)kk * ldb + col;
        T* pb = reinterpret_cast<T*>(&bv);
        if (col + VEC <= n) {
          bv = *reinterpret_cast<const V*>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VEC; ++e) pb[e] = col + e < n ? src[e] : T(0);
        }
      }
      const T* b = reinterpret_cast<const T*>(&bv);
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const T a = As[rg * RPT + r][kk];
#pragma unroll
        for (int e = 0; e < VEC; ++e) acc[r][e] = fma(a, b[e], acc[r][e]);
      }
    }
    if (col >= n) continue;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int row = m0 + rg * RPT + r;
      if (row >= m) break;
      T* o = C + (int64_t)row * ldc + col;
      if (col + VEC <= n) {
        V cv, ov;
        if (beta != T(0)) cv = *reinterpret_cast<const V*>(o);
        const T* pc = reinterpret_cast<const T*>(&cv);
        T* po = reinterpret_cast<T*>(&ov);
#pragma unroll
        for (int e = 0; e < VEC; ++e) po[e] = apply_epi(combine(acc[r][e], alpha, beta, pc + e), epi);
        *reinterpret_cast<V*>(o) = ov;
      } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e)
          if (col + e < n) o[e] = apply_epi(combine(acc[r][e], alpha, beta, o + e), epi);
      }
    }
  }
}

// Thin kernel: each thread takes KV = VEC consecutive k per step (one
// 16-byte load per row of the 8-row A block, KV rows of 8 B values).
template <typename T>
__global__ void __launch_bounds__(256)
    thin_kernel(const T* __restrict__ A, int64_t lda, const T* __restrict__ B, int64_t ldb, T* out, int64_t ldo,
                int m, int n, int k, int64_t kchunk, int groups_n, T alpha, T beta, int epi, int partial,
                int64_t split_stride) {
  constexpr int S = skinny::kThin;
  constexpr int KV = Vec<T>::n;
  using V = typename Vec<T>::type;
  const int gm = blockIdx.x / groups_n, gn = blockIdx.x - gm * groups_n;
  const int m0 = gm * S, n0 = gn * S;
  const int rows = min(S, m - m0), cols = min(S, n - n0);
  const int64_t kb = (int64_t)blockIdx.y * kchunk, ke = min((int64_t)k, kb + kchunk);  // kchunk % KV == 0
  T acc[S][S];
#pragma unroll
  for (int i = 0; i < S; ++i)
#pragma unroll
    for (int j = 0; j < S; ++j) acc[i][j] = T(0);
  for (int64_t k0 = kb + (int64_t)KV * threadIdx.x; k0 < ke; k0 += 256 * KV) {
    T a[S][KV];
    const bool full = k0 + KV <= ke;
#pragma unroll
    for (int i = 0; i < S; ++i) {
      const T* src = A + (int64_t)(m0 + i) * lda + k0;
      if (i < rows && full) {
        const V v = *reinterpret_cast<const V*>(src);  // k0 % KV == 0 and 16-byte rows
        const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int q = 0; q < KV; ++q) a[i][q] = pv[q];
      } else {
#pragma unroll
        for (int q = 0; q < KV; ++q) a[i][q] = (i < rows && k0 + q < ke) ? src[q] : T(0);
      }
    }
#pragma unroll
    for (int q = 0; q < KV; ++q) {
      if (k0 + q >= ke) break;
      T b[S];
      const T* brow = B + (k0 + q) * ldb + n0;
      if (cols == S) {
        // 8 elements from a 16-byte aligned address (n0 % 8 == 0, 16-byte rows)
#pragma unroll
        for (int h = 0; h < S / KV; ++h) {
          const V v = *reinterpret_cast<const V*>(brow + h * KV);
          const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
          for (int e = 0; e < KV; ++e) b[h * KV + e] = pv[e];
        }
      } else {
#pragma unroll
        for (int j = 0; j < S; ++j) b[j] = j < cols ? brow[j] : T(0);
      }
#pragma unroll
      for (int i = 0; i < S; ++i)
#pragma unroll
        for (int j = 0; j < S; ++j) acc[i][j] = fma(a[i][q], b[j], acc[i][j]);
    }
  }
  // Fixed-order reduction: butterfly within each warp, then warps 0..7 in order.
  __shared__ T red[8][S * S];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < S; ++i)
#pragma unroll
    for (int j = 0; j < S; ++j) {
      T x = acc[i][j];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if (lane == 0) red[warp][i * S + j] = x;
    }
  __syncthreads();
  if (threadIdx.x < S * S) {
    const int i = threadIdx.x / S, j = threadIdx.x % S;
    T s = red[0][threadIdx.x];
#pragma unroll
    for (int w = 1; w < 8; ++w) s += red[w][threadIdx.x];
    if (i < rows && j < cols) {
      const int64_t r = m0 + i, c = n0 + j;
      if (partial) {
        out[(int64_t)blockIdx.y * split_stride + r * ldo + c] = s;
      } else {
        T* o = out + r * ldo + c;
        *o = apply_epi(combine(s, alpha, beta, o), epi);
      }
    }
  }
}

// Reduction of many splits for few outputs: one warp per output element,
// lanes sum splits lane, lane + 32, ... in order, then a fixed butterfly --
// deterministic, and not serialised on load latency like a sequential sum
// over hundreds of splits would be.
template <typename T>
__global__ void __launch_bounds__(256)
    thin_reduce_kernel(const T* __restrict__ ws, int64_t split_stride, int64_t ldw, int splits, T* C, int64_t ldc,
                       int m, int n, T alpha, T beta, int epi) {
  const int64_t o = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (o >= (int64_t)m * n) return;
  const int64_t r = o / n, c = o - r * n;
  const T* w = ws + r * ldw + c;
  T s = T(0);
  int z = lane;
  for (; z + 32 * 7 < splits; z += 32 * 8) {  // loads of a batch issued before its adds (order kept)
    T v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = w[(int64_t)(z + 32 * j) * split_stride];
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
  }
  for (; z < splits; z += 32) s += w[(int64_t)z * split_stride];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) {
    T* po = C + r * ldc + c;
    *po = apply_epi(combine(s, alpha, beta, po), epi);
  }
}

SkinnyPlan plan_skinny(int64_t m, int64_t n, int64_t k, int dtype_bytes, int split_k, int tile, int sms) {
  SkinnyPlan p{};
  if (tile == 1 || tile == 2 || m <= 0 || n <= 0 || k <= 0) return p;  // tile ids 1, 2: always the tile kernel
  const int vec = 16 / dtype_bytes;
  if (k <= skinny::kMaxSmallK) {
    p.kind = 1;
    p.splits = 1;
    // 8 x (256 vec) blocks when M <= 8, else 64 x (64 vec)
    p.tile_m = m <= skinny::kThin ? skinny::kThin : 64;
    p.tile_n = m <= skinny::kThin ? 256 * vec : 64 * vec;
    return p;
  }
  if (m > skinny::kThin && n > skinny::kThin) return p;
  p.kind = 2;
  p.tile_m = p.tile_n = skinny::kThin;
  const int64_t groups = ceil_div(m, skinny::kThin) * ceil_div(n, skinny::kThin);
  int64_t splits = split_k > 0 ? split_k : ceil_div(4 * (int64_t)sms, groups);
  splits = std::max<int64_t>(1, std::min<int64_t>({splits, ceil_div(k, 256), 65535}));
  p.kchunk = round_up(ceil_div(k, splits), vec);  // whole 16-byte steps per split
  p.splits = (int)ceil_div(k, p.kchunk);
  p.ldw = round_up(n, vec);
  p.ws_bytes = p.splits > 1 ? (size_t)p.splits * (size_t)m * (size_t)p.ldw * dtype_bytes : 0;
  return p;
}

template <typename T>
cudaError_t launch_skinny(const SkinnyPlan& pl, const T* A, int64_t lda, const T* B, int64_t ldb, T* C, int64_t ldc,
                          int m, int n, int k, double alpha, double beta, int epi, void* ws, int sms,
                          cudaStream_t st) {
  if (pl.kind == 1) {
    const int tiles_n = (int)ceil_div(n, pl.tile_n);
    const int64_t tiles = ceil_div(m, pl.tile_m) * (int64_t)tiles_n;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sms * 8));
    if (pl.tile_m == skinny::kThin)  // M <= 8: one row group, B straight from global memory
      smallk_kernel<T, 1, skinny::kThin><<<(unsigned)grid, 256, 0, st>>>(A, lda, B, ldb, C, ldc, m, n, k, (T)alpha,
                                                                         (T)beta, epi, tiles_n, tiles);
    else
      smallk_kernel<T, 4, 16><<<(unsigned)grid, 256, 0, st>>>(A, lda, B, ldb, C, ldc, m, n, k, (T)alpha, (T)beta, epi,
                                                              tiles_n, tiles);
    return cudaGetLastError();
  }
  const int groups_n = (int)ceil_div(n, skinny::kThin);
  const int64_t groups = ceil_div(m, skinny::kThin) * (int64_t)groups_n;
  const dim3 grid((unsigned)groups, (unsigned)pl.splits);
  if (pl.splits == 1) {
    thin_kernel<T><<<grid, 256, 0, st>>>(A, lda, B, ldb, C, ldc, m, n, k, pl.kchunk, groups_n, (T)alpha, (T)beta, epi,
                                         0, 0);
    return cudaGetLastError();
  }
  T* w = static_cast<T*>(ws);
  const int64_t stride = (int64_t)m * pl.ldw;
  thin_kernel<T><<<grid, 256, 0, st>>>(A, lda, B, ldb, w, pl.ldw, m, n, k, pl.kchunk, groups_n, (T)alpha, (T)beta, epi,
                                       1, stride);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (pl.splits >= 32 && (int64_t)m * n <= (int64_t)sms * 64) {
    thin_reduce_kernel<T><<<(unsigned)ceil_div((int64_t)m * n, 8), 256, 0, st>>>(w, stride, pl.ldw, pl.splits, C, ldc,
                                                                                   m, n, (T)alpha, (T)beta, epi);
    return cudaGetLastError();
  }
  return simt::launch_reduce<T>(w, stride, pl.ldw, pl.splits, C, ldc, m, n, alpha, beta, epi, sms, st);
}

template cudaError_t launch_skinny<float>(const SkinnyPlan&, const float*, int64_t, const float*, int64_t, float*,
                                          int64_t, int, int, int, double, double, int, void*, int, cudaStream_t);
template cudaError_t launch_skinny<double>(const SkinnyPlan&, const double*, int64_t, const double*, int64_t, double*,
                                           int64_t, int, int, int, double, double, int, void*, int, cudaStream_t);

}  // namespace cucosma
