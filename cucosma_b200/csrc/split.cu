// split.cu -- operand pre-passes of the tensor-core precision paths.
//
// BF16 split (BF16x3 / BF16x6 SGEMM): every FP32 entry x becomes terms
// t0 + t1 (+ t2) with t_i = RN_bf16(x - t0 - ... - t_{i-1}); each residual
// subtraction is exact in FP32.  A (M x K, row-major) keeps its layout;
// B (K x N, row-major) is written transposed (N x K) so that both operands
// are K-major for the tensor cores.  Planes: [nterms][rows][kpad].
//
// Ozaki slicing (INT8 DGEMM): per row of A / per column of B the exponent
// e with |x| < 2^e over the row / column; x * 2^-e is cut into s signed
// 7-bit integer slices q_t = trunc(r * 2^7), r <- r * 2^7 - q_t, exact in
// FP64.  Slices of A rows are stored packed (packed_index), those of B
// columns stacked (stacked_index); kpad = K rounded up to the 32-wide k-block.
//
// All pre-passes are HBM-bound elementwise / transpose kernels.
#include <cuda_bf16.h>

#include "split.cuh"
#include "split_device.cuh"

namespace cucosma {

// ------------------------------------------------------------------ BF16
// Loads v[0..7] = src[c .. c+7] (zero past cols); c % 8 == 0 and src rows
// 16-byte aligned, so the full case is two 16-byte loads.
__device__ __forceinline__ void load8(const float* __restrict__ src, int c, int cols, float (&v)[8]) {
  if (c + 8 <= cols) {
    const float4 a = *reinterpret_cast<const float4*>(src + c);
    const float4 b = *reinterpret_cast<const float4*>(src + c + 4);
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
  } else {
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = c + e < cols ? src[c + e] : 0.f;
  }
}

// A: rows x cols (ld elements) -> planes [NT][rows][kpad], same layout.
// Rows stride over grid.y, 8-column groups over grid.x; each thread converts
// 8 consecutive columns (two 16-byte loads, one 16-byte store per plane).
// Columns cols..kpad-1 are written as 0 (kpad % 8 == 0).
template <int MODE, int NT>
__global__ void __launch_bounds__(256)
    split_bf16_rows_kernel(const float* __restrict__ A, int64_t lda, int rows, int cols, int64_t kpad,
                           __nv_bfloat16* __restrict__ out, const float* __restrict__ Y, int64_t ldy, float scale) {
  const int ng = (int)(kpad / 8);
  const int64_t plane = (int64_t)rows * kpad;
  for (int r = blockIdx.y; r < rows; r += gridDim.y) {
    const float* srow = A + (int64_t)r * lda;
    __nv_bfloat16* drow = out + (int64_t)r * kpad;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
      const int c = g * 8;
      float v[8];
      load8(srow, c, cols, v);
      if constexpr (MODE != kXformNone) {
        float y[8];
        load8(Y + (int64_t)r * ldy, c, cols, y);
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = xform<MODE>(v[e], y[e], scale);
      }
      uint32_t pk[NT][4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        __nv_bfloat16 t0[NT], t1[NT];
        split_bf16_n<NT>(v[2 * e], t0);
        split_bf16_n<NT>(v[2 * e + 1], t1);
#pragma unroll
        for (int i = 0; i < NT; ++i) pk[i][e] = pack_bf16x2(t0[i], t1[i]);
      }
#pragma unroll
      for (int i = 0; i < NT; ++i)
        *reinterpret_cast<uint4*>(drow + i * plane + c) = make_uint4(pk[i][0], pk[i][1], pk[i][2], pk[i][3]);
    }
  }
}

// B: K x N (ld elements) -> planes [NT][N][kpad] (transposed), through a
// 64 (k) x 64 (n) shared-memory tile; 256 threads.  Loads: 16 lanes cover a
// 256-byte row of B (float4 each).  Stores: a lane converts 4 consecutive k
// of one output row (8 bytes per plane), so 16 lanes write 128 contiguous
// bytes per plane.
template <int MODE, int NT>
__global__ void __launch_bounds__(256)
    split_bf16_cols_kernel(const float* __restrict__ B, int64_t ldb, int krows, int ncols, int64_t kpad,
                           __nv_bfloat16* __restrict__ out, const float* __restrict__ Y, int64_t ldy, float scale) {
  __shared__ float tile[64][65];
  const int k0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const int64_t plane = (int64_t)ncols * kpad;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;  // 16 x 16
#pragma unroll
  for (int i = ty; i < 64; i += 16) {
    const int k = k0 + i, n = n0 + 4 * tx;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (k < krows) {
      const float* src = B + (int64_t)k * ldb + n;
      if (n + 4 <= ncols) {
        const float4 q = *reinterpret_cast<const float4*>(src);  // n % 4 == 0, ldb % 4 == 0
        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = n + e < ncols ? src[e] : 0.f;
      }
      if constexpr (MODE != kXformNone) {
        const float* ysrc = Y + (int64_t)k * ldy + n;
        float y[4] = {0.f, 0.f, 0.f, 0.f};
        if (n + 4 <= ncols) {
          const float4 q = *reinterpret_cast<const float4*>(ysrc);
          y[0] = q.x, y[1] = q.y, y[2] = q.z, y[3] = q.w;
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) y[e] = n + e < ncols ? ysrc[e] : 0.f;
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = xform<MODE>(v[e], y[e], scale);
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) tile[i][4 * tx + e] = v[e];
  }
  __syncthreads();
  const int k = k0 + 4 * tx;
#pragma unroll
  for (int i = ty; i < 64; i += 16) {
    const int n = n0 + i;
    if (n < ncols && k < kpad) {  // kpad % 8 == 0, so k + 3 < kpad as well
      uint32_t pk[NT][2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        __nv_bfloat16 t0[NT], t1[NT];
        split_bf16_n<NT>(tile[4 * tx + 2 * e][i], t0);
        split_bf16_n<NT>(tile[4 * tx + 2 * e + 1][i], t1);
#pragma unroll
        for (int j = 0; j < NT; ++j) pk[j][e] = pack_bf16x2(t0[j], t1[j]);
      }
      __nv_bfloat16* dst = out + (int64_t)n * kpad + k;
#pragma unroll
      for (int j = 0; j < NT; ++j) *reinterpret_cast<uint2*>(dst + j * plane) = make_uint2(pk[j][0], pk[j][1]);
    }
  }
}

// ----------------------------------------------------------------- Ozaki
// Column exponents of B start at this sentinel (a byte memset); columns that
// are all zero keep it until ozaki_rows_kernel turns it into exp_of(0) = 0.
constexpr int32_t kExpSentinel = (int32_t)0x80808080;

// Column exponents of B (K x N): a block covers 64 rows of K and 512 columns
// (two per thread, 16-byte loads).  Each block's column maxima enter eb by
// atomicMax of their exponents -- exact, since the exponent of a maximum is
// the maximum of the exponents (frexp is monotonic in |x|); zero maxima stay
// out so that they cannot raise a column's exponent.
__global__ void __launch_bounds__(256)
    ozaki_col_exp_kernel(const double* __restrict__ B, int64_t ldb, int krows, int ncols, int32_t* eb) {
  const int c = (blockIdx.x * 256 + threadIdx.x) * 2;
  const int k0 = blockIdx.y * 64, k1 = min(krows, k0 + 64);
  if (c >= ncols) return;
  double m0 = 0.0, m1 = 0.0;
  if (c + 1 < ncols) {
#pragma unroll 8
    for (int k = k0; k < k1; ++k) {
      const double2 v = *reinterpret_cast<const double2*>(B + (int64_t)k * ldb + c);  // c even, 16-byte rows
      m0 = fmax(m0, fabs(v.x));
      m1 = fmax(m1, fabs(v.y));
    }
  } else {
    for (int k = k0; k < k1; ++k) m0 = fmax(m0, fabs(B[(int64_t)k * ldb + c]));
  }
  if (m0 != 0.0) atomicMax(&eb[c], exp_of(m0));
  if (c + 1 < ncols && m1 != 0.0) atomicMax(&eb[c + 1], exp_of(m1));
}

// A rows of up to kRowRegK padded columns -> row exponents and packed
// slices: a 256-thread block per row.  The row is read once into registers
// (4 consecutive columns per thread and step, two 16-byte loads), the
// maximum is reduced across the block, and the slices are cut from the
// registers; a thread's 4 columns give one 4-byte store per slice.  With
// rowsum, also the row's magnitude sum sum_k floor(|a_rk| 2^(30 - e_r))
// (integer, so exact and order-free) into rowsum[r].  Longer rows take the
// chunked kernels below.
constexpr int kRowSteps = 8;                    // steps of 1024 columns held in registers
constexpr int kRowRegK = kRowSteps * 1024;
static_assert(kRowRegK == kOzakiRowChunk, "row chunk");

__device__ __forceinline__ void load4(const double* __restrict__ src, int c, int cols, double (&v)[4]) {
  if (c + 4 <= cols) {
    const double2 v0 = *reinterpret_cast<const double2*>(src + c);  // c % 4 == 0, 16-byte rows
    const double2 v1 = *reinterpret_cast<const double2*>(src + c + 2);
    v[0] = v0.x, v[1] = v0.y, v[2] = v1.x, v[3] = v1.y;
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = c + j < cols ? src[c + j] : 0.0;
  }
}

// Slices of 4 consecutive columns of row r (one 4-byte store per slice);
// returns their magnitude sum (see slice4_packed).
template <int S>
__device__ __forceinline__ unsigned long long store_slices4(int8_t* __restrict__ out, int64_t r, int c, int64_t kpad,
                                                            const double (&v)[4], int e) {
  uint32_t w[S];
  const unsigned long long mag = slice4_packed<S>(v, e, w);
#pragma unroll
  for (int t = 0; t < S; ++t) *reinterpret_cast<uint32_t*>(out + packed_index<S>(r, c, kpad, t)) = w[t];
  return mag;
}

template <int S>
__global__ void __launch_bounds__(256)
    ozaki_rows_kernel(const double* __restrict__ A, int64_t lda, int rows, int cols, int64_t kpad,
                      int32_t* __restrict__ ea, int8_t* __restrict__ out, unsigned long long* __restrict__ rowsum) {
  const bool stats = rowsum != nullptr;
  __shared__ double red[8];
  __shared__ unsigned long long red_sum[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const double* src = A + (int64_t)r * lda;
    double v[kRowSteps][4];
    double m = 0.0;
#pragma unroll
    for (int j = 0; j < kRowSteps; ++j) {
      const int c = (tid + 256 * j) * 4;
      if (c < kpad) {
        load4(src, c, cols, v[j]);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) v[j][q] = 0.0;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) m = fmax(m, fabs(v[j][q]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) red[warp] = m;
    __syncthreads();
    m = red[0];
#pragma unroll
    for (int w = 1; w < 8; ++w) m = fmax(m, red[w]);
    __syncthreads();  // red is reused by the next row
    const int e = exp_of(m);
    if (tid == 0) ea[r] = e;
    unsigned long long sum = 0;
#pragma unroll
    for (int j = 0; j < kRowSteps; ++j) {
      const int c = (tid + 256 * j) * 4;
      if (c < kpad) {
        const unsigned long long mg = store_slices4<S>(out, r, c, kpad, v[j], e);
        if (stats) sum += mg;
      }
    }
    if (stats) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0) red_sum[warp] = sum;
      __syncthreads();
      if (tid == 0) {
        unsigned long long t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += red_sum[w];
        rowsum[r] = t;
      }
      __syncthreads();  // red_sum is reused by the next row
    }
  }
}

// Rows longer than kRowRegK in chunks of kRowRegK columns (grid.x chunks,
// rows over grid.y), so that a few long rows still fill the GPU.  The first
// kernel takes each chunk's maximum into ea[r] by atomicMax of its exponent
// (ea starts at kExpSentinel; the exponent of a maximum is the maximum of
// the exponents, so this is exact); the second cuts the chunk's slices and
// adds its magnitude sum into rowsum[r] (integer atomics: exact and
// independent of the order of the blocks).  Rows that are all zero keep the
// sentinel until the second kernel's first chunk turns it into 0; every
// block reads the sentinel as 0.
__global__ void __launch_bounds__(256)
    ozaki_row_exp_kernel(const double* __restrict__ A, int64_t lda, int rows, int cols, int32_t* __restrict__ ea) {
  __shared__ double red[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.x * kRowRegK;
  for (int r = blockIdx.y; r < rows; r += gridDim.y) {
    const double* src = A + (int64_t)r * lda;
    double m = 0.0;
#pragma unroll
    for (int j = 0; j < kRowSteps; ++j) {
      const int c = c0 + (tid + 256 * j) * 4;
      if (c < cols) {
        double w[4];
        load4(src, c, cols, w);
#pragma unroll
        for (int q = 0; q < 4; ++q) m = fmax(m, fabs(w[q]));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) red[warp] = m;
    __syncthreads();
    m = red[0];
#pragma unroll
    for (int w = 1; w < 8; ++w) m = fmax(m, red[w]);
    __syncthreads();  // red is reused by the next row
    if (tid == 0 && m != 0.0) atomicMax(&ea[r], exp_of(m));
  }
}

template <int S>
__global__ void __launch_bounds__(256)
    ozaki_row_slice_kernel(const double* __restrict__ A, int64_t lda, int rows, int cols, int64_t kpad,
                           int32_t* __restrict__ ea, int8_t* __restrict__ out, unsigned long long* __restrict__ rowsum) {
  __shared__ unsigned long long red_sum[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.x * kRowRegK;
  for (int r = blockIdx.y; r < rows; r += gridDim.y) {
    const double* src = A + (int64_t)r * lda;
    int e = ea[r];
    if (e == kExpSentinel) {
      e = 0;
      if (blockIdx.x == 0 && tid == 0) ea[r] = 0;
    }
    unsigned long long sum = 0;
#pragma unroll
    for (int j = 0; j < kRowSteps; ++j) {
      const int c = c0 + (tid + 256 * j) * 4;
      if (c < kpad) {
        double w[4];
        load4(src, c, cols, w);
        const unsigned long long mg = store_slices4<S>(out, r, c, kpad, w, e);
        if (rowsum) sum += mg;
      }
    }
    if (rowsum) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0) red_sum[warp] = sum;
      __syncthreads();
      if (tid == 0) {
        unsigned long long t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += red_sum[w];
        if (t) atomicAdd(&rowsum[r], t);
      }
      __syncthreads();  // red_sum is reused by the next row
    }
  }
}

// B (K x N) -> stacked slices of its columns, through a 64 (k) x 64 (n)
// shared-memory tile (two 32-wide k-blocks: eight 16-byte loads per thread
// in flight before the barrier).  Loads: 16 lanes cover 64 doubles of a row
// of B.  Stores, per k-block: a lane slices 4 consecutive k of one column
// into one 4-byte store per slice; 8 lanes cover a column's 32 bytes and a
// warp 4 adjacent columns (128 contiguous bytes per slice).  The second
// k-block of the last tile may lie past kpad and is then skipped.
// Also finishes the column exponents (the blocks of the first k-tile turn
// the all-zero columns' sentinel into exp_of(0) = 0; every block reads the
// sentinel as 0) and, with colsum, adds each column's fixed-point magnitude
// sum sum_k floor(|b_kn| 2^(30 - e_n)) by integer atomics (exact, so the
// totals do not depend on the order of the blocks).
constexpr int kColTileK = 64;

template <int S>
__global__ void __launch_bounds__(256)
    ozaki_slice_cols_kernel(const double* __restrict__ B, int64_t ldb, int krows, int ncols, int64_t kpad,
                            int32_t* __restrict__ eb, int8_t* __restrict__ out, unsigned long long* __restrict__ colsum) {
  __shared__ double tile[kColTileK][65];
  const int k0 = blockIdx.y * kColTileK, n0 = blockIdx.x * 64, t = threadIdx.x;
#pragma unroll
  for (int p = 0; p < kColTileK / 16; ++p) {
    const int i = p * 16 + t / 16, c = (t % 16) * 4;
    const int k = k0 + i, n = n0 + c;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (k < krows) {
      const double* src = B + (int64_t)k * ldb + n;
      if (n + 4 <= ncols) {
        const double2 v0 = *reinterpret_cast<const double2*>(src);
        const double2 v1 = *reinterpret_cast<const double2*>(src + 2);
        v[0] = v0.x, v[1] = v0.y, v[2] = v1.x, v[3] = v1.y;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = n + j < ncols ? src[j] : 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) tile[i][c + j] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int p = 0; p < kColTileK / 16; ++p) {
    const int half = p >> 1;  // k-block of the tile
    const int item = (p & 1) * 256 + t, nl = item / 8, kq = item % 8;
    const int n = n0 + nl, kl = half * 32 + kq * 4, k = k0 + kl;
    if (k0 + half * 32 >= kpad) break;  // past the last k-block (uniform over the block)
    unsigned long long part = 0;
    if (n < ncols) {
      int e = eb[n];
      if (e == kExpSentinel) {
        e = 0;
        if (blockIdx.y == 0 && kl == 0) eb[n] = 0;
      }
      const double v[4] = {tile[kl][nl], tile[kl + 1][nl], tile[kl + 2][nl], tile[kl + 3][nl]};
      uint32_t w[S];
      const unsigned long long mg = slice4_packed<S>(v, e, w);
#pragma unroll
      for (int s_ = 0; s_ < S; ++s_) *reinterpret_cast<uint32_t*>(out + stacked_index<S>(n, k, ncols, s_)) = w[s_];
      if (colsum) part = mg;
    }
    if (colsum) {
      // the 8 lanes of a column are consecutive: reduce over them
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (kq == 0 && n < ncols && part) atomicAdd(&colsum[n], part);
    }
  }
}

// Minima of the row and column magnitude sums over the nonzero rows and
// columns into stats->min_row / min_col; the last block to finish then
// makes the path choice (see ozaki_choice) from both minima.
__device__ __forceinline__ unsigned long long block_min_nonzero(const unsigned long long* __restrict__ v, int count,
                                                                unsigned long long* red) {
  unsigned long long m = ~0ull;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const unsigned long long x = v[i];
    if (x != 0 && x < m) m = x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
    m = w < m ? w : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  for (int w = 0; w < 8; ++w) m = red[w] < m ? red[w] : m;
  __syncthreads();  // red is reused
  return m;
}

__global__ void __launch_bounds__(256) ozaki_decide_kernel(const unsigned long long* __restrict__ rowsum, int nrows,
                                                           const unsigned long long* __restrict__ colsum, int ncols,
                                                           int64_t k, OzakiStats* stats) {
  __shared__ unsigned long long red[8];
  const unsigned long long mrow = block_min_nonzero(rowsum, nrows, red);
  const unsigned long long m = block_min_nonzero(colsum, ncols, red);
  if (threadIdx.x == 0) {
    if (mrow != ~0ull) atomicMin(&stats->min_row, mrow);
    if (m != ~0ull) atomicMin(&stats->min_col, m);
    __threadfence();
    const unsigned prev = atomicAdd(&stats->done_blocks, 1u);
    if (prev == gridDim.x - 1) {
      __threadfence();
      const unsigned long long mr = atomicAdd(&stats->min_row, 0ull), mc = atomicAdd(&stats->min_col, 0ull);
      stats->choice = ozaki_choice(mr, mc, k);
    }
  }
}

// ---------------------------------------------------------------- launch
static unsigned grid_for(int64_t work, int threads, int sms) {
  int64_t b = ceil_div(work, threads);
  b = std::min<int64_t>(b, (int64_t)sms * 16);
  return (unsigned)std::max<int64_t>(b, 1);
}

template <int MODE, int NT>
static void split_bf16_launch_nt(const float* A, int64_t lda, int rows, int cols, int64_t kpad, void* out,
                                 bool transpose, int sms, cudaStream_t st, const float* Y, int64_t ldy, float scale) {
  if (!transpose) {
    const int64_t gx = std::max<int64_t>(1, std::min<int64_t>(ceil_div(kpad / 8, 256), 16));
    const int64_t gy = std::max<int64_t>(1, std::min<int64_t>({(int64_t)rows, (int64_t)sms * 16 / gx, 65535}));
    split_bf16_rows_kernel<MODE, NT><<<dim3((unsigned)gx, (unsigned)gy), 256, 0, st>>>(
        A, lda, rows, cols, kpad, static_cast<__nv_bfloat16*>(out), Y, ldy, scale);
  } else {
    // A is K x N here (krows = rows, ncols = cols); output N x kpad.
    dim3 grid((unsigned)ceil_div(cols, 64), (unsigned)ceil_div(kpad, 64));
    split_bf16_cols_kernel<MODE, NT><<<grid, 256, 0, st>>>(A, lda, rows, cols, kpad,
                                                          static_cast<__nv_bfloat16*>(out), Y, ldy, scale);
  }
}
template <int MODE>
static void split_bf16_launch(const float* A, int64_t lda, int rows, int cols, int64_t kpad, int nterms, void* out,
                              bool transpose, int sms, cudaStream_t st, const float* Y, int64_t ldy, float scale) {
  if (nterms == 3)
    split_bf16_launch_nt<MODE, 3>(A, lda, rows, cols, kpad, out, transpose, sms, st, Y, ldy, scale);
  else
    split_bf16_launch_nt<MODE, 2>(A, lda, rows, cols, kpad, out, transpose, sms, st, Y, ldy, scale);
}

cudaError_t launch_split_bf16(const float* A, int64_t lda, int rows, int cols, int64_t kpad, int nterms, void* out,
                              bool transpose, int sms, cudaStream_t st, int xform, const float* Y, int64_t ldy,
                              float scale) {
  switch (xform) {
    case kXformNone: split_bf16_launch<kXformNone>(A, lda, rows, cols, kpad, nterms, out, transpose, sms, st, Y, ldy, scale); break;
    case kXformScale: split_bf16_launch<kXformScale>(A, lda, rows, cols, kpad, nterms, out, transpose, sms, st, Y, ldy, scale); break;
    case kXformSigmoidGrad: split_bf16_launch<kXformSigmoidGrad>(A, lda, rows, cols, kpad, nterms, out, transpose, sms, st, Y, ldy, scale); break;
    case kXformReluGrad: split_bf16_launch<kXformReluGrad>(A, lda, rows, cols, kpad, nterms, out, transpose, sms, st, Y, ldy, scale); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int S>
static cudaError_t prep_b_s(const double* B, int64_t ldb, int k, int n, int64_t kpad, int32_t* eb, int8_t* sb,
                            unsigned long long* colsum, cudaStream_t st) {
  dim3 grid((unsigned)ceil_div(n, 64), (unsigned)ceil_div(kpad, kColTileK));
  ozaki_slice_cols_kernel<S><<<grid, 256, 0, st>>>(B, ldb, k, n, kpad, eb, sb, colsum);
  return cudaGetLastError();
}

template <int S>
static cudaError_t prep_a_s(const double* A, int64_t lda, int m, int k, int64_t kpad, int32_t* ea, int8_t* sa,
                            unsigned long long* rowsum, int sms, cudaStream_t st) {
  if (kpad <= kRowRegK) {
    const unsigned rows_grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(m, (int64_t)sms * 8));
    ozaki_rows_kernel<S><<<rows_grid, 256, 0, st>>>(A, lda, m, k, kpad, ea, sa, rowsum);
    return cudaGetLastError();
  }
  cudaError_t e = cudaMemsetAsync(ea, 0x80, (size_t)m * sizeof(int32_t), st);
  if (e == cudaSuccess && rowsum) e = cudaMemsetAsync(rowsum, 0, (size_t)m * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)ceil_div(kpad, kRowRegK), (unsigned)std::min<int64_t>(m, 65535));
  ozaki_row_exp_kernel<<<grid, 256, 0, st>>>(A, lda, m, k, ea);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ozaki_row_slice_kernel<S><<<grid, 256, 0, st>>>(A, lda, m, k, kpad, ea, sa, rowsum);
  return cudaGetLastError();
}

cudaError_t launch_ozaki_prep_b(int s, const double* B, int64_t ldb, int k, int n, int64_t kpad, int32_t* eb,
                                int8_t* sb, unsigned long long* colsum, OzakiStats* stats, int sms, cudaStream_t st) {
  (void)sms;
  cudaError_t e = cudaMemsetAsync(eb, 0x80, (size_t)n * sizeof(int32_t), st);
  if (e == cudaSuccess && colsum) e = cudaMemsetAsync(colsum, 0, (size_t)n * sizeof(unsigned long long), st);
  if (e == cudaSuccess && stats) e = cudaMemsetAsync(&stats->min_col, 0xFF, sizeof(stats->min_col), st);
  if (e != cudaSuccess) return e;
  if (k > 0) {
    const dim3 grid((unsigned)ceil_div(n, 512), (unsigned)ceil_div(k, 64));
    ozaki_col_exp_kernel<<<grid, 256, 0, st>>>(B, ldb, k, n, eb);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  switch (s) {
    case 4: return prep_b_s<4>(B, ldb, k, n, kpad, eb, sb, colsum, st);
    case 5: return prep_b_s<5>(B, ldb, k, n, kpad, eb, sb, colsum, st);
    case 6: return prep_b_s<6>(B, ldb, k, n, kpad, eb, sb, colsum, st);
    case 7: return prep_b_s<7>(B, ldb, k, n, kpad, eb, sb, colsum, st);
    case 8: return prep_b_s<8>(B, ldb, k, n, kpad, eb, sb, colsum, st);
    case 9: return prep_b_s<9>(B, ldb, k, n, kpad, eb, sb, colsum, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_ozaki_prep_a(int s, const double* A, int64_t lda, int m, int k, int64_t kpad, int32_t* ea,
                                int8_t* sa, unsigned long long* rowsum, OzakiStats* stats, int sms, cudaStream_t st) {
  if (stats) {
    // min_row, done_blocks and choice restart for every A (min_col belongs to B)
    cudaError_t e = cudaMemsetAsync(&stats->min_row, 0xFF, sizeof(stats->min_row), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&stats->done_blocks, 0, sizeof(stats->done_blocks), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&stats->choice, 0xFF, sizeof(stats->choice), st);
    if (e != cudaSuccess) return e;
  }
  switch (s) {
    case 4: return prep_a_s<4>(A, lda, m, k, kpad, ea, sa, stats ? rowsum : nullptr, sms, st);
    case 5: return prep_a_s<5>(A, lda, m, k, kpad, ea, sa, stats ? rowsum : nullptr, sms, st);
    case 6: return prep_a_s<6>(A, lda, m, k, kpad, ea, sa, stats ? rowsum : nullptr, sms, st);
    case 7: return prep_a_s<7>(A, lda, m, k, kpad, ea, sa, stats ? rowsum : nullptr, sms, st);
    case 8: return prep_a_s<8>(A, lda, m, k, kpad, ea, sa, stats ? rowsum : nullptr, sms, st);
    case 9: return prep_a_s<9>(A, lda, m, k, kpad, ea, sa, stats ? rowsum : nullptr, sms, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_ozaki_decide(const unsigned long long* rowsum, int m, const unsigned long long* colsum, int n,
                                int64_t k, OzakiStats* stats, int sms, cudaStream_t st) {
  const unsigned blocks =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(std::max(m, n), 256), (int64_t)sms * 2));
  ozaki_decide_kernel<<<blocks, 256, 0, st>>>(rowsum, m, colsum, n, k, stats);
  return cudaGetLastError();
}

}  // namespace cucosma
