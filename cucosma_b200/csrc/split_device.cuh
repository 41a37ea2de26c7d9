// split_device.cuh -- per-element device helpers of the operand pre-passes,
// shared by the single-problem (split.cu) and grouped (grouped.cu) kernels.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace cucosma {

// x = t0 + t1 (+ t2) + residual: each term the round-to-nearest-even BF16 of
// what is left; every subtraction is exact in FP32 (Sterbenz).
__device__ __forceinline__ void split_bf16_value(float x, int nterms, __nv_bfloat16 (&t)[3]) {
  float r = x;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (i < nterms) {
      t[i] = __float2bfloat16_rn(r);
      r = r - __bfloat162float(t[i]);
    }
  }
}

// The same with the term count known at compile time (no local memory).
template <int NT>
__device__ __forceinline__ void split_bf16_n(float x, __nv_bfloat16 (&t)[NT]) {
  float r = x;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    t[i] = __float2bfloat16_rn(r);
    r = r - __bfloat162float(t[i]);
  }
}

// Two values at once: w[i] holds term i of x0 in its low half and of x1 in
// its high half (cvt.rn.bf16x2.f32 rounds each to nearest even, as
// __float2bfloat16_rn does), so the words equal pack_bf16x2 of
// split_bf16_n's terms bit for bit.
template <int NT>
__device__ __forceinline__ void split_bf16x2_n(float x0, float x1, uint32_t (&w)[NT]) {
  float r0 = x0, r1 = x1;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(w[i]) : "f"(r1), "f"(r0));
    if (i + 1 < NT) {
      r0 = r0 - __uint_as_float(w[i] << 16);
      r1 = r1 - __uint_as_float(w[i] & 0xffff0000u);
    }
  }
}

__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  __nv_bfloat162 v = __halves2bfloat162(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// frexp-style exponent of the largest magnitude: |x| < 2^e for all x.
__device__ __forceinline__ int exp_of(double amax) {
  if (amax == 0.0) return 0;
  int e;
  frexp(amax, &e);
  return e;
}

// Ozaki slices of one value scaled into (-1, 1): the restatement's sequence
// r <- v * 2^-e, then per slice r <- r * 2^7, q = trunc(r), r <- r - q is
// exact in FP64, so q_t is the sign of v times the t-th 7-bit group of the
// binary expansion of |v| * 2^-e.  Computed here from the bits of v with
// integer operations (one 64-bit shift instead of 2 S FP64 conversions):
// |v| = M * 2^(E - 1075) with the 53-bit significand M (E the biased
// exponent; M without the hidden bit and E = 1 for subnormals), so the
// first 7 S bits F = floor(|v| * 2^(7 S - e)) = M shifted by
// 7 S - e + E - 1075 (right when negative); q_t = +-((F >> 7 (S - 1 - t)) & 127).
// fixed_of returns F and the sign of v.
template <int S>
__device__ __forceinline__ uint64_t fixed_of(double v, int e, bool& neg) {
  static_assert(S * 7 <= 63, "slices exceed a 64-bit fixed-point value");
  const uint64_t bits = (uint64_t)__double_as_longlong(v);
  const int E = (int)((bits >> 52) & 0x7ff);
  const uint64_t mant = bits & ((1ull << 52) - 1);
  const uint64_t M = E ? (mant | (1ull << 52)) : mant;
  const int sh = 7 * S - e + (E ? E : 1) - 1075;  // F = M * 2^sh
  neg = (bits >> 63) != 0;
  if (sh >= 0) return sh >= 64 ? 0 : (M << sh);  // |v| < 2^e bounds F below 2^(7 S)
  return -sh >= 64 ? 0 : (M >> -sh);
}

// Fixed-point magnitudes of four values of a row (column) with exponent e:
// sum_j floor(|v_j| 2^(30 - e)), each term below 2^30 since |v_j| < 2^e.
__device__ __forceinline__ unsigned long long magnitude_fx4(const double (&v)[4], int e) {
  unsigned long long t = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) t += __double2ull_rz(ldexp(fabs(v[j]), 30 - e));
  return t;
}

// Bits [o, o + 7) of the 64-bit value hi:lo moved to bits [p, p + 7), all
// other bits zero (o and p are constants once the callers' loops unroll:
// one shift and one masked OR per digit).
__device__ __forceinline__ uint32_t digit_at(uint32_t lo, uint32_t hi, int o, int p) {
  const int n = o - p;
  uint32_t x;
  if (n >= 32)
    x = hi >> (n - 32);
  else if (n > 0)
    x = __funnelshift_r(lo, hi, n);
  else
    x = lo << (-n);
  return x & (127u << p);
}

// The slices of four values, packed: byte j of w[t] is slice_value's q_t of
// v[j] (the 4-byte word the packed and stacked layouts store for four
// consecutive k).  The digits of |v_j| are gathered into the word first and
// the negative values' bytes negated together: per byte, 0x80 - g never
// borrows for g <= 127, and (0x80 - g) ^ 0x80 = -g mod 256 (0 for g = 0).
// Returns the magnitude sum of magnitude_fx4, from the same fixed-point
// values when 7 S >= 30: floor(F 2^-(7S - 30)) = floor(|v| 2^(30 - e)).
template <int S>
__device__ __forceinline__ unsigned long long slice4_packed(const double (&v)[4], int e, uint32_t (&w)[S]) {
  uint32_t lo[4], hi[4], nm = 0;
  unsigned long long mag = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    bool neg;
    const uint64_t F = fixed_of<S>(v[j], e, neg);
    lo[j] = (uint32_t)F;
    hi[j] = (uint32_t)(F >> 32);
    nm |= neg ? 0xffu << (8 * j) : 0u;
    if constexpr (7 * S >= 30) mag += F >> (7 * S - 30);
  }
#pragma unroll
  for (int t = 0; t < S; ++t) {
    const int o = 7 * (S - 1 - t);
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) x |= digit_at(lo[j], hi[j], o, 8 * j);
    const uint32_t nx = (0x80808080u - x) ^ 0x80808080u;
    w[t] = (x & ~nm) | (nx & nm);
  }
  if constexpr (7 * S < 30) mag = magnitude_fx4(v, e);
  return mag;
}

// Packed slice layout shared by both operands: for row r (a row of A, or a
// column of B), k-block kb = k / 32 and slice p, the 32 bytes of k-block kb
// of slice p are at r * (kpad * S) + kb * (32 * S) + p * 32.  Four slices of
// one k-block thus fill one 128-byte row, the span of the 128-byte swizzle
// the tensor cores read, and one TMA box row is 128 contiguous bytes.
template <int S>
__device__ __forceinline__ int64_t packed_index(int64_t r, int k, int64_t kpad, int p) {
  return r * (kpad * S) + (int64_t)(k >> 5) * (32 * S) + p * 32 + (k & 31);
}
// Stacked layout of the B slices: [k-block][slice][column][32 bytes of K],
// so one TMA box brings all slices of a run of columns as a K-major matrix
// whose rows are (slice, column) -- the B operand of the stacked-N MMAs.
template <int S>
__device__ __forceinline__ int64_t stacked_index(int64_t n, int k, int64_t ncols, int p) {
  return ((int64_t)(k >> 5) * S + p) * (ncols * 32) + n * 32 + (k & 31);
}

// Backward-pass source transforms of the BF16 split (see SplitXform).
template <int MODE>
__device__ __forceinline__ float xform(float v, float y, float scale) {
  if constexpr (MODE == 1) return scale * v;
  if constexpr (MODE == 2) return scale * v * (y * (1.0f - y));
  if constexpr (MODE == 3) return y > 0.0f ? scale * v : 0.0f;
  return v;
}

}  // namespace cucosma
