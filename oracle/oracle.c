/*
 * oracle.c -- CPU restatement of the cuCOSMA GEMM path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * and bench.py's cpu_baseline leg load it.  The product library
 * (cucosma_b200/libcucosma.so) never links, loads or calls anything here.
 *
 * What it restates (paths relative to the cuCOSMA project root):
 *   - the product C = A*B of Matrix<T>::operator* (Kernel/cuda/src/Matrix.h:183-201),
 *     same i-j-k order, but accumulating in double (the reference accumulates in T);
 *   - the alpha/beta epilogue of cosmaSgemm_kernel: acc *= ALPHA; acc += BETA*C
 *     (Kernel/cuda/src/cuCOSMAV100.cuh:1582-1593, load_C_OneRow_Vector :894-912),
 *     with C left unread when BETA == 0 (:1589);
 *   - the split-K reduction C = BETA*c + ALPHA*sum_z ws[z], z ascending
 *     (Kernel/cuda/src/cosmaSplitKReduce.cuh:31-40);
 *   - the optional sigmoid epilogue 1/(1+exp(-x)) applied to the final value
 *     (Kernel/cuda/src/cuCOSMAV100.cuh:2472-2476, sigmoid4.cuh:19-22).
 * Beyond the reference (its algorithms are published, restated here):
 *   - double-double dot products (Ogita, Rump, Oishi, "Accurate sum and dot
 *     product", SIAM J. Sci. Comput. 26(6), 2005: TwoSum / TwoProduct / Dot2);
 *   - the BF16 hi/lo(/lo2) split of FP32 operands (round-to-nearest-even);
 *   - the Ozaki scheme (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of
 *     matrix multiplication by using fast routines of matrix multiplication and
 *     its applications", Numer. Algorithms 59, 2012) in its integer-slice form:
 *     per-row / per-column power-of-two scaling, 7-bit signed int8 slices,
 *     exact integer slice products grouped by diagonal, FP64 recombination.
 *
 * Parity pinning: oracle_gemm_f64 is checked bit for bit against the
 * reference's own Matrix<double>::operator* (built from the reference sources
 * into oracle/_ref/) and against the committed fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPI_NONE 0
#define EPI_SIGMOID 1
#define EPI_RELU 2

static double apply_epilogue(double v, int epi) {
    if (epi == EPI_SIGMOID) return 1.0 / (1.0 + exp(-v));
    if (epi == EPI_RELU) return v > 0.0 ? v : 0.0;
    return v;
}

static void set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* B^T copy so the k loop reads contiguous memory; the summation order (k
 * ascending per (i,j)) is unchanged, so results equal the naive i-j-k loop. */
static double *transpose_b(int64_t k, int64_t n, const double *B, int64_t ldb) {
    double *bt = (double *)malloc(sizeof(double) * (size_t)(k * n > 0 ? k * n : 1));
    for (int64_t kk = 0; kk < k; ++kk)
        for (int64_t j = 0; j < n; ++j) bt[j * k + kk] = B[kk * ldb + j];
    return bt;
}

/*
 * out[i][j] = epi(alpha * sum_k A[i][k]*B[k][j] + beta * Cin[i][j])
 * Product: Matrix.h:183-201 (acc += a*b, k ascending), accumulated in double.
 * Epilogue: cuCOSMAV100.cuh:1582-1593 (alpha first, then beta*C; C unread if beta == 0).
 */
void oracle_gemm_f64(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                     const double *B, int64_t ldb, const double *Cin, int64_t ldc,
                     double alpha, double beta, int epilogue, double *out, int64_t ldo,
                     int threads) {
    set_threads(threads);
    double *bt = transpose_b(k, n, B, ldb);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < m; ++i) {
        const double *a = A + i * lda;
        for (int64_t j = 0; j < n; ++j) {
            const double *b = bt + j * k;
            double acc = 0.0;
            for (int64_t kk = 0; kk < k; ++kk) acc += a[kk] * b[kk];
            double v = acc;
            if (alpha != 1.0) v = alpha * v;
            if (beta != 0.0) v = v + beta * Cin[i * ldc + j];
            out[i * ldo + j] = apply_epilogue(v, epilogue);
        }
    }
    free(bt);
}

/* Error-free transformations (Ogita-Rump-Oishi 2005, Alg. 3.1 TwoSum, Alg. 3.3
 * TwoProduct with a fused multiply-add). */
static inline void two_sum(double a, double b, double *s, double *e) {
    double x = a + b;
    double z = x - a;
    *e = (a - (x - z)) + (b - z);
    *s = x;
}
static inline void two_prod(double a, double b, double *p, double *e) {
    double x = a * b;
    *e = fma(a, b, -x);
    *p = x;
}

/*
 * Same contract as oracle_gemm_f64 but the dot products use Dot2 (result as
 * accurate as if computed in twice the working precision, then rounded), and
 * the epilogue is evaluated on the double-double value.  out_lo (optional)
 * receives the low word of the double-double product alpha*AB + beta*C.
 */
void oracle_gemm_dd(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                    const double *B, int64_t ldb, const double *Cin, int64_t ldc,
                    double alpha, double beta, int epilogue, double *out, int64_t ldo,
                    double *out_lo, int threads) {
    set_threads(threads);
    double *bt = transpose_b(k, n, B, ldb);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < m; ++i) {
        const double *a = A + i * lda;
        for (int64_t j = 0; j < n; ++j) {
            const double *b = bt + j * k;
            double p = 0.0, s = 0.0;
            for (int64_t kk = 0; kk < k; ++kk) {
                double h, r, q;
                two_prod(a[kk], b[kk], &h, &r);
                two_sum(p, h, &p, &q);
                s += q + r;
            }
            /* (p, s) -> normalised double-double (hi, lo) */
            double hi, lo;
            two_sum(p, s, &hi, &lo);
            if (alpha != 1.0) {
                double ph, pe;
                two_prod(alpha, hi, &ph, &pe);
                lo = pe + alpha * lo;
                two_sum(ph, lo, &hi, &lo);
            }
            if (beta != 0.0) {
                double ch, ce, sh, se;
                two_prod(beta, Cin[i * ldc + j], &ch, &ce);
                two_sum(hi, ch, &sh, &se);
                lo = se + lo + ce;
                two_sum(sh, lo, &hi, &lo);
            }
            if (epilogue != EPI_NONE) {
                double v = apply_epilogue(hi + lo, epilogue);
                hi = v;
                lo = 0.0;
            }
            out[i * ldo + j] = hi;
            if (out_lo) out_lo[i * ldo + j] = lo;
        }
    }
    free(bt);
}

/* Split-K restatement: ws holds splits partial sums [splits][m][n] (row stride n);
 * C = beta*c + alpha*sum_z ws[z] with z ascending, the sum accumulated in the
 * element type (cosmaSplitKReduce.cuh:31-40).  is_f32 selects float arithmetic. */
void oracle_splitk_reduce_f32(int64_t m, int64_t n, int splits, const float *ws, float *C,
                              int64_t ldc, float alpha, float beta) {
    for (int64_t i = 0; i < m; ++i)
        for (int64_t j = 0; j < n; ++j) {
            float v = 0.0f;
            for (int z = 0; z < splits; ++z) v += ws[(int64_t)z * m * n + i * n + j];
            float c = C[i * ldc + j];
            C[i * ldc + j] = beta * c + alpha * v;
        }
}

/* ---------------------------------------------------------------- BF16 split */

static inline uint16_t f32_to_bf16_rn(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) { /* inf / nan: truncate, keep nan quiet */
        uint16_t h = (uint16_t)(u >> 16);
        if (u & 0x007fffffu) h |= 0x0040u;
        return h;
    }
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}
static inline float bf16_to_f32(uint16_t h) {
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* x = t0 + t1 (+ t2) + residual, each term the round-to-nearest-even BF16 of
 * the remaining residual; every residual subtraction is exact in FP32
 * (Sterbenz).  out holds nterms planes of n values. */
void oracle_split_bf16(const float *x, int64_t n, int nterms, uint16_t *out) {
    for (int64_t i = 0; i < n; ++i) {
        float r = x[i];
        for (int t = 0; t < nterms; ++t) {
            uint16_t h = f32_to_bf16_rn(r);
            out[(int64_t)t * n + i] = h;
            r = r - bf16_to_f32(h);
        }
    }
}

/* ------------------------------------------------------------------- Ozaki */

/* Exponent e with |x| < 2^e for every x of the vector (frexp convention:
 * x = f*2^e, 0.5 <= |f| < 1).  Zero vectors give 0. */
static int vec_exponent(const double *x, int64_t n, int64_t stride) {
    int best = INT32_MIN;
    for (int64_t t = 0; t < n; ++t) {
        double v = x[t * stride];
        if (v != 0.0) {
            int e;
            frexp(v, &e);
            if (e > best) best = e;
        }
    }
    return best == INT32_MIN ? 0 : best;
}

/* Per-row exponents of A (m x k, row stride lda) and per-column exponents of
 * B (k x n, row stride ldb). */
void oracle_ozaki_exponents(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                            const double *B, int64_t ldb, int32_t *ea, int32_t *eb) {
    for (int64_t i = 0; i < m; ++i) ea[i] = vec_exponent(A + i * lda, k, 1);
    for (int64_t j = 0; j < n; ++j) eb[j] = vec_exponent(B + j, k, ldb);
}

/* Slices of one value scaled into (-1,1): r <- r*2^7, q = trunc(r), r <- r-q.
 * Every step is exact in FP64 (power-of-two scaling and removal of the
 * integer part), so x*2^-e = sum_t q_t 2^(-7(t+1)) + rem with |rem| < 2^(-7s). */
static inline void slice_value(double v, int e, int s, int8_t *q, int64_t plane) {
    double r = ldexp(v, -e);
    for (int t = 0; t < s; ++t) {
        r = r * 128.0;
        double w = trunc(r);
        q[(int64_t)t * plane] = (int8_t)w;
        r = r - w;
    }
}

/* A slices, layout [s][m][k] (K contiguous); B slices, layout [s][n][k]
 * (B transposed so that K is contiguous for both operands). */
void oracle_ozaki_slices(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                         const double *B, int64_t ldb, const int32_t *ea, const int32_t *eb,
                         int s, int8_t *sa, int8_t *sb) {
    for (int64_t i = 0; i < m; ++i)
        for (int64_t kk = 0; kk < k; ++kk)
            slice_value(A[i * lda + kk], ea[i], s, sa + i * k + kk, m * k);
    for (int64_t j = 0; j < n; ++j)
        for (int64_t kk = 0; kk < k; ++kk)
            slice_value(B[kk * ldb + j], eb[j], s, sb + j * k + kk, n * k);
}

/*
 * Full Ozaki product restatement, bit-exact target for the GPU path.
 *   for every K chunk c (length kchunk, last one ragged):
 *     S_d = sum_{p+q=d} sum_{k in c} A_p[i][k] * B_q[j][k]          (exact, int64)
 *     part_c = sum_{d = s-1 .. 0} double(S_d) * 2^(-7(d+2))        (FP64, d descending)
 *   tot = sum_c part_c  (c ascending; the deterministic split-K reduction)
 *   r   = ldexp(tot, ea[i] + eb[j])
 *   out = beta == 0 ? alpha*r : fma(alpha, r, beta*C)
 */
void oracle_ozaki_gemm(int64_t m, int64_t n, int64_t k, const int8_t *sa, const int8_t *sb,
                       const int32_t *ea, const int32_t *eb, int s, int64_t kchunk,
                       const double *Cin, int64_t ldc, double alpha, double beta, int epilogue,
                       double *out, int64_t ldo, int threads) {
    set_threads(threads);
    if (kchunk <= 0) kchunk = k > 0 ? k : 1;
    int64_t nchunks = k > 0 ? (k + kchunk - 1) / kchunk : 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < m; ++i) {
        int64_t *S = (int64_t *)malloc(sizeof(int64_t) * (size_t)s);
        for (int64_t j = 0; j < n; ++j) {
            double tot = 0.0;
            for (int64_t c = 0; c < nchunks; ++c) {
                int64_t k0 = c * kchunk, k1 = k0 + kchunk < k ? k0 + kchunk : k;
                for (int d = 0; d < s; ++d) S[d] = 0;
                for (int p = 0; p < s; ++p)
                    for (int q = 0; p + q < s; ++q) {
                        const int8_t *a = sa + (int64_t)p * m * k + i * k;
                        const int8_t *b = sb + (int64_t)q * n * k + j * k;
                        int64_t acc = 0;
                        for (int64_t kk = k0; kk < k1; ++kk) acc += (int64_t)a[kk] * (int64_t)b[kk];
                        S[p + q] += acc;
                    }
                double part = 0.0;
                for (int d = s - 1; d >= 0; --d) part += ldexp((double)S[d], -7 * (d + 2));
                tot = c == 0 ? part : tot + part;
            }
            double r = ldexp(tot, ea[i] + eb[j]);
            double v = beta == 0.0 ? alpha * r : fma(alpha, r, beta * Cin[i * ldc + j]);
            out[i * ldo + j] = apply_epilogue(v, epilogue);
        }
        free(S);
    }
}
