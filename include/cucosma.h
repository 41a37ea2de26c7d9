/*
 * cucosma.h -- C ABI of the cuCOSMA-compatible GEMM library for NVIDIA B200 (sm_100a).
 *
 * Computes C = epi(alpha * A*B + beta * C) on row-major matrices in device
 * memory: A is m x k (row stride lda), B is k x n (ldb), C is m x n (ldc),
 * strides in elements.  This replaces the reference's kernel API
 *     cublasStatus_t cosmaSgemm(const TYPE* A, int lda, const TYPE* B, int ldb,
 *                               TYPE* C, int ldc)          (Kernel/cuda/src/cuCOSMAV100.cuh:2774-2776)
 * whose M, N, K, ALPHA, BETA, TYPE and tiling were compile-time macros
 * (Kernel/cuda/src/config.h:9-31).  Here they are fields of a descriptor (or
 * arguments), tiling and split-K are chosen by the library (or its tuner),
 * and the compile-time template form lives in cucosma.hpp.
 *
 * Plain C: pointers, sizes and integers only.  No entry point throws or
 * exits; all return a cucosma_status.  All GPU work is enqueued on the
 * caller's stream (a cudaStream_t passed as void*; NULL = legacy default).
 *
 * Alignment: A, B and C must be 16-byte aligned and every row must start on
 * a 16-byte boundary (lda, ldb, ldc * sizeof(element) multiples of 16), the
 * reference's "aligned rows" contract (cudaMallocPitch pitches,
 * Kernel/cuda/src/test_correctness.h:55-58).  Otherwise the call returns
 * CUCOSMA_STATUS_MISALIGNED and launches nothing.
 */
#ifndef CUCOSMA_H_
#define CUCOSMA_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUCOSMA_VERSION 200 /* 0.2.0 */

#if defined(__GNUC__)
#define CUCOSMA_API __attribute__((visibility("default")))
#else
#define CUCOSMA_API
#endif

typedef enum cucosma_status {
  CUCOSMA_STATUS_SUCCESS = 0,
  CUCOSMA_STATUS_INVALID_VALUE = 1,       /* bad size, stride, null pointer or enum */
  CUCOSMA_STATUS_MISALIGNED = 2,          /* pointer or row stride not 16-byte aligned */
  CUCOSMA_STATUS_NOT_SUPPORTED = 3,       /* combination not implemented (e.g. BF16X3 on FP64) */
  CUCOSMA_STATUS_WORKSPACE_TOO_SMALL = 4, /* workspace_bytes below cucosma_gemm_workspace_size */
  CUCOSMA_STATUS_LAUNCH_FAILED = 5,       /* a CUDA launch or API call failed */
  CUCOSMA_STATUS_TIMEOUT = 6,             /* a device-side bounded wait expired (see cucosma_device_status) */
  CUCOSMA_STATUS_ARCH_MISMATCH = 7,       /* current device is not sm_100 */
  CUCOSMA_STATUS_ALLOC_FAILED = 8,        /* library-managed workspace could not be allocated */
  CUCOSMA_STATUS_INTERNAL_ERROR = 9
} cucosma_status;

typedef enum cucosma_dtype { CUCOSMA_R_32F = 0, CUCOSMA_R_64F = 1 } cucosma_dtype;

typedef enum cucosma_precision {
  CUCOSMA_PRECISION_NATIVE = 0, /* FFMA (FP32) / DFMA (FP64) SIMT kernels */
  CUCOSMA_PRECISION_BF16X3 = 1, /* FP32: hi/lo BF16 split, 3 tensor-core products, FP32 accumulation */
  CUCOSMA_PRECISION_BF16X6 = 2, /* FP32: hi/mid/lo BF16 split, 6 tensor-core products */
  CUCOSMA_PRECISION_OZAKI = 3   /* FP64: INT8 slices, exact INT32 products, FP64 recombination */
} cucosma_precision;

typedef enum cucosma_epilogue {
  CUCOSMA_EPILOGUE_NONE = 0,
  CUCOSMA_EPILOGUE_SIGMOID = 1, /* 1/(1+exp(-x)) of the final value (cuCOSMAV100.cuh:2472-2476) */
  CUCOSMA_EPILOGUE_RELU = 2     /* max(x, 0) (cuCOSMAV100.cuh:2466-2470) */
} cucosma_epilogue;

typedef struct cucosma_gemm_desc {
  int64_t m, n, k;        /* M, N, K of config.h */
  int64_t lda, ldb, ldc;  /* row strides in elements */
  int32_t dtype;          /* cucosma_dtype (TYPE of config.h) */
  int32_t precision;      /* cucosma_precision */
  int32_t slices;         /* Ozaki slice count 4..9; 0 = chosen on the device per call: 8 or 9 slices,
                           * or native FP64, from the operands' magnitude spread (see cucosma_plan_info) */
  int32_t epilogue;       /* cucosma_epilogue */
  double alpha, beta;     /* ALPHA, BETA of config.h; C is not read when beta == 0 */
  int32_t split_k;        /* SPLIT_K: 0 = library/tuner choice, >= 1 forced */
  int32_t swizzle;        /* SWIZZLE: 0 = library choice, >= 1 forced block-index remap width */
  int32_t tile;           /* 0 = library/tuner choice, else a kernel configuration id:
                           * NATIVE 1 = always the 128 x 128 tile kernel (no skinny-shape kernels),
                           *        2 = the 64 x 128 tile kernel (FP32; FP64 runs 128 x 128);
                           * BF16X3 1 = 128 x 256 without promotion, 2 = 128 x 128 promoted,
                           *        3 = 128 x 256 promoted, 4 = 256 x 256 CTA pair (default when m > 128),
                           *        5 = 256 x 128 pair with the split fused in;
                           * BF16X6 1 = 128 x 128, 2 = 256 x 128 CTA pair,
                           *        3 = 256 x 256 CTA pair (default when m > 128),
                           *        4 = 256 x 128 pair with the split fused in.
                           * Auto (0) picks the fused kernels where the separate split pass
                           * would cost more than a quarter of the GEMM (large K, large N) */
  int32_t flags;          /* 0, or CUCOSMA_FLAG_TEST_SKIP_STAGE */
} cucosma_gemm_desc;

/* Test hook for the failure path (no counterpart in the reference, which
 * exits the process on any CUDA error): on a tensor-core precision path the
 * producer of every CTA leaves its first shared-memory stage unfilled, so the
 * consumers' bounded waits expire; the call itself returns SUCCESS, the
 * kernel stops early (C is left partly written) and cucosma_device_status
 * then reports CUCOSMA_STATUS_TIMEOUT.  The CUDA context stays usable.  Pair
 * it with a short cucosma_set_wait_timeout_ns. */
#define CUCOSMA_FLAG_TEST_SKIP_STAGE (1 << 30)

/* Fill *d with defaults: FP32, native, alpha = 1, beta = 0, no epilogue, auto split-K. */
CUCOSMA_API void cucosma_gemm_desc_init(cucosma_gemm_desc* d);

/* Bytes of device workspace cucosma_gemm needs for *d (0 when none). */
CUCOSMA_API cucosma_status cucosma_gemm_workspace_size(const cucosma_gemm_desc* d, size_t* bytes);

/* The execution plan cucosma_gemm would use for *d on the current device:
 * the compile-time tiling of config.h (THREADBLOCK_TILE_M/N, LOAD_K,
 * SPLIT_K, SWIZZLE) as chosen at run time, plus the workspace layout of the
 * precision paths (offsets of the operand planes inside the workspace). */
typedef struct cucosma_plan_info {
  int32_t path;     /* 0 native SIMT, 1 BF16x3, 2 BF16x6, 3 Ozaki */
  int32_t tile_m, tile_n, tile_k;
  int32_t splits;   /* split-K factor */
  int32_t band;     /* raster band / block-index remap width */
  int32_t slices;   /* operand planes (BF16 terms or Ozaki slices) */
  int32_t launches; /* kernels one cucosma_gemm call enqueues */
  int64_t kchunk;   /* K extent of one split */
  int64_t kpad;     /* padded K of the operand planes */
  uint64_t workspace_bytes, off_a, off_b, off_ea, off_eb, off_part;
  /* Ozaki with slices = 0 (the default): the slice count is chosen on the
   * device from the operands (8 or 9 slices, or native FP64 when 9 cannot
   * reach FP64 accuracy; see cucosma_gemm_desc.slices).  The call writes its
   * choice as an int32 at workspace offset off_choice: 8, 9, or 0 = native
   * FP64.  0 for every other path. */
  uint64_t off_choice;
  int32_t layout_slices; /* Ozaki: slices per 32-wide k-block in the workspace layout */
  int32_t fused;         /* BF16 paths: 1 = the split is done inside the GEMM kernel (operands read once
                          * from the caller's buffers; no planes in the workspace) */
} cucosma_plan_info;
CUCOSMA_API cucosma_status cucosma_gemm_get_plan(const cucosma_gemm_desc* d, cucosma_plan_info* info);

/* C = epi(alpha*A*B + beta*C).  workspace may be NULL when the size is 0.
 * Allocation-free; asynchronous on stream.  Replaces cosmaSgemm
 * (cuCOSMAV100.cuh:2774-2848) including its split-K workspace path
 * (:2824-2838, which allocated and freed the workspace on every call). */
CUCOSMA_API cucosma_status cucosma_gemm(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* workspace,
                            size_t workspace_bytes, void* stream);

/* cucosma_gemm with a library-managed workspace (the same per-device,
 * per-stream buffer as cucosma_sgemm below, with the same rules on stream
 * capture) instead of a caller-owned one: the reference's split-K path
 * allocated its workspace inside the call (cuCOSMAV100.cuh:2828-2838); this
 * keeps that interface for every precision without allocating per call.
 * Used by the C++ drop-in (cucosma.hpp). */
CUCOSMA_API cucosma_status cucosma_gemm_managed(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                                void* stream);

/* Reference-shaped FP32 / FP64 entry points: the compile-time M, N, K, ALPHA,
 * BETA of config.h become arguments (cuCOSMAV100.cuh:2774; the FP64 form is
 * the TYPE=double instantiation).  Native arithmetic, no epilogue; any split-K
 * workspace is library-managed (one buffer per device and stream, allocated
 * and grown on demand, like the reference's internal cudaMalloc but not per
 * call).  Growing it synchronises the stream and frees the old buffer, so any
 * call that needs a larger workspace than the stream's buffer holds must not
 * be inside a stream capture: during a capture such a call returns
 * CUCOSMA_STATUS_ALLOC_FAILED instead of allocating.  The buffer is keyed by
 * the stream handle and kept until the process exits; a stream that is
 * destroyed while work on it still uses the buffer must not have its handle
 * reused by a new stream before that work completes. */
CUCOSMA_API cucosma_status cucosma_sgemm(int m, int n, int k, float alpha, const float* A, int lda, const float* B, int ldb,
                             float beta, float* C, int ldc, void* stream);
CUCOSMA_API cucosma_status cucosma_dgemm(int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb,
                             double beta, double* C, int ldc, void* stream);

/* ------------------------------------------------------------------ tuner
 * Replaces the reference's ScheduleGenerator (ScheduleGenerator/
 * ScheduleGeneratorv4.h:13, a host-side brute force ranked by a
 * communication-volume model): candidate split-K factors, raster bands /
 * block-index remap widths and tile variants of *d are run on the device on
 * the caller's buffers (C is overwritten: pass scratch) and the fastest is
 * cached for (SM count, dtype, precision, slices, m, n, k).  Candidates whose
 * workspace exceeds workspace_bytes are skipped; max_candidates <= 0 = all.
 * cucosma_gemm uses the cached choice whenever split_k, swizzle and tile are
 * all 0.  The cache is saved / loaded as a text file; $CUCOSMA_TUNE_CACHE is
 * loaded on first use, CUCOSMA_TUNE=off disables lookups. */
typedef struct cucosma_tune_result {
  int32_t split_k, swizzle, tile; /* the chosen configuration */
  int32_t candidates;             /* configurations measured */
  int32_t occupancy;              /* resident CTAs per SM of the chosen kernel */
  int32_t reserved;
  double ms, tflops;              /* measured time of one call of the chosen configuration */
  double l2_hit_rate;             /* L2 hit rate (percent) of one call of it, read from the hardware
                                   * counters (lts__t_sector_hit_rate, CUPTI range profiler); -1 when
                                   * profiling is unavailable or CUCOSMA_TUNE_COUNTERS=off */
  double dram_bytes;              /* DRAM bytes read + written by that call (counters), -1 likewise */
  int32_t counter_passes;         /* profiled calls the counter reading took */
  int32_t reserved2;
} cucosma_tune_result;
CUCOSMA_API cucosma_status cucosma_tune(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                        void* workspace, size_t workspace_bytes, int max_candidates,
                                        cucosma_tune_result* out, void* stream);
CUCOSMA_API cucosma_status cucosma_tune_cache_save(const char* path);
CUCOSMA_API cucosma_status cucosma_tune_cache_load(const char* path);
CUCOSMA_API cucosma_status cucosma_tune_cache_clear(void);
CUCOSMA_API int cucosma_tune_cache_size(void);

/* --------------------------------------------------------------- backward
 * Gradients of the forward Y = epi(alpha*A*B + beta*C0) computed by
 * cucosma_gemm with descriptor *fwd (FP32, precision BF16X3 or BF16X6; no
 * counterpart in the reference, which has no backward pass).  Saved operands
 * A, B and the forward output Y (row stride ldy; unused when the epilogue is
 * NONE) and the upstream gradient dY give
 *     G  = alpha * dY (.) epi'(Z),  epi' = Y(1-Y) (sigmoid), [Y > 0] (ReLU), 1
 *     dA = G * B^T   (m x k, row stride ldda)      dB = A^T * G   (k x n, lddb)
 * on the tensor cores, with epi' fused into the operand pre-pass; either of
 * dA / dB may be NULL to skip it.  Overwrites dA and dB. */
CUCOSMA_API cucosma_status cucosma_gemm_backward_workspace_size(const cucosma_gemm_desc* fwd, size_t* bytes);
CUCOSMA_API cucosma_status cucosma_gemm_backward(const cucosma_gemm_desc* fwd, const void* A, const void* B,
                                                 const void* Y, int64_t ldy, const void* dY, int64_t lddy, void* dA,
                                                 int64_t ldda, void* dB, int64_t lddb, void* workspace,
                                                 size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------ host buffers
 * C = epi(alpha*A*B + beta*C) with A, B and C in host memory (pinned, for the
 * copies to overlap; lda/ldb/ldc are the host row strides).  No counterpart
 * in the reference, whose callers copy around cosmaSgemm themselves.  B is
 * copied first; A (and C when beta != 0) follow in row blocks, each block's
 * GEMM runs when its rows have arrived and its C rows are copied back while
 * later blocks still copy in, on three library streams per device (created
 * by the first call on that device) ordered after the work queued on stream;
 * stream waits for the last copy back.  device_buffer (256-byte aligned, of
 * cucosma_gemm_host_buffer_size bytes) holds the device copies and the GEMM
 * workspace; calls sharing it must be ordered on the same stream. */
CUCOSMA_API cucosma_status cucosma_gemm_host_buffer_size(const cucosma_gemm_desc* d, size_t* bytes);
CUCOSMA_API cucosma_status cucosma_gemm_host(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                             void* device_buffer, size_t buffer_bytes, void* stream);

/* ---------------------------------------------------------------- grouped
 * Many independent GEMMs of uneven sizes in one persistent launch (no
 * counterpart in the reference, whose sizes are compile-time macros: one
 * build per shape).  Every problem shares the descriptor's dtype, precision
 * (BF16X3, BF16X6 or OZAKI), slices, epilogue, alpha and beta; the m, n, k,
 * ld* fields of the descriptor are ignored.  A plan binds the problems (their
 * device pointers and sizes) to a caller workspace: plan creation encodes one
 * pair of TMA descriptors per problem and uploads the problem table into the
 * workspace (synchronous).  cucosma_gemm_grouped then enqueues exactly two
 * kernels (BF16 paths: operand split, GEMM) or three (Ozaki: exponents,
 * slices, GEMM), allocates nothing and copies nothing from the host, so it
 * can be captured in a CUDA graph and replayed while the plan lives. */
typedef struct cucosma_gemm_problem {
  int64_t m, n, k;
  int64_t lda, ldb, ldc;
  const void* A;
  const void* B;
  void* C;
} cucosma_gemm_problem;

typedef struct cucosma_grouped_plan_st* cucosma_grouped_plan;

CUCOSMA_API cucosma_status cucosma_grouped_workspace_size(const cucosma_gemm_desc* d,
                                                          const cucosma_gemm_problem* problems, int count,
                                                          size_t* bytes);
CUCOSMA_API cucosma_status cucosma_grouped_plan_create(const cucosma_gemm_desc* d,
                                                       const cucosma_gemm_problem* problems, int count,
                                                       void* workspace, size_t workspace_bytes,
                                                       cucosma_grouped_plan* plan);
CUCOSMA_API cucosma_status cucosma_gemm_grouped(cucosma_grouped_plan plan, void* stream);
CUCOSMA_API cucosma_status cucosma_grouped_plan_destroy(cucosma_grouped_plan plan);
/* The plan's tile: descriptor tile id (BF16X3 1 = 128 x 128 promoted,
 * 2 = 128 x 256 promoted, 3 = 256 x 256 CTA pair; BF16X6 1 = 128 x 128,
 * 2 = 256 x 256 pair; Ozaki 1), its rows and columns, and whether it came
 * from the tuning cache (descriptor tile 0 with a cucosma_tune_grouped entry
 * for this batch; otherwise tile 0 means 1). */
CUCOSMA_API cucosma_status cucosma_grouped_plan_get_tile(cucosma_grouped_plan plan, int32_t* tile, int32_t* tile_m,
                                                         int32_t* tile_n, int32_t* from_cache);

/* The grouped launch's counterpart: its candidate tiles (BF16X3: 128 x 128,
 * 128 x 256, 256 x 256 CTA pair; BF16X6: 128 x 128, 256 x 256 pair; Ozaki:
 * one) are run on the problems (their C is overwritten) and the fastest is
 * cached for this batch's shape mix (SM count, dtype, precision, slices and
 * the problems' m, n, k in order).  cucosma_grouped_plan_create uses it when
 * the descriptor's tile is 0.  out->tile is the chosen grouped tile id. */
CUCOSMA_API cucosma_status cucosma_tune_grouped(const cucosma_gemm_desc* d, const cucosma_gemm_problem* problems,
                                                int count, void* workspace, size_t workspace_bytes,
                                                cucosma_tune_result* out, void* stream);


/* Allocation-free FP32 split-K GEMM.  No counterpart in the reference (whose
 * split-K path cudaMallocs its workspace on every call).  For callers that
 * must not allocate device memory -- e.g. a plugin whose host framework owns
 * the whole device pool, or a latency-critical caller that cannot afford
 * cudaMalloc's implicit synchronisation.  Same arithmetic as cucosma_sgemm
 * with SPLIT_K = split_k (0 = library choice); the split-K partial sums live
 * in a fixed device array of CUCOSMA_STATIC_SCRATCH_BYTES inside the library,
 * held by every device that loads it until the process exits (the library's
 * own split_k choice is capped to fit it).  Problems whose
 * partials (splits * m * round_up(n, 4) floats) exceed it return
 * CUCOSMA_STATUS_WORKSPACE_TOO_SMALL without launching.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress), so make
 * that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race, and must be ordered by the caller. */
#define CUCOSMA_STATIC_SCRATCH_BYTES (16u << 20)
CUCOSMA_API cucosma_status cucosma_sgemm_splitk_static(int m, int n, int k, float alpha, const float* A, int lda,
                                                       const float* B, int ldb, float beta, float* C, int ldc,
                                                       int split_k, void* stream);

/* Synchronises the device, then returns and clears the device status word:
 * CUCOSMA_STATUS_TIMEOUT if any kernel gave up on a bounded wait since the
 * last call, CUCOSMA_STATUS_LAUNCH_FAILED on a CUDA error, else SUCCESS.
 * *detail (optional) receives the raw device code. */
CUCOSMA_API cucosma_status cucosma_device_status(int* detail);

/* Limit for every device-side wait (default 4 s).  Applies to later launches. */
CUCOSMA_API cucosma_status cucosma_set_wait_timeout_ns(uint64_t ns);

CUCOSMA_API const char* cucosma_get_error_string(cucosma_status s);
CUCOSMA_API int cucosma_get_version(void);

/* Observability (no counterpart in the reference, which timed its kernel with
 * nvprof, Kernel/cuda/run.sh:291).
 * cucosma_launch_count: kernels this library has enqueued in this process.
 * cucosma_profile_start / _stop: while on, every call records CUDA events on
 * its stream around its main GEMM kernel; _stop synchronises those events and
 * returns the summed kernel time (ms) and the number of timed launches. */
CUCOSMA_API unsigned long long cucosma_launch_count(void);
CUCOSMA_API cucosma_status cucosma_profile_start(void);
CUCOSMA_API cucosma_status cucosma_profile_stop(double* total_ms, int64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* CUCOSMA_H_ */
