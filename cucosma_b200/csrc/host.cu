// host.cu -- GEMM on host (pinned) buffers with the copies overlapped.
//
// No counterpart in the reference, whose callers copy operands in and out
// themselves around cosmaSgemm (test_correctness.h).  The caller's device
// buffer holds device copies of A, B and C and the GEMM workspace.  B goes
// over first; A (and C when beta != 0) follow in row blocks, each block's
// GEMM (a row slice of the problem) runs as soon as its rows have arrived,
// and its C rows go back while later blocks still copy in -- so the
// host-to-device and device-to-host transfers run concurrently with each
// other and with the compute.  On the tensor-core paths B's operand planes
// (BF16 split or Ozaki slices, with its exponents) are prepared once, by the
// first block, and reused by the others.  Three streams per device (created
// on first use) carry the copies in, the GEMMs and the copies out; the
// events that order them are created for each call, so calls from several
// host threads never share one.  The caller's stream waits for the last
// copy out.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/cucosma.h"
#include "api_internal.cuh"
#include "common.cuh"

namespace cucosma {
namespace {

constexpr int kMaxBlocks = 16;

struct HostStreams {
  cudaStream_t in = nullptr, gemm = nullptr, out = nullptr;
  bool ok = false;
};

// The events of one call (destroyed when the call returns; CUDA releases an
// event that is still pending once its work completes).
struct CallEvents {
  cudaEvent_t start = nullptr, b_in = nullptr, done = nullptr;
  cudaEvent_t a_in[kMaxBlocks] = {}, c_ready[kMaxBlocks] = {};
  bool create(int blocks) {
    auto mk = [](cudaEvent_t* e) { return cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess; };
    if (!mk(&start) || !mk(&b_in) || !mk(&done)) return false;
    for (int i = 0; i < blocks; ++i)
      if (!mk(&a_in[i]) || !mk(&c_ready[i])) return false;
    return true;
  }
  ~CallEvents() {
    for (cudaEvent_t e : {start, b_in, done})
      if (e) cudaEventDestroy(e);
    for (int i = 0; i < kMaxBlocks; ++i) {
      if (a_in[i]) cudaEventDestroy(a_in[i]);
      if (c_ready[i]) cudaEventDestroy(c_ready[i]);
    }
  }
};

HostStreams* streams_for_current_device() {
  static std::mutex mu;
  static HostStreams per_device[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  HostStreams& h = per_device[dev];
  if (!h.ok) {
    const bool good = cudaStreamCreateWithFlags(&h.in, cudaStreamNonBlocking) == cudaSuccess &&
                      cudaStreamCreateWithFlags(&h.gemm, cudaStreamNonBlocking) == cudaSuccess &&
                      cudaStreamCreateWithFlags(&h.out, cudaStreamNonBlocking) == cudaSuccess;
    if (!good) return nullptr;
    h.ok = true;
  }
  return &h;
}

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

struct HostLayout {
  int blocks;
  int64_t rows_per_block;
  size_t off_a, off_b, off_c, off_ws, ws_bytes, total;
  int64_t lda, ldb, ldc;  // device row strides (16-byte rows)
};

cucosma_status host_layout(const cucosma_gemm_desc* d, HostLayout* L) {
  if (!d || d->m <= 0 || d->n <= 0 || d->k <= 0) return CUCOSMA_STATUS_INVALID_VALUE;
  const int es = d->dtype == CUCOSMA_R_32F ? 4 : 8;
  const int64_t vec = 16 / es;
  L->lda = round_up(d->k, vec);
  L->ldb = round_up(d->n, vec);
  L->ldc = round_up(d->n, vec);
  // Row blocks of at least 512 rows (two 256-row pair tiles: a block still
  // fills most of the SMs), at most kMaxBlocks of them.  More, smaller blocks
  // shorten the tail after the last input copy (that block's GEMM and the
  // copy-out of its C): 8192^3 BF16x6 went from 8 to 16 blocks.
  L->blocks = (int)std::max<int64_t>(1, std::min<int64_t>(kMaxBlocks, d->m / 512));
  L->rows_per_block = round_up(ceil_div(d->m, L->blocks), 128);
  L->blocks = (int)ceil_div(d->m, L->rows_per_block);
  // The regular entry point's workspace for a full row block and for the
  // last (possibly shorter) one; the larger serves every block in turn.
  L->ws_bytes = 0;
  const int64_t sizes[2] = {std::min<int64_t>(d->m, L->rows_per_block),
                            d->m - (int64_t)(L->blocks - 1) * L->rows_per_block};
  for (int64_t rows : sizes) {
    cucosma_gemm_desc sub = *d;
    sub.m = rows;
    sub.lda = L->lda;
    sub.ldb = L->ldb;
    sub.ldc = L->ldc;
    size_t b = 0;
    cucosma_status s = cucosma_gemm_workspace_size(&sub, &b);
    if (s != CUCOSMA_STATUS_SUCCESS) return s;
    if (L->blocks > 1 && (d->precision == CUCOSMA_PRECISION_BF16X3 || d->precision == CUCOSMA_PRECISION_BF16X6)) {
      // several row blocks run the pre-pass path (B's planes shared): its plan's workspace
      const DeviceInfo* di = device_info();
      if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
      cucosma_gemm_desc tuned;
      cucosma_plan_info pi;
      tc_plan_info(apply_tuning(&sub, &tuned, di), di, &pi, false);
      b = std::max(b, (size_t)pi.workspace_bytes);
    }
    L->ws_bytes = std::max(L->ws_bytes, b);
  }
  size_t off = 0;
  L->off_a = off;
  off = al256(off + (size_t)d->m * L->lda * es);
  L->off_b = off;
  off = al256(off + (size_t)d->k * L->ldb * es);
  L->off_c = off;
  off = al256(off + (size_t)d->m * L->ldc * es);
  L->off_ws = off;
  off = al256(off + L->ws_bytes);
  L->total = off;
  return CUCOSMA_STATUS_SUCCESS;
}

}  // namespace
}  // namespace cucosma

using namespace cucosma;

extern "C" cucosma_status cucosma_gemm_host_buffer_size(const cucosma_gemm_desc* d, size_t* bytes) {
  if (!bytes) return CUCOSMA_STATUS_INVALID_VALUE;
  HostLayout L;
  cucosma_status s = host_layout(d, &L);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  *bytes = L.total;
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_gemm_host(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                            void* device_buffer, size_t buffer_bytes, void* stream) {
  HostLayout L;
  cucosma_status s = host_layout(d, &L);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (!A || !B || !C) return CUCOSMA_STATUS_INVALID_VALUE;
  if (d->lda < d->k || d->ldb < d->n || d->ldc < d->n) return CUCOSMA_STATUS_INVALID_VALUE;
  if (!device_buffer || buffer_bytes < L.total) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  if (reinterpret_cast<uintptr_t>(device_buffer) & 255) return CUCOSMA_STATUS_MISALIGNED;
  HostStreams* h = streams_for_current_device();
  if (!h) return CUCOSMA_STATUS_LAUNCH_FAILED;
  CallEvents ev;
  if (!ev.create(L.blocks)) return CUCOSMA_STATUS_LAUNCH_FAILED;
  // Several row blocks share B's planes, prepared by the first (the fused
  // split, which keeps none, is not used then: per block it would read and
  // split B again -- 512-row blocks of 8192^3 BF16x6 chose it and ran 12 %
  // slower end to end).  A single block may take the fused kernel.
  bool b_shared = true;
  const int no_fused = L.blocks > 1 ? kNoFused : 0;
  if (L.blocks == 1 && (d->precision == CUCOSMA_PRECISION_BF16X3 || d->precision == CUCOSMA_PRECISION_BF16X6)) {
    const DeviceInfo* di = device_info();
    if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
    cucosma_gemm_desc first = *d;
    first.m = std::min<int64_t>(L.rows_per_block, d->m);
    first.lda = L.lda;
    first.ldb = L.ldb;
    first.ldc = L.ldc;
    cucosma_gemm_desc tuned;
    b_shared = !tc_plan_is_fused(apply_tuning(&first, &tuned, di), di);
  }
  const size_t es = d->dtype == CUCOSMA_R_32F ? 4 : 8;
  uint8_t* w = static_cast<uint8_t*>(device_buffer);
  uint8_t* dA = w + L.off_a;
  uint8_t* dB = w + L.off_b;
  uint8_t* dC = w + L.off_c;
  void* ws = L.ws_bytes ? w + L.off_ws : nullptr;
  const uint8_t* hA = static_cast<const uint8_t*>(A);
  const uint8_t* hB = static_cast<const uint8_t*>(B);
  uint8_t* hC = static_cast<uint8_t*>(C);
  cudaStream_t caller = static_cast<cudaStream_t>(stream);
  auto fail = [](cudaError_t e) { return e != cudaSuccess; };

  // Everything starts after the work already queued on the caller's stream.
  if (fail(cudaEventRecord(ev.start, caller)) || fail(cudaStreamWaitEvent(h->in, ev.start, 0)) ||
      fail(cudaStreamWaitEvent(h->gemm, ev.start, 0)) || fail(cudaStreamWaitEvent(h->out, ev.start, 0)))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (fail(cudaMemcpy2DAsync(dB, L.ldb * es, hB, d->ldb * es, d->n * es, d->k, cudaMemcpyHostToDevice, h->in)) ||
      fail(cudaEventRecord(ev.b_in, h->in)) || fail(cudaStreamWaitEvent(h->gemm, ev.b_in, 0)))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  for (int i = 0; i < L.blocks; ++i) {
    const int64_t r0 = i * L.rows_per_block, rows = std::min<int64_t>(L.rows_per_block, d->m - r0);
    if (fail(cudaMemcpy2DAsync(dA + r0 * L.lda * es, L.lda * es, hA + r0 * d->lda * es, d->lda * es, d->k * es, rows,
                               cudaMemcpyHostToDevice, h->in)))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    if (d->beta != 0.0 &&
        fail(cudaMemcpy2DAsync(dC + r0 * L.ldc * es, L.ldc * es, hC + r0 * d->ldc * es, d->ldc * es, d->n * es, rows,
                               cudaMemcpyHostToDevice, h->in)))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    if (fail(cudaEventRecord(ev.a_in[i], h->in)) || fail(cudaStreamWaitEvent(h->gemm, ev.a_in[i], 0)))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    cucosma_gemm_desc sub = *d;
    sub.m = rows;
    sub.lda = L.lda;
    sub.ldb = L.ldb;
    sub.ldc = L.ldc;
    // B's operand planes: prepared by the first block, reused by the rest.
    s = gemm_ex(&sub, dA + r0 * L.lda * es, dB, dC + r0 * L.ldc * es, ws, L.ws_bytes, h->gemm,
                ((i == 0 || !b_shared) ? (kPrepA | kPrepB) : kPrepA) | no_fused);
    if (s != CUCOSMA_STATUS_SUCCESS) return s;
    if (fail(cudaEventRecord(ev.c_ready[i], h->gemm)) || fail(cudaStreamWaitEvent(h->out, ev.c_ready[i], 0)) ||
        fail(cudaMemcpy2DAsync(hC + r0 * d->ldc * es, d->ldc * es, dC + r0 * L.ldc * es, L.ldc * es, d->n * es, rows,
                               cudaMemcpyDeviceToHost, h->out)))
      return CUCOSMA_STATUS_LAUNCH_FAILED;
  }
  if (fail(cudaEventRecord(ev.done, h->out)) || fail(cudaStreamWaitEvent(caller, ev.done, 0)))
    return CUCOSMA_STATUS_LAUNCH_FAILED;
  return CUCOSMA_STATUS_SUCCESS;
}
