// backward.cu -- gradients of the fused forward Y = epi(alpha * A*B + beta*C0).
//
// No counterpart in the reference (forward only; its sigmoid epilogue is the
// commented block at cuCOSMAV100.cuh:2472-2476).  With G = alpha * dY (.)
// epi'(Z), epi' = Y(1-Y) for the sigmoid, [Y > 0] for ReLU, 1 for none:
//   dA = G * B^T   (m x k)        dB = A^T * G   (k x n)
// Both products run on the tcgen05 BF16 kernel of the forward precision.  The
// transposed operands are never materialised: the split pre-pass writes the
// K-major planes each product needs straight from the saved operands --
//   dA: A-planes = rows of G (computed from dY and Y inside the split),
//       B-planes = rows of B itself (B^T's K-major layout is B);
//   dB: A-planes = columns of A (A^T, transposing split),
//       B-planes = columns of G (G^T, transposing split, G computed again).
// Six launches (four splits, two GEMMs), one caller workspace reused by both
// products in stream order.
#include <algorithm>

#include "../../include/cucosma.h"
#include "api_internal.cuh"
#include "split.cuh"

namespace cucosma {
namespace {

bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

void sub_desc(const cucosma_gemm_desc* f, int64_t m, int64_t n, int64_t k, int64_t ldc, cucosma_gemm_desc* d) {
  cucosma_gemm_desc_init(d);
  d->m = m;
  d->n = n;
  d->k = k;
  d->lda = k;  // operand strides unused: the planes are prepared here
  d->ldb = n;
  d->ldc = ldc;
  d->dtype = CUCOSMA_R_32F;
  d->precision = f->precision;
  d->tile = f->tile;
  d->split_k = 0;
  d->alpha = 1.0;
  d->beta = 0.0;
}

int xform_of(int epilogue) {
  return epilogue == CUCOSMA_EPILOGUE_SIGMOID ? kXformSigmoidGrad
         : epilogue == CUCOSMA_EPILOGUE_RELU  ? kXformReluGrad
                                               : kXformScale;
}

cucosma_status check_bwd(const cucosma_gemm_desc* f) {
  if (!f) return CUCOSMA_STATUS_INVALID_VALUE;
  if (f->m <= 0 || f->n <= 0 || f->k <= 0 || f->m > INT32_MAX || f->n > INT32_MAX || f->k > INT32_MAX)
    return CUCOSMA_STATUS_INVALID_VALUE;
  if (f->dtype != CUCOSMA_R_32F) return CUCOSMA_STATUS_NOT_SUPPORTED;
  if (f->precision != CUCOSMA_PRECISION_BF16X3 && f->precision != CUCOSMA_PRECISION_BF16X6)
    return CUCOSMA_STATUS_NOT_SUPPORTED;
  if (f->epilogue < 0 || f->epilogue > CUCOSMA_EPILOGUE_RELU || f->flags) return CUCOSMA_STATUS_INVALID_VALUE;
  return CUCOSMA_STATUS_SUCCESS;
}

}  // namespace
}  // namespace cucosma

using namespace cucosma;

extern "C" cucosma_status cucosma_gemm_backward_workspace_size(const cucosma_gemm_desc* f, size_t* bytes) {
  if (!bytes) return CUCOSMA_STATUS_INVALID_VALUE;
  cucosma_status s = check_bwd(f);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  // Each product's plan as the backward call builds it: tuned, and with its
  // planes prepared here (never the fused-split kernel, which keeps none).
  auto need = [&](int64_t m, int64_t n, int64_t k, int64_t ldc) {
    cucosma_gemm_desc d0, tuned;
    cucosma_plan_info pi;
    sub_desc(f, m, n, k, ldc, &d0);
    tc_plan_info(apply_tuning(&d0, &tuned, di), di, &pi, false);
    return pi.workspace_bytes;
  };
  *bytes = std::max(need(f->m, f->k, f->n, f->k), need(f->k, f->n, f->m, f->n));
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_gemm_backward(const cucosma_gemm_desc* f, const void* A, const void* B,
                                                const void* Y, int64_t ldy, const void* dY, int64_t lddy, void* dA,
                                                int64_t ldda, void* dB, int64_t lddb, void* workspace,
                                                size_t workspace_bytes, void* stream) {
  cucosma_status s = check_bwd(f);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  const int64_t m = f->m, n = f->n, k = f->k;
  if (!dY || (!dA && !dB)) return CUCOSMA_STATUS_INVALID_VALUE;
  if (f->epilogue != CUCOSMA_EPILOGUE_NONE && (!Y || ldy < n)) return CUCOSMA_STATUS_INVALID_VALUE;
  if (lddy < n || (dA && (!B || f->ldb < n || ldda < k)) || (dB && (!A || f->lda < k || lddb < n)))
    return CUCOSMA_STATUS_INVALID_VALUE;
  auto bad16 = [](const void* p, int64_t ld) { return p && (!al16(p) || (ld * 4) % 16); };
  if (bad16(dY, lddy) || (f->epilogue != CUCOSMA_EPILOGUE_NONE && bad16(Y, ldy)) || (dA && bad16(B, f->ldb)) ||
      (dB && bad16(A, f->lda)) || bad16(dA, ldda) || bad16(dB, lddb))
    return CUCOSMA_STATUS_MISALIGNED;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  if (di->cc_major != 10 || di->cc_minor != 0) return CUCOSMA_STATUS_ARCH_MISMATCH;
  size_t need = 0;
  if ((s = cucosma_gemm_backward_workspace_size(f, &need)) != CUCOSMA_STATUS_SUCCESS) return s;
  if (!workspace || workspace_bytes < need) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  if (!al16(workspace)) return CUCOSMA_STATUS_MISALIGNED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint8_t* w = static_cast<uint8_t*>(workspace);
  const int nt = f->precision == CUCOSMA_PRECISION_BF16X6 ? 3 : 2;
  const int xf = xform_of(f->epilogue);
  const float scale = (float)f->alpha;
  const float* fY = static_cast<const float*>(Y);
  const float* fdY = static_cast<const float*>(dY);
  cucosma_plan_info pi;
  // Each product's descriptor is resolved against the tuning cache once and
  // that one descriptor gives both the plan (plane offsets, partials region)
  // and the launch, so the two cannot disagree; the plan must fit the
  // caller's workspace (the cache may have changed since it was sized).
  auto resolve = [&](cucosma_gemm_desc* d, cucosma_gemm_desc* tuned) -> const cucosma_gemm_desc* {
    const cucosma_gemm_desc* r = apply_tuning(d, tuned, di);
    tc_plan_info(r, di, &pi, false);  // the planes are prepared here: never the fused kernel
    return r;
  };
  if (dA) {
    // dA (m x k) = G (m x n) * B^T: K' = n.
    cucosma_gemm_desc d0, tuned;
    sub_desc(f, m, k, n, ldda, &d0);
    const cucosma_gemm_desc* d = resolve(&d0, &tuned);
    if (pi.workspace_bytes > workspace_bytes) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
    if (launch_split_bf16(fdY, lddy, (int)m, (int)n, pi.kpad, nt, w + pi.off_a, false, di->sms, st, xf, fY, ldy,
                          scale) != cudaSuccess ||
        launch_split_bf16(static_cast<const float*>(B), f->ldb, (int)k, (int)n, pi.kpad, nt, w + pi.off_b, false,
                          di->sms, st) != cudaSuccess)
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    note_launches(2);
    if ((s = tc_gemm_ex(d, nullptr, nullptr, dA, workspace, workspace_bytes, di, st, 0)) != CUCOSMA_STATUS_SUCCESS) return s;
  }
  if (dB) {
    // dB (k x n) = A^T (k x m) * G (m x n): K' = m.
    cucosma_gemm_desc d0, tuned;
    sub_desc(f, k, n, m, lddb, &d0);
    const cucosma_gemm_desc* d = resolve(&d0, &tuned);
    if (pi.workspace_bytes > workspace_bytes) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
    if (launch_split_bf16(static_cast<const float*>(A), f->lda, (int)m, (int)k, pi.kpad, nt, w + pi.off_a, true,
                          di->sms, st) != cudaSuccess ||
        launch_split_bf16(fdY, lddy, (int)m, (int)n, pi.kpad, nt, w + pi.off_b, true, di->sms, st, xf, fY, ldy,
                          scale) != cudaSuccess)
      return CUCOSMA_STATUS_LAUNCH_FAILED;
    note_launches(2);
    if ((s = tc_gemm_ex(d, nullptr, nullptr, dB, workspace, workspace_bytes, di, st, 0)) != CUCOSMA_STATUS_SUCCESS) return s;
  }
  return CUCOSMA_STATUS_SUCCESS;
}
