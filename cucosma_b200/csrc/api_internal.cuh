// api_internal.cuh -- host-side declarations shared by the C ABI translation units.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/cucosma.h"

namespace cucosma {

struct DeviceInfo {
  bool valid = false;
  int sms = 0, cc_major = 0, cc_minor = 0, l2_bytes = 0, smem_optin = 0;
  int* status = nullptr;  // device address of the status word on this device
};
const DeviceInfo* device_info();
struct WaitCtl;
// Wait control for launches on the current device.
void wait_ctl(const DeviceInfo* di, int** status, unsigned long long* timeout_ns);

// Operand pre-passes of the tensor-core paths (see tc_gemm_ex).
// kNoFused: never the fused-split kernel, even with both pre-passes (the
// host-buffer call's row blocks share B's planes, which it does not write).
enum : int { kPrepA = 1, kPrepB = 2, kNoFused = 4 };

struct NativePlan {
  int bm;  // CTA tile rows: 128, or 64 (FP32 only); 128 columns either way
  int tiles_m, tiles_n, splits, swizzle;
  int64_t kchunk, ldw;
  size_t ws_bytes;
};
// Plan of the tile kernel (tile height and split-K factor); an automatic
// split-K factor is chosen so that its partial sums fit max_ws bytes.
NativePlan plan_native(const cucosma_gemm_desc* d, int sms, size_t max_ws = SIZE_MAX);

cucosma_status validate(const cucosma_gemm_desc* d, const void* A, const void* B, const void* C);
cucosma_status gemm(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws, size_t ws_bytes,
                    cudaStream_t st);
// The same with a choice of operand pre-passes for the tensor-core paths
// (kPrepA / kPrepB; the native paths have none).
cucosma_status gemm_ex(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws, size_t ws_bytes,
                       cudaStream_t st, int prep);

bool encode_2d(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, const void* base, uint64_t inner,
               uint64_t outer, uint64_t row_stride_elems, uint32_t box_inner, uint32_t box_outer,
               CUtensorMapSwizzle swz);
bool encode_3d(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, const void* base, uint64_t d0, uint64_t d1,
               uint64_t d2, uint64_t stride1_elems, uint64_t stride2_elems, uint32_t b0, uint32_t b1, uint32_t b2,
               CUtensorMapSwizzle swz);

// Tensor-core paths (BF16x3 / BF16x6 / Ozaki), tc_gemm.cu.
cucosma_status tc_workspace_size(const cucosma_gemm_desc* d, size_t* bytes, const DeviceInfo* di);
// allow_fused = false: the plan of a call whose operand planes are prepared
// by the caller (the fused-split kernel is then never chosen).
void tc_plan_info(const cucosma_gemm_desc* d, const DeviceInfo* di, cucosma_plan_info* info, bool allow_fused = true);
// Whether a plain call with *d runs the fused-split kernel.
bool tc_plan_is_fused(const cucosma_gemm_desc* d, const DeviceInfo* di);
// prep: which operand pre-passes run (kPrepA | kPrepB for a plain call).  An
// operand left out must already be in ws at the plan's offsets -- written by
// the caller (the backward pass), or by an earlier call on the same B (row
// blocks of one problem: B's planes / slices, exponents and magnitude sums
// sit first in the workspace and depend on N, K and the slice layout only).
// ws_bytes: the caller's workspace size; the plan actually run must fit it
// (WORKSPACE_TOO_SMALL otherwise, before anything is launched).
cucosma_status tc_gemm_ex(const cucosma_gemm_desc* d, const void* A, const void* B, void* C, void* ws,
                          size_t ws_bytes, const DeviceInfo* di, cudaStream_t st, int prep);

// The native tile kernel (no skinny-shape kernels) with plan pl; with a gate
// every kernel it enqueues runs only if *gate == gate_value on the device.
// Counts its launches; does not take part in the main-kernel profiling.
cucosma_status native_gemm_gated(const cucosma_gemm_desc* d, const NativePlan& pl, const void* A, const void* B,
                                 void* C, void* ws, const DeviceInfo* di, cudaStream_t st, const int* gate,
                                 int gate_value);

void* managed_workspace(size_t bytes, cudaStream_t st);

// Tuning cache (tune.cu): when d leaves split_k, swizzle and tile at 0 and the
// cache holds a choice for it, returns tmp filled with that choice, else d.
const cucosma_gemm_desc* apply_tuning(const cucosma_gemm_desc* d, cucosma_gemm_desc* tmp, const DeviceInfo* di);
// The grouped tile the tuner chose for this batch of shapes (cucosma_tune_grouped), 0 if none.
int grouped_tuned_tile(const cucosma_gemm_desc* d, const cucosma_gemm_problem* pr, int count, const DeviceInfo* di);

// Launch accounting and optional timing of the main GEMM kernel of each call:
// note_launches() counts every kernel the library enqueues; prof_begin /
// prof_end bracket the main kernel with CUDA events while profiling is on.
void note_launches(int n);
void prof_begin(cudaStream_t st);
void prof_end(cudaStream_t st);

}  // namespace cucosma
