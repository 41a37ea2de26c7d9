// tc_gemm.cuh -- parameters of the tcgen05 precision-path kernel.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace cucosma {

constexpr int kOzakiDefaultSlices = 8;

namespace tc {

constexpr int kThreads = 192;  // producer warp, MMA warp, 4 epilogue warps

struct TcParams {
  int m, n, k;
  int tiles_m, tiles_n;
  int kblocks;       // k-blocks of the whole K
  int kb_per_split;  // k-blocks per split-K unit
  int splits;
  int band;          // raster band height (tiles of M visited together)
  int epilogue;
  int partial;       // 1: raw partial sums into the workspace (split-K)
  double alpha, beta;
  void* out;
  int64_t ldo;
  int64_t ws_split_stride;
  const int32_t* ea;  // Ozaki row exponents of A
  const int32_t* eb;  // Ozaki column exponents of B
  WaitCtl ctl;
};

}  // namespace tc
}  // namespace cucosma
