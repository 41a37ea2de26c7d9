// tc_gemm.cu -- tensor-core precision paths (filled in below as they land).
#include "api_internal.cuh"

namespace cucosma {
cucosma_status tc_workspace_size(const cucosma_gemm_desc*, size_t* bytes, const DeviceInfo*) {
  *bytes = 0;
  return CUCOSMA_STATUS_NOT_SUPPORTED;
}
cucosma_status tc_gemm(const cucosma_gemm_desc*, const void*, const void*, void*, void*, const DeviceInfo*,
                       cudaStream_t) {
  return CUCOSMA_STATUS_NOT_SUPPORTED;
}
}  // namespace cucosma
