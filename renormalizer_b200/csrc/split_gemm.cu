// Split-precision tensor-core GEMM (placeholder until the tcgen05 path lands).
#include "split_gemm.cuh"

namespace reno {
size_t split_gemm_workspace_bytes(int64_t a_elems, int64_t b_elems) { return 0; }
cudaError_t split_gemm(const GemmParams& p, int prec, void* ws, size_t ws_bytes, cudaStream_t st) {
  return cudaErrorNotSupported;
}
}  // namespace reno
