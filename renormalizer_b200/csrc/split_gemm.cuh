// Split-precision tensor-core GEMM entry (BF16x3 / TF32x3 on tcgen05).
#pragma once
#include "reno_common.cuh"
#include "gemm_fp64.cuh"

namespace reno {
// workspace bytes split_gemm needs for this GEMM at this precision (0 for FP64)
size_t split_gemm_required_bytes(const GemmParams& p, int prec);
// legacy coarse bound on the workspace for operands of a_elems / b_elems elements
size_t split_gemm_workspace_bytes(int64_t a_elems, int64_t b_elems);
// C = opA(A) opB(B) with the operands rounded to hi/lo pairs of the chosen
// format (three products, FP32 accumulation), FP64 output
cudaError_t split_gemm(const GemmParams& p, int prec, void* ws, size_t ws_bytes, cudaStream_t st);
// first timed-out mbarrier wait since the last call (0 = none); clears it
int split_gemm_take_error();
}  // namespace reno
