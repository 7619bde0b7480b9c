// Split-precision tensor-core GEMM entry (BF16x3 / TF32x3 on tcgen05).
#pragma once
#include "reno_common.cuh"
#include "gemm_fp64.cuh"

namespace reno {
// bytes of staging memory the split GEMM needs for operands with at most
// a_elems / b_elems complex elements
size_t split_gemm_workspace_bytes(int64_t a_elems, int64_t b_elems);
// C = opA(A) opB(B) with the operands rounded to hi/lo pairs of the chosen
// format; returns cudaErrorNotSupported for shapes it does not take.
cudaError_t split_gemm(const GemmParams& p, int prec, void* ws, size_t ws_bytes, cudaStream_t st);
}  // namespace reno
