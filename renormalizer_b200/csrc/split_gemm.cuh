// Split-precision tensor-core GEMM entry (BF16x3 / TF32x3 on tcgen05).
#pragma once
#include "reno_common.cuh"
#include "gemm_fp64.cuh"

namespace reno {
// Operand modes of the packed planes (rows x K', K-major, hi and lo):
//   0 real rows; 1 [re | im] along K (K' = 2K); 2 doubled complex rows
//   [re, -im] / [im, re] (K' = 2K); 3 doubled split rows re / im (K' = K)
enum SplitMode { SPLIT_REAL = 0, SPLIT_CAT = 1, SPLIT_DBL_CPLX = 2, SPLIT_DBL_SPLIT = 3 };

struct SplitPacked {
  void* hi;
  void* lo;
  int64_t pitch, rows, nb, kext;  // row pitch (elements), packed rows per batch, batches, K'
  int mode;
};

// multi-level source row order for split_pack: row r = (r2*D1 + r1)*D0 + r0 at
// r0*s_outer + r1*s_r1 + r2*s_r2 (D0 = 0: the operand's single row stride)
struct SplitRows {
  int D0 = 0, D1 = 1;
  int64_t s_r1 = 0, s_r2 = 0;
};

// where an epilogue writes the next stage's packed operand: element (m, n, ri)
// of batch bz -> bz*s_b + (m/Dm)*s_m1 + (m%Dm)*s_m0 + (n/Dn)*s_n1 + (n%Dn)*s_n0 + ri*s_ri
struct SplitPackOut {
  void* hi;
  void* lo;
  int64_t s_b, s_m1, s_m0, s_n1, s_n0, s_ri;
  int Dm, Dn;
};

int split_esz(int prec);
int64_t split_pitch(int64_t kext, int prec);
// bytes of a packed operand (both planes)
size_t split_packed_bytes(int64_t rows, int64_t kext, int64_t nb, int prec);
SplitPacked split_packed_at(void* base, int64_t rows, int64_t kext, int64_t nb, int mode, int prec);
// pack R rows x K of op (per batch) into dst (dst.mode decides the embedding)
cudaError_t split_pack(const GemmOperand& op, int R, int K, int nb, const SplitRows& rs, const SplitPacked& dst,
                       int prec, cudaStream_t st);
// C' = A' B'^T (M, N logical output dims) into C (c) or the next packed operand (po)
cudaError_t split_run(const SplitPacked& A, const SplitPacked& B, int M, int N, int batch, const GemmParams* c,
                      const SplitPackOut* po, int prec, cudaStream_t st);

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
