/*
 * reno_b200.h -- C ABI of the B200 sweep engine for Renormalizer's MPS sweep
 * hot path (effective-Hamiltonian matvec, environment updates, Krylov /
 * Davidson vector kernels, quantum-number block gather/scatter).
 *
 * Conventions
 *  - Every entry point returns an int status; RENO_OK (0) is success.  The
 *    message of the last failure is returned by reno_last_error().
 *  - Tensor arguments are DEVICE pointers owned by the caller, C-contiguous, in
 *    the reference's index order (cited per entry point).  complex128 is
 *    interleaved (re, im) doubles, 16-byte aligned.
 *  - Hot calls never allocate: scratch memory ("workspace") is passed in by
 *    the caller and sized by the matching *_workspace_bytes query.
 *  - Work is enqueued on the context's stream (reno_ctx_set_stream); calls are
 *    asynchronous unless documented otherwise.  One context per host thread.
 *
 * Reference interfaces replaced (paths inside the Renormalizer project):
 *  - reno_heff_apply   <- renormalizer/mps/hop_expr.py:7-117  hop_expr(...)(psi)
 *  - reno_env_update   <- renormalizer/mps/lib.py:169-250     contract_one_site
 *  - reno_vec_*        <- renormalizer/lib/krylov/krylov.py:27-84 (vdot, norm,
 *                         axpy, V @ coeffs, allclose) and the vector algebra
 *                         of renormalizer/lib/davidson/davidson.py:154-441
 *  - reno_qn_gather / reno_qn_scatter
 *                      <- renormalizer/mps/svd_qn.py:177-213 (block take) and
 *                         svd_qn.py:89-96 blockrecover, lib.py:302-316
 *                         select_basis column copy
 *  - reno_heff_diag    <- renormalizer/mps/gs.py:419-445 hdiag einsums
 *  - reno_lanczos_expm <- renormalizer/lib/krylov/krylov.py:27-84 expm_krylov
 *                         with the hop_expr operator
 *  - reno_qr_blocks    <- renormalizer/mps/svd_qn.py:195-204 (QR per QN block)
 *  - reno_qn_svd_truncate <- svd_qn.py:99-240 + lib.py:253-322 select_basis
 *                         + configs.py:196-219 compute_m_trunc (the sweeps'
 *                         truncation, mp.py:693-778)
 *  - reno_heev_*       <- svd_qn.py:12-49 / mp.py:693-778 (the truncation's
 *                         per-block factorisation, as a Gram eigenproblem)
 *  - reno_heff_backward   (no counterpart: gradients of the matvec)
 */
#ifndef RENO_B200_H
#define RENO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the Python shim maps them onto the reference's exceptions) */
enum {
  RENO_OK = 0,
  RENO_ERR_INVALID = 1,   /* shape / argument violation   -> AssertionError/ValueError */
  RENO_ERR_OOM = 2,       /* device allocation failure    -> MemoryError */
  RENO_ERR_CUDA = 3,      /* CUDA runtime error           -> RuntimeError */
  RENO_ERR_WORKSPACE = 4, /* workspace smaller than query -> MemoryError */
  RENO_ERR_NONFINITE = 5, /* NaN/Inf met                  -> FloatingPointError */
  RENO_ERR_UNSUPPORTED = 6
};

/* element types */
enum { RENO_F64 = 0, RENO_C128 = 1 };

/* arithmetic used for the tensor contractions */
enum {
  RENO_PREC_FP64 = 0,   /* FP64 DMMA, complex as four real products          */
  RENO_PREC_BF16X3 = 1, /* BF16 hi/lo split, three products, FP32 accumulate */
  RENO_PREC_TF32X3 = 2  /* TF32 hi/lo split, three products, FP32 accumulate */
};

typedef struct reno_ctx reno_ctx;

int reno_version(void);
int reno_ctx_create(int device, reno_ctx** out);
int reno_ctx_destroy(reno_ctx* ctx);
/* stream: a cudaStream_t (NULL = legacy default stream) */
int reno_ctx_set_stream(reno_ctx* ctx, void* stream);
const char* reno_last_error(const reno_ctx* ctx);
/* blocks until the context's stream is idle */
int reno_ctx_synchronize(reno_ctx* ctx);
/* number of kernels this library has launched in the process so far */
int reno_launch_count(long long* count);

/* ------------------------------------------------------------------------
 * Effective Hamiltonian matvec, hop_expr.py:57-103 (single layer, no ancilla)
 *   nsite 0:  y[a,l]     = sum L[a,b,c] R[l,b,k] C[c,k]                 (57-67)
 *   nsite 1:  y[a,d,l]   = sum L[a,b,c] W1[b,d,e,f] R[l,f,k] psi[c,e,k] (68-79)
 *   nsite 2:  y[a,d,g,l] = sum L[a,b,c] W1[b,d,e,f] W2[f,g,h,j]
 *                              R[l,j,k] psi[c,e,h,k]                     (92-103)
 * Shapes: L (ml, wl, ml); R (mr, wr, mr) (nsite 0: wr == wl);
 *         W1 (wl, d1, d1, wm) for nsite 2 and (wl, d1, d1, wr) for nsite 1;
 *         W2 (wm, d2, d2, wr); psi / y (ml, [d1, [d2,]] mr).
 * ---------------------------------------------------------------------- */
typedef struct {
  int32_t nsite;
  int32_t ml, mr;
  int32_t wl, wm, wr;
  int32_t d1, d2;
  int32_t psi_dtype; /* RENO_F64 / RENO_C128; y has the result dtype */
  int32_t env_dtype; /* dtype of L and R */
  int32_t mpo_dtype; /* dtype of W1 / W2 */
  int32_t prec;      /* RENO_PREC_* */
} reno_heff_desc;

int reno_heff_workspace_bytes(const reno_heff_desc* desc, size_t* bytes);
int reno_heff_apply(reno_ctx* ctx, const reno_heff_desc* desc, const void* L,
                    const void* W1, const void* W2, const void* R,
                    const void* psi, void* y, void* workspace,
                    size_t workspace_bytes);

/* Plain strided GEMM on the engine's kernels (bond-absorb products of the
 * sweeps, mps.py:1361/1394 tensordot; also the unit under test of the split
 * tensor-core path):
 *   C[m, n] = sum_k opA(A)[m, k] opB(B)[k, n],  C row stride c_rs, unit column
 *   stride; A[m,k] at m*a_rs + k*a_cs, B[k,n] at k*b_rs + n*b_cs; *_conj
 *   conjugates an operand; C is complex128 if A or B is.  prec RENO_PREC_FP64
 *   needs no workspace; the split modes need reno_gemm_workspace_bytes. */
int reno_gemm_workspace_bytes(int32_t M, int32_t N, int32_t K, int32_t a_dtype,
                              int32_t b_dtype, int32_t prec, size_t* bytes);
int reno_gemm(reno_ctx* ctx, int32_t M, int32_t N, int32_t K, const void* A,
              int32_t a_dtype, int64_t a_rs, int64_t a_cs, int32_t a_conj,
              const void* B, int32_t b_dtype, int64_t b_rs, int64_t b_cs,
              int32_t b_conj, void* C, int64_t c_rs, int32_t prec, void* ws,
              size_t ws_bytes);
/* Reads and clears the device-side error word of the tensor-core kernels:
 * 0 = none, 1000 + site = an mbarrier wait that ran out its bounded spin
 * (the kernel then skipped its remaining work and freed its TMEM). */
int reno_device_error(reno_ctx* ctx, int32_t* code);

/* Wall-clock limit of every bounded device wait -- the pipeline mbarriers of
 * the tensor-core GEMM and the grid barriers of the eigensolver reduction --
 * for launches made after the call; 1 ms .. 60 s, default 2 s. */
int reno_set_wait_limit_ns(uint64_t ns);
/* Promoted accumulation of the split-precision products (no counterpart in
 * the reference, which computes in FP64 on the host): the tensor cores'
 * FP32 accumulation truncates toward zero, so its relative error is a bias
 * that grows linearly with K.  With k_elems > 0, split GEMMs launched after
 * the call accumulate each run of k_elems K elements (rounded to whole 64-
 * (BF16) / 32- (TF32) element K tiles, at least one) in tensor memory and
 * add the runs' partial sums into round-to-nearest FP32 registers; the bias
 * then grows with k_elems instead of K.  0 (the default) turns it off. */
int reno_set_split_accumulation_chunk(int32_t k_elems);
/* Test hook of the failure path (no counterpart in the reference, which has
 * no device code): the NEXT launch of the named kernel has CTA 0 leave one
 * wait without its arrival, so that wait runs out after the limit above and
 * the kernel returns with its error status set (reno_device_error 1000 + site
 * for RENO_SKIP_SPLIT_STAGE, where `at` is the CTA's k-stage left unloaded;
 * the reduction's status word = 1 for RENO_SKIP_HETRD_ARRIVAL, where `at` is
 * the column whose barrier it skips).  at = -1 cancels.  Nothing faults: the
 * kernel drains its own copies, frees its tensor memory and exits. */
enum { RENO_SKIP_SPLIT_STAGE = 1, RENO_SKIP_HETRD_ARRIVAL = 2 };
int reno_test_skip_arrival(int32_t kind, int32_t at);

/* Allocation-free variant of reno_heff_apply.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory (hosts
 * that own the whole GPU through their own pool, foreign-language hosts that
 * cannot keep a device allocation alive) and pass only inputs and outputs.
 * Its scratch is a fixed array inside the library, RENO_NOALLOC_SCRATCH_BYTES
 * on every GPU that loads the library, held until the process exits; larger
 * problems are rejected with RENO_ERR_WORKSPACE.  All calls share the array
 * (calls that overlap on the GPU race, so serialise them); nothing in it has
 * to start at zero.  The first call on a device looks up the array's address
 * and should come before any stream capture. */
#define RENO_NOALLOC_SCRATCH_BYTES (128u << 20)
int reno_heff_apply_noalloc(reno_ctx* ctx, const reno_heff_desc* desc,
                            const void* L, const void* W1, const void* W2,
                            const void* R, const void* psi, void* y);

/* Grouped FP64 matvec for many independent local problems (static-disorder
 * realisations advanced in lockstep; the reference evolves each MPS on its
 * own through hop_expr.py:57-103): count (1..128) descriptors with the same
 * nsite and dtypes, each with its own dimensions; L, W1, W2, R, psi, y are
 * host arrays of count device pointers (W1 / W2 unused below 1 / 2 sites).
 * One launch transposes every MPO tensor, then each contraction stage is one
 * grouped GEMM launch; every problem's result is its reno_heff_apply result
 * at RENO_PREC_FP64.  Workspace from reno_heff_grouped_workspace_bytes. */
int reno_heff_grouped_workspace_bytes(int32_t count,
                                      const reno_heff_desc* descs,
                                      size_t* bytes);
int reno_heff_apply_grouped(reno_ctx* ctx, int32_t count,
                            const reno_heff_desc* descs, const void* const* L,
                            const void* const* W1, const void* const* W2,
                            const void* const* R, const void* const* psi,
                            void* const* y, void* ws, size_t ws_bytes);

/* Leading eigenpairs of a Hermitian Gram block for the truncation
 * (svd_qn.py:12-49 optimized_svd / mp.py:693-778, where the reference takes
 * LAPACK gesdd of the block; the engine diagonalises the block's Gram matrix).
 * reno_heev_top reduces A (n x n complex128, row-major, both triangles, a
 * private copy: reflector k is written into row k) to a real tridiagonal
 * matrix (d[n], e[n-1], tau[n-1] complex128) in one cooperative launch, then
 * writes the kt largest eigenvalues (ascending) to w and the matching
 * eigenvectors of the tridiagonal matrix (inverse iteration, not yet
 * orthonormalised) to Z (n x kt float64, row-major).  1 <= kt <= n <= 4096.
 * The caller orthonormalises Z and passes it as K (n x kt complex128);
 * reno_heev_backtransform overwrites K with Q K (blocked WY, FP64 GEMMs; A's
 * reflector rows are cleaned in place, same ws).  The int at
 * reno_heev_status_offset in ws is 0, or 1 when a grid-barrier wait of the
 * reduction timed out (results invalid). */
int reno_heev_workspace_bytes(int32_t n, int32_t kt, size_t* bytes);
int reno_heev_top(reno_ctx* ctx, int32_t n, int32_t kt, void* A, double* d,
                  double* e, void* tau, double* w, double* Z, void* ws,
                  size_t ws_bytes);
int reno_heev_backtransform(reno_ctx* ctx, int32_t n, int32_t kt, void* A,
                            const void* tau, void* K, void* ws,
                            size_t ws_bytes);
int reno_heev_status_offset(size_t* offset);

/* The same for up to RENO_HEEV_MAX_BATCH matrices at once (the QN blocks of
 * one bond): the matrices above 256 share one cooperative reduction launch,
 * the grid divided among them in proportion to n^2.  status[i] (device int)
 * receives problem i's status word.  k is used by the back-transformation
 * only.  Workspace from reno_heev_batched_workspace_bytes. */
#define RENO_HEEV_MAX_BATCH 32
typedef struct {
  int32_t n, kt;
  void* a;      /* n x n complex128, private copy, overwritten */
  double* d;    /* n */
  double* e;    /* n - 1 */
  void* tau;    /* n - 1 complex128 */
  double* w;    /* kt eigenvalues, ascending */
  double* z;    /* n x kt tridiagonal eigenvectors */
  void* k;      /* n x kt complex128: in Z (orthonormalised), out Q Z */
} reno_heev_problem;
int reno_heev_batched_workspace_bytes(int32_t count,
                                      const reno_heev_problem* probs,
                                      size_t* bytes);
int reno_heev_top_batched(reno_ctx* ctx, int32_t count,
                          const reno_heev_problem* probs, int32_t* status,
                          void* ws, size_t ws_bytes);
int reno_heev_backtransform_batched(reno_ctx* ctx, int32_t count,
                                    const reno_heev_problem* probs, void* ws,
                                    size_t ws_bytes);

/* Householder QR of the QN blocks of one site tensor, svd_qn.py:195-204
 * (scipy.linalg.qr(mode="economic") per block; the RQ of system "R" is the
 * QR of the reversed conjugate transpose, done by the caller).  LAPACK
 * conventions (zgeqrf/dgeqrf + zungqr/dorgqr): R's diagonal is
 * beta_j = -sign(Re alpha_j) |column|, so Q and R carry scipy's signs.
 * Each block: a (m x k, row-major, overwritten), q (m x min(m,k)), r
 * (min(m,k) x k, upper trapezoidal), all of one dtype.  1 <= count <=
 * RENO_QR_MAX_BLOCKS; m up to 81920.  Workspace from reno_qr_workspace_bytes. */
#define RENO_QR_MAX_BLOCKS 16
typedef struct {
  int32_t m, k, dtype, reserved;
  void* a;
  void* q;
  void* r;
} reno_qr_block;
int reno_qr_workspace_bytes(int32_t count, const reno_qr_block* blocks,
                            size_t* bytes);
int reno_qr_blocks(reno_ctx* ctx, int32_t count, const reno_qr_block* blocks,
                   void* workspace, size_t ws_bytes);

/* Lanczos exponential psi <- exp(dt H_eff) psi, krylov.py:27-84 expm_krylov
 * with the matvec of reno_heff_apply (desc, L, W1, W2, R as there; psi
 * complex128, dt = dt_re + i dt_im): the reference's stopping rule (results
 * of successive even steps j > 3 allclose at rtol 1e-5 / atol 1e-8, or a
 * breakdown beta_j < 100 n eps) and count, returned in out_k.  The host
 * synchronises at those checks only.  Fails with RENO_ERR_WORKSPACE when more
 * than kmax Krylov vectors would be needed.  Workspace from
 * reno_lanczos_workspace_bytes(desc, kmax). */
int reno_lanczos_workspace_bytes(const reno_heff_desc* desc, int32_t kmax,
                                 size_t* bytes);
int reno_lanczos_expm(reno_ctx* ctx, const reno_heff_desc* desc, const void* L,
                      const void* W1, const void* W2, const void* R,
                      double dt_re, double dt_im, void* psi, int32_t kmax,
                      int32_t* out_k, void* ws, size_t ws_bytes);

/* QN-blocked truncation of one coefficient matrix (rows x cols, row-major):
 * svd_qn.py:99-240 with select_basis lib.py:253-322 (percent 0) and
 * compute_m_trunc configs.py:196-219, as the sweeps use them (mp.py:693-778).
 * Per QN sector (left label nl, right label qntot - nl) the block's Gram
 * matrix of its smaller side goes through the device eigensolver (all blocks
 * in one batched call), Householder QR and the back-transformation; the
 * singular values are the norms of the projected vectors.  The kept triplets
 * are chosen like the reference: every block's values in block order, a
 * stable descending sort, then the count from the rule -- FIXED: min(m_max,
 * number of values); THRESHOLD: values with sigma / ||sigma|| > threshold;
 * BOTH: the smaller.  Outputs: left (rows x ldm) and right (ldm x cols), the
 * first *out_m columns / rows filled and the rest zero; keep_left = 1 gives
 * left = U (orthonormal columns) and right = sigma V^H, keep_left = 0 gives
 * left = U sigma and right = V^H (orthonormal rows).  sigma (host, ldm) and
 * qn_out (host, ldm x qn_size: the kept side's sector label of each column)
 * describe the kept columns.  Sectors are visited in the caller's order
 * (sectors, nsectors x qn_size; the reference iterates a Python set) or, with
 * nsectors = 0, in order of first appearance among the rows.  Zero-sigma
 * completion columns (full_matrices=True) are not produced.  At most
 * RENO_HEEV_MAX_BATCH sectors, smaller sides up to 4096; a block whose
 * eigensolver check fails returns RENO_ERR_UNSUPPORTED.  Workspace from
 * reno_qn_svd_truncate_workspace_bytes (same descriptor). */
enum { RENO_TRUNC_FIXED = 0, RENO_TRUNC_THRESHOLD = 1, RENO_TRUNC_BOTH = 2 };
typedef struct {
  int32_t rows, cols, qn_size, dtype;
  int32_t keep_left, mode, m_max, nsectors;
  double threshold;
  const int32_t* qn_rows;  /* host, rows x qn_size */
  const int32_t* qn_cols;  /* host, cols x qn_size */
  const int32_t* qntot;    /* host, qn_size */
  const int32_t* sectors;  /* host, nsectors x qn_size, or NULL */
} reno_trunc_desc;
int reno_qn_svd_truncate_workspace_bytes(const reno_trunc_desc* desc,
                                         size_t* bytes);
int reno_qn_svd_truncate(reno_ctx* ctx, const reno_trunc_desc* desc,
                         const void* coef, void* left, void* right,
                         int32_t ldm, double* sigma, int32_t* qn_out,
                         int32_t* out_m, void* ws, size_t ws_bytes);

/* Diagonal of the 1/2-site effective Hamiltonian, gs.py:419-445:
 *   nsite 1: hdiag[a,c,f]   = sum L[a,b,a] W1[b,c,c,g] R[f,g,f]
 *   nsite 2: hdiag[a,c,d,f] = sum L[a,b,a] W1[b,c,c,e] W2[e,d,d,g] R[f,g,f]
 * Only the real part is kept (the Davidson preconditioner is real). */
int reno_heff_diag(reno_ctx* ctx, const reno_heff_desc* desc, const void* L,
                   const void* W1, const void* W2, const void* R,
                   double* hdiag);

/* Reverse mode of reno_heff_apply.  No counterpart in the reference (it has
 * no gradients): for y = H_eff psi (hop_expr.py:57-103) and gy the gradient
 * with respect to y (torch's convention for complex tensors), writes
 *   gpsi = the matvec with conjugate-transposed L, W and R applied to gy
 *          (desc->prec, the fused split chains included);
 *   gL, gR, gW1, gW2 = contractions of gy with the conjugates of the other
 *          operands (FP64), each in the operand's own shape.
 * Every output pointer may be NULL (not computed).  Outputs are complex128
 * when any operand is complex, float64 otherwise (a caller holding a real
 * operand takes the real part).  gy has the type of y.  The workspace holds
 * the permuted operand copies and contraction intermediates; its size comes
 * from reno_heff_backward_workspace_bytes. */
int reno_heff_backward_workspace_bytes(const reno_heff_desc* desc, size_t* bytes);
int reno_heff_backward(reno_ctx* ctx, const reno_heff_desc* desc, const void* L,
                       const void* W1, const void* W2, const void* R,
                       const void* psi, const void* gy, void* gpsi, void* gL,
                       void* gW1, void* gW2, void* gR, void* ws,
                       size_t ws_bytes);

/* ------------------------------------------------------------------------
 * Environment update, lib.py:169-250 contract_one_site (3-leg site tensors).
 *  side 0 ("L", lib.py:200-205):
 *    out[f,g,h] = sum E[a,b,c] bra[a,d,f] W[b,d,e,g] ket[c,e,h]
 *    E (mb_in, w_in, mk_in); bra (mb_in, d, mb_out); ket (mk_in, d, mk_out);
 *    W (w_in, d, d, w_out); out (mb_out, w_out, mk_out)
 *  side 1 ("R", lib.py:232-237):
 *    out[f,g,h] = sum bra[f,d,a] E[a,b,c] W[g,d,e,b] ket[h,e,c]
 *    E (mb_in, w_in, mk_in); bra (mb_out, d, mb_in); ket (mk_out, d, mk_in);
 *    W (w_out, d, d, w_in); out (mb_out, w_out, mk_out)
 *  bra is the ALREADY-CONJUGATED bra tensor (the reference's ms_conj); pass
 *  NULL to use conj(ket) as the reference does when ms_conj is None.
 * ---------------------------------------------------------------------- */
typedef struct {
  int32_t side;
  int32_t d;
  int32_t w_in, w_out;
  int32_t mk_in, mk_out;
  int32_t mb_in, mb_out;
  int32_t env_dtype, ket_dtype, bra_dtype, mpo_dtype;
  int32_t prec;
} reno_env_desc;

int reno_env_workspace_bytes(const reno_env_desc* desc, size_t* bytes);
int reno_env_update(reno_ctx* ctx, const reno_env_desc* desc, const void* E,
                    const void* W, const void* ket, const void* bra, void* out,
                    void* workspace, size_t workspace_bytes);

/* ------------------------------------------------------------------------
 * Vector kernels for the Lanczos exponential (krylov.py:27-84) and Davidson
 * (davidson.py:154-441).  n counts elements of type dtype.  Scalars that the
 * reference keeps on the host live in caller-owned DEVICE double arrays here
 * (complex scalars as (re, im) pairs) so that no host sync is needed between
 * kernels.  All reductions are two-pass and deterministic (no atomics).
 * workspace: reno_vec_workspace_bytes(n) bytes.
 * ---------------------------------------------------------------------- */
int reno_vec_workspace_bytes(int64_t n, size_t* bytes);
/* out[0..1] = sum_i conj(x_i) * y_i  (numpy vdot(x, y)) */
int reno_vec_dotc(reno_ctx* ctx, int64_t n, int32_t dtype, const void* x,
                  const void* y, double* out, void* workspace, size_t ws_bytes);
/* out[0] = ||x||_2 (the caller checks it for NaN/Inf) */
int reno_vec_norm(reno_ctx* ctx, int64_t n, int32_t dtype, const void* x,
                  double* out, void* workspace, size_t ws_bytes);
/* Lanczos three-term step, krylov.py:244-245:
 *   w -= ab[2*j] * v + (j > 0 ? ab[2*j-1] * vprev : 0);  ab[2*j+1] = ||w||
 * where ab is the device array (alpha_0, beta_0, alpha_1, beta_1, ...). */
int reno_krylov_orth(reno_ctx* ctx, int64_t n, int32_t dtype, void* w,
                     const void* v, const void* vprev, double* ab, int32_t j,
                     void* workspace, size_t ws_bytes);
/* alpha_j = Re vdot(w, v) into ab[2*j], krylov.py:231 */
int reno_krylov_alpha(reno_ctx* ctx, int64_t n, int32_t dtype, const void* w,
                      const void* v, double* ab, int32_t j, void* workspace,
                      size_t ws_bytes);
/* out = x / s[0]   (krylov.py:256, V[j+1] = w / beta[j]) */
int reno_vec_scale_inv(reno_ctx* ctx, int64_t n, int32_t dtype, const void* x,
                       const double* s, void* out);
/* out = sum_{j<k} coef[j] * V[j]  with V rows of stride ldv elements;
 * coef complex (re, im) pairs on the device (krylov.py:24 V @ coeffs). */
int reno_vec_lincomb(reno_ctx* ctx, int64_t n, int32_t k, int32_t dtype,
                     const void* V, int64_t ldv, const double* coef, void* out);
/* flag[0] = 1.0 if allclose(a, b, rtol, atol) elementwise (numpy semantics,
 * |a-b| <= atol + rtol*|b|, complex modulus) else 0.0   (krylov.py:252) */
int reno_vec_allclose(reno_ctx* ctx, int64_t n, int32_t dtype, const void* a,
                      const void* b, double rtol, double atol, double* flag,
                      void* workspace, size_t ws_bytes);
/* y += c[0..1] * x   (complex scalar on the device; c_sign multiplies it) */
int reno_vec_axpy(reno_ctx* ctx, int64_t n, int32_t dtype, void* y,
                  const void* x, const double* c, double c_sign);
/* Davidson preconditioner, gs.py:532: out = r / (hdiag - e[0] + shift) */
int reno_vec_precond(reno_ctx* ctx, int64_t n, int32_t dtype, const void* r,
                     const double* hdiag, const double* e, double shift,
                     void* out);

/* ------------------------------------------------------------------------
 * Grouped vector kernels: one operation on up to RENO_VEC_GROUP_MAX
 * independent vectors of their own lengths and types in one or two launches
 * (the Lanczos exponentials of many static-disorder realisations advanced
 * in lockstep; the reference runs krylov.py:27-84 once per realisation).
 * Every item's result is bitwise the one of the single call above: the same
 * per-item block partition and summation order.
 *   RENO_VOP_NORM      scalars[0] = ||x||                 (reno_vec_norm)
 *   RENO_VOP_ALPHA     scalars[2j] = Re vdot(x, y)        (reno_krylov_alpha,
 *                      x = w, y = v, scalars = ab)
 *   RENO_VOP_ORTH      out -= ab[2j] x + ab[2j-1] y;  ab[2j+1] = ||out||
 *                      (reno_krylov_orth, out = w, x = v, y = vprev,
 *                      scalars = ab)
 *   RENO_VOP_SCALE_INV out = x / s[0]                     (reno_vec_scale_inv)
 *   RENO_VOP_LINCOMB   out = sum_{i<j} s[2i..2i+1] x[i ldv ..] (reno_vec_lincomb,
 *                      k = j vectors)
 *   RENO_VOP_ALLCLOSE  scalars[0] = allclose(x, y, rtol, atol)
 *                      (reno_vec_allclose)
 * workspace: reno_vec_grouped_workspace_bytes(count) bytes.
 * ---------------------------------------------------------------------- */
enum {
  RENO_VOP_NORM = 0,
  RENO_VOP_ALPHA = 1,
  RENO_VOP_ORTH = 2,
  RENO_VOP_SCALE_INV = 3,
  RENO_VOP_LINCOMB = 4,
  RENO_VOP_ALLCLOSE = 5
};
#define RENO_VEC_GROUP_MAX 128
typedef struct {
  int64_t n;           /* elements of each vector of this item */
  int32_t dtype;       /* RENO_F64 or RENO_C128 */
  int32_t j;           /* Krylov index (ALPHA, ORTH); vector count (LINCOMB) */
  const void* x;
  const void* y;
  void* out;
  double* scalars;
  const double* s;
  int64_t ldv;         /* LINCOMB: row stride of x in elements */
} reno_vec_item;
int reno_vec_grouped_workspace_bytes(int32_t count, size_t* bytes);
int reno_vec_grouped(reno_ctx* ctx, int32_t op, int32_t count,
                     const reno_vec_item* items, double rtol, double atol,
                     void* workspace, size_t ws_bytes);

/* ------------------------------------------------------------------------
 * Quantum-number block movers (svd_qn.py:177-213, 89-96; lib.py:302-316).
 * reno_qn_gather: out[i, j] = src[rows[i] * ld + cols[j]]   (nr x nc, dense out)
 * reno_qn_scatter: dst[rows[i] * dst_rs + dcols[j] * dst_cs] =
 *                     scale_j * src[i * src_rs + scols[j] * src_cs]
 *   with scale_j = (sigma ? sigma[j] : 1); rows/scols/dcols are int64 device
 *   arrays.  Places selected singular vectors (optionally sigma-weighted) of a
 *   QN block directly into a new site tensor.
 * ---------------------------------------------------------------------- */
int reno_qn_gather(reno_ctx* ctx, int32_t dtype, const void* src, int64_t ld,
                   const int64_t* rows, int64_t nr, const int64_t* cols,
                   int64_t nc, void* out);
int reno_qn_scatter(reno_ctx* ctx, int32_t dtype, const void* src,
                    int64_t src_rs, int64_t src_cs, const int64_t* rows,
                    int64_t nr, const int64_t* scols, const int64_t* dcols,
                    int64_t nc, const double* sigma, void* dst, int64_t dst_rs,
                    int64_t dst_cs);

#ifdef __cplusplus
}
#endif
#endif /* RENO_B200_H */
