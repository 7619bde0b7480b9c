// Effective-Hamiltonian matvec (hop_expr) and environment update
// (contract_one_site) as chains of strided GEMM stages.
//
// Stage order (all operands in the reference's C-order layouts, no permutes):
//   1-site  (hop_expr.py:68-79):  T1[a,b,e,k] = L[ab,c] psi[c,ek]
//                                  T2[a,d,f,k] = Wt[df,be] T1[a][be,k]   (batched over a)
//                                  y[a,d,l]    = T2[ad,fk] R[l,fk]
//   2-site  (hop_expr.py:92-103): T1 = L.psi ; T2 = Wt1.T1[a] ; T3 = Wt2.T2[a,d] ; y = T3.R^T
//   0-site  (hop_expr.py:57-67):  T1[a,b,k] = L[ab,c] C[c,k] ; y[a,l] = T1[a,bk] R[l,bk]
//   env L   (lib.py:200-205):     T1 = E.ket ; T2 = Wt.T1[a] ; out[f,gh] = bra[ad,f] T2[ad,gh]
//   env R   (lib.py:232-237):     the L form on the bond-transposed bra/ket and W with its
//                                  two MPO bonds swapped (an R update is an L update of the
//                                  mirrored chain)
#include "reno_common.cuh"
#include "gemm_fp64.cuh"
#include "split_gemm.cuh"
#include <algorithm>
#include <memory>
#include <vector>

namespace reno {

static inline int64_t esz(int dt) { return dt == RENO_C128 ? 16 : 8; }
static inline int promote(int a, int b) { return (a == RENO_C128 || b == RENO_C128) ? RENO_C128 : RENO_F64; }
static inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Wt[(dd, r), (c, e)] from W.  mode 0: W is (nc, d, d, nr) indexed [c,dd,e,r];
// mode 1: W is (nr, d, d, nc) indexed [r,dd,e,c] (MPO bonds swapped).
template <typename T>
__global__ void wt_kernel(const T* __restrict__ W, T* __restrict__ Wt, int nc, int d, int nr, int mode) {
  const int64_t total = (int64_t)d * nr * nc * d;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int e = idx % d;
    const int c = (idx / d) % nc;
    const int r = (idx / ((int64_t)d * nc)) % nr;
    const int dd = idx / ((int64_t)d * nc * nr);
    int64_t widx;
    if (mode == 0)
      widx = (((int64_t)c * d + dd) * d + e) * nr + r;
    else
      widx = (((int64_t)r * d + dd) * d + e) * nc + c;
    Wt[idx] = W[widx];
  }
}

// out[c,e,h] = in[h,e,c] : in (n0, d, n2) -> out (n2, d, n0)
template <typename T>
__global__ void swap13_kernel(const T* __restrict__ in, T* __restrict__ out, int n0, int d, int n2) {
  const int64_t total = (int64_t)n0 * d * n2;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int h = idx % n0;
    const int e = (idx / n0) % d;
    const int c = idx / ((int64_t)n0 * d);
    out[idx] = in[((int64_t)h * d + e) * n2 + c];
  }
}

static int grid_for(int64_t total) {
  int64_t g = ceil_div(total, 256);
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

static cudaError_t launch_wt(const void* W, void* Wt, int dt, int nc, int d, int nr, int mode, cudaStream_t st) {
  const int64_t total = (int64_t)d * nr * nc * d;
  count_launch();
  if (dt == RENO_C128)
    wt_kernel<double2><<<grid_for(total), 256, 0, st>>>((const double2*)W, (double2*)Wt, nc, d, nr, mode);
  else
    wt_kernel<double><<<grid_for(total), 256, 0, st>>>((const double*)W, (double*)Wt, nc, d, nr, mode);
  return cudaGetLastError();
}

static cudaError_t launch_swap13(const void* in, void* out, int dt, int n0, int d, int n2, cudaStream_t st) {
  const int64_t total = (int64_t)n0 * d * n2;
  count_launch();
  if (dt == RENO_C128)
    swap13_kernel<double2><<<grid_for(total), 256, 0, st>>>((const double2*)in, (double2*)out, n0, d, n2);
  else
    swap13_kernel<double><<<grid_for(total), 256, 0, st>>>((const double*)in, (double*)out, n0, d, n2);
  return cudaGetLastError();
}

static GemmOperand opnd(const void* p, int dt, int64_t s_outer, int64_t s_k, int64_t s_b = 0, int conj = 0,
                        int f32 = 0) {
  GemmOperand o;
  o.ptr = p;
  o.is_complex = dt == RENO_C128;
  o.s_outer = s_outer;
  o.s_k = s_k;
  o.s_batch = s_b;
  o.conj = conj;
  o.is_f32 = f32;
  return o;
}

// an intermediate operand: FP32 storage between split-precision stages
static GemmOperand iopnd(const void* p, int dt, int f32, int64_t s_outer, int64_t s_k, int64_t s_b = 0) {
  return opnd(p, dt, s_outer, s_k, s_b, 0, f32);
}

static GemmParams to_f32(GemmParams p, int f32) {
  p.c_f32 = f32;
  return p;
}

static GemmParams gp(int M, int N, int K, int batch, GemmOperand A, GemmOperand B, void* C, int64_t sCm,
                     int64_t sCn, int64_t sCb = 0) {
  GemmParams p;
  p.M = M;
  p.N = N;
  p.K = K;
  p.batch = batch;
  p.A = A;
  p.B = B;
  p.C = C;
  p.sCm = sCm;
  p.sCn = sCn;
  p.sCb = sCb;
  return p;
}

// One GEMM stage of a contraction chain at a given arithmetic.
struct Stage {
  GemmParams p;
  int prec;
};

static cudaError_t run_stage(const Stage& s, void* split_ws, size_t split_ws_bytes, cudaStream_t st) {
  if (s.prec == RENO_PREC_FP64) return gemm_fp64(s.p, st);
  return split_gemm(s.p, s.prec, split_ws, split_ws_bytes, st);
}

static size_t split_need(const std::vector<Stage>& stages) {
  size_t m = 0;
  for (const Stage& s : stages) m = std::max(m, split_gemm_required_bytes(s.p, s.prec));
  return m;
}

// ---------------------------------------------------------------- heff
// Intermediates (T1, T2, T3) are FP64 on the FP64 path and FP32 between
// split-precision stages, whose tensor-core accumulators are FP32 anyway.
struct HeffLayout {
  int dt_T1, dt_T2, dt_y, t32;
  size_t off_wt1, off_wt2, off_t1, off_t2, off_split;
};

static int validate_heff(const reno_heff_desc* d) {
  if (!d) return RENO_ERR_INVALID;
  if (d->nsite < 0 || d->nsite > 2) return RENO_ERR_INVALID;
  if (d->ml <= 0 || d->mr <= 0 || d->wl <= 0 || d->wr <= 0) return RENO_ERR_INVALID;
  if (d->nsite >= 1 && d->d1 <= 0) return RENO_ERR_INVALID;
  if (d->nsite == 2 && (d->d2 <= 0 || d->wm <= 0)) return RENO_ERR_INVALID;
  if (d->nsite == 0 && d->wl != d->wr) return RENO_ERR_INVALID;
  for (int t : {d->psi_dtype, d->env_dtype, d->mpo_dtype})
    if (t != RENO_F64 && t != RENO_C128) return RENO_ERR_INVALID;
  if (d->prec < RENO_PREC_FP64 || d->prec > RENO_PREC_TF32X3) return RENO_ERR_INVALID;
  return RENO_OK;
}

static HeffLayout heff_layout(const reno_heff_desc* d) {
  HeffLayout p{};
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wm = d->wm, wr = d->wr, d1 = d->d1, d2 = d->d2;
  p.dt_T1 = promote(d->env_dtype, d->psi_dtype);
  p.dt_T2 = d->nsite == 0 ? p.dt_T1 : promote(p.dt_T1, d->mpo_dtype);
  p.dt_y = promote(p.dt_T2, d->env_dtype);
  p.t32 = d->prec != RENO_PREC_FP64;
  int64_t n_wt1 = 0, n_wt2 = 0, n_t1 = 0, n_t2 = 0;
  if (d->nsite == 0) {
    n_t1 = ml * wl * mr;
  } else if (d->nsite == 1) {
    n_wt1 = d1 * wr * wl * d1;
    n_t1 = ml * wl * d1 * mr;
    n_t2 = ml * d1 * wr * mr;
  } else {
    n_wt1 = d1 * wm * wl * d1;
    n_wt2 = d2 * wr * wm * d2;
    n_t1 = std::max(ml * wl * d1 * d2 * mr, ml * d1 * d2 * wr * mr);  // T1, later reused for T3
    n_t2 = ml * d1 * wm * d2 * mr;
  }
  size_t off = 0;
  p.off_wt1 = off;
  off = align256(off + n_wt1 * esz(d->mpo_dtype));
  p.off_wt2 = off;
  off = align256(off + n_wt2 * esz(d->mpo_dtype));
  const int64_t tsz = esz(p.dt_T2) / (p.t32 ? 2 : 1);
  p.off_t1 = off;
  off = align256(off + n_t1 * tsz);
  p.off_t2 = off;
  off = align256(off + n_t2 * tsz);
  p.off_split = off;
  return p;
}

// the GEMM stages of hop_expr.py:57-103 with the reference's C-order strides
static std::vector<Stage> heff_stages(const reno_heff_desc* d, const HeffLayout& lay, char* w, const void* L,
                                      const void* R, const void* psi, void* y) {
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wm = d->wm, wr = d->wr, d1 = d->d1, d2 = d->d2;
  const int ev = d->env_dtype, pv = d->psi_dtype, mv = d->mpo_dtype, pr = d->prec;
  void* Wt1 = w + lay.off_wt1;
  void* Wt2 = w + lay.off_wt2;
  void* T1 = w + lay.off_t1;
  void* T2 = w + lay.off_t2;
  const int f = lay.t32;
  std::vector<Stage> s;
  if (d->nsite == 0) {
    s.push_back({to_f32(gp(ml * wl, mr, ml, 1, opnd(L, ev, ml, 1), opnd(psi, pv, 1, mr), T1, mr, 1), f), pr});
    s.push_back({gp(ml, mr, wl * mr, 1, iopnd(T1, lay.dt_T1, f, wl * mr, 1), opnd(R, ev, wl * mr, 1), y, mr, 1), pr});
  } else if (d->nsite == 1) {
    s.push_back(
        {to_f32(gp(ml * wl, d1 * mr, ml, 1, opnd(L, ev, ml, 1), opnd(psi, pv, 1, d1 * mr), T1, d1 * mr, 1), f), pr});
    s.push_back({to_f32(gp(d1 * wr, mr, wl * d1, ml, opnd(Wt1, mv, wl * d1, 1),
                           iopnd(T1, lay.dt_T1, f, 1, mr, wl * d1 * mr), T2, mr, 1, d1 * wr * mr),
                        f),
                 pr});
    s.push_back(
        {gp(ml * d1, mr, wr * mr, 1, iopnd(T2, lay.dt_T2, f, wr * mr, 1), opnd(R, ev, wr * mr, 1), y, mr, 1), pr});
  } else {
    const int64_t n12 = d1 * d2 * mr;
    void* T3 = T1;
    s.push_back({to_f32(gp(ml * wl, n12, ml, 1, opnd(L, ev, ml, 1), opnd(psi, pv, 1, n12), T1, n12, 1), f), pr});
    s.push_back({to_f32(gp(d1 * wm, d2 * mr, wl * d1, ml, opnd(Wt1, mv, wl * d1, 1),
                           iopnd(T1, lay.dt_T1, f, 1, d2 * mr, wl * d1 * d2 * mr), T2, d2 * mr, 1, d1 * wm * d2 * mr),
                        f),
                 pr});
    s.push_back({to_f32(gp(d2 * wr, mr, wm * d2, ml * d1, opnd(Wt2, mv, wm * d2, 1),
                           iopnd(T2, lay.dt_T2, f, 1, mr, wm * d2 * mr), T3, mr, 1, d2 * wr * mr),
                        f),
                 pr});
    s.push_back({gp(ml * d1 * d2, mr, wr * mr, 1, iopnd(T3, lay.dt_T2, f, wr * mr, 1), opnd(R, ev, wr * mr, 1), y, mr, 1),
                 pr});
  }
  return s;
}

// ---------------------------------------------------------------- fused split 2-site matvec
// The four stages of the 2-site matvec with every intermediate written by the
// producing GEMM's epilogue straight into the consumer's packed hi/lo operand
// (no FP64/FP32 intermediate, no separate pack pass):
//   S1  T1 = L . psi      N order (k, h, e): e runs along the consumer's K
//   S2  T2 = Wt1 . T1[a]  written as S3's B, N order (k, h): h along K
//   S3  T3 = Wt2 . T2[ad] written as S4's A ([re | im] along K = (w, k))
//   S4  y  = T3 . R^T     FP64 output
// Used for complex L, R, psi with a real MPO (TDVP) and for all-real
// operands (DMRG); other combinations take the staged path.
struct Fused2 {
  SplitPacked s1a, s1b, s2a, s2b, s3a, s3b, s4a, s4b;
  size_t bytes;
};

static bool fused2_eligible(const reno_heff_desc* d) {
  if (d->nsite != 2 || d->prec == RENO_PREC_FP64 || d->mpo_dtype != RENO_F64) return false;
  const bool allc = d->env_dtype == RENO_C128 && d->psi_dtype == RENO_C128;
  const bool allr = d->env_dtype == RENO_F64 && d->psi_dtype == RENO_F64;
  return allc || allr;
}

static Fused2 fused2_layout(const reno_heff_desc* d, char* base) {
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wm = d->wm, wr = d->wr, d1 = d->d1, d2 = d->d2;
  const bool c = d->env_dtype == RENO_C128;
  const int pr = d->prec;
  const int64_t x2 = c ? 2 : 1;
  // (rows, kext, nb, mode) of each packed operand
  struct Spec { int64_t rows, kext, nb; int mode; };
  const Spec s1a{x2 * ml * wl, x2 * ml, 1, c ? SPLIT_DBL_CPLX : SPLIT_REAL};
  const Spec s1b{d1 * d2 * mr, x2 * ml, 1, c ? SPLIT_CAT : SPLIT_REAL};
  const Spec s2a{d1 * wm, wl * d1, 1, SPLIT_REAL};
  const Spec s2b{x2 * d2 * mr, wl * d1, ml, c ? SPLIT_DBL_SPLIT : SPLIT_REAL};
  const Spec s3a{d2 * wr, wm * d2, 1, SPLIT_REAL};
  const Spec s3b{x2 * mr, wm * d2, ml * d1, c ? SPLIT_DBL_SPLIT : SPLIT_REAL};
  const Spec s4a{ml * d1 * d2, x2 * wr * mr, 1, c ? SPLIT_CAT : SPLIT_REAL};
  const Spec s4b{x2 * mr, x2 * wr * mr, 1, c ? SPLIT_DBL_CPLX : SPLIT_REAL};
  auto sz = [&](const Spec& q) { return split_packed_bytes(q.rows, q.kext, q.nb, pr); };
  auto at = [&](size_t off, const Spec& q) {
    return split_packed_at(base ? base + off : nullptr, q.rows, q.kext, q.nb, q.mode, pr);
  };
  Fused2 f{};
  size_t off = 0;
  f.s1a = at(off, s1a);
  off = align256(off + sz(s1a));
  f.s2a = at(off, s2a);
  off = align256(off + sz(s2a));
  f.s3a = at(off, s3a);
  off = align256(off + sz(s3a));
  f.s4b = at(off, s4b);
  off = align256(off + sz(s4b));
  // region P: psi packed (S1's B), later S3's B; region Q: S2's B, later S4's A
  const size_t P = off;
  off = align256(off + std::max(sz(s1b), sz(s3b)));
  const size_t Q = off;
  off = align256(off + std::max(sz(s2b), sz(s4a)));
  f.s1b = at(P, s1b);
  f.s3b = at(P, s3b);
  f.s2b = at(Q, s2b);
  f.s4a = at(Q, s4a);
  f.bytes = off;
  return f;
}

static cudaError_t fused2_run(const reno_heff_desc* d, const Fused2& f, const void* L, const void* Wt1,
                              const void* Wt2, const void* R, const void* psi, void* y, cudaStream_t st) {
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wm = d->wm, wr = d->wr, d1 = d->d1, d2 = d->d2;
  const int ev = d->env_dtype, pv = d->psi_dtype, pr = d->prec;
  const bool c = ev == RENO_C128;
  const int64_t x2 = c ? 2 : 1;
  cudaError_t e = split_pack(opnd(L, ev, ml, 1), (int)(ml * wl), (int)ml, 1, SplitRows{}, f.s1a, pr, st);
  // psi rows in (k, h, e) order: e at stride d2*mr, h at mr, k at 1; K = c at d1*d2*mr
  SplitRows khe;
  khe.D0 = (int)d1;
  khe.D1 = (int)d2;
  khe.s_r1 = mr;
  khe.s_r2 = 1;
  if (e == cudaSuccess)
    e = split_pack(opnd(psi, pv, d2 * mr, d1 * d2 * mr), (int)(d1 * d2 * mr), (int)ml, 1, khe, f.s1b, pr, st);
  if (e == cudaSuccess)
    e = split_pack(opnd(Wt1, RENO_F64, wl * d1, 1), (int)(d1 * wm), (int)(wl * d1), 1, SplitRows{}, f.s2a, pr, st);
  if (e == cudaSuccess)
    e = split_pack(opnd(Wt2, RENO_F64, wm * d2, 1), (int)(d2 * wr), (int)(wm * d2), 1, SplitRows{}, f.s3a, pr, st);
  if (e == cudaSuccess)
    e = split_pack(opnd(R, ev, wr * mr, 1), (int)mr, (int)(wr * mr), 1, SplitRows{}, f.s4b, pr, st);
  if (e != cudaSuccess) return e;
  // S1: rows (a, b) of L, columns (k, h, e) -> S2's B[a][(k, h) re/im][(b, e)]
  SplitPackOut o1{f.s2b.hi, f.s2b.lo, 0, f.s2b.rows * f.s2b.pitch, d1, x2 * f.s2b.pitch, 1, f.s2b.pitch,
                  (int)wl, (int)d1};
  e = split_run(f.s1a, f.s1b, (int)(ml * wl), (int)(d1 * d2 * mr), 1, nullptr, &o1, pr, st);
  // S2 (batch a): rows (d', w), columns (k, h) -> S3's B[(a, d')][k re/im][(w, h)]
  SplitPackOut o2{f.s3b.hi, f.s3b.lo, d1 * f.s3b.rows * f.s3b.pitch, f.s3b.rows * f.s3b.pitch, d2,
                  x2 * f.s3b.pitch, 1, f.s3b.pitch, (int)wm, (int)d2};
  if (e == cudaSuccess) e = split_run(f.s2a, f.s2b, (int)(d1 * wm), (int)(d2 * mr), (int)ml, nullptr, &o2, pr, st);
  // S3 (batch (a, d')): rows (h', w2), columns k -> S4's A[(a, d', h')][re/im | (w2, k)]
  SplitPackOut o3{f.s4a.hi, f.s4a.lo, d2 * f.s4a.pitch, f.s4a.pitch, mr, 0, 1, wr * mr, (int)wr, (int)mr};
  if (e == cudaSuccess) e = split_run(f.s3a, f.s3b, (int)(d2 * wr), (int)mr, (int)(ml * d1), nullptr, &o3, pr, st);
  // S4: y[(a, d', h'), l] = T3 . R^T
  GemmParams out;
  out.C = y;
  out.sCm = mr;
  out.sCn = 1;
  if (e == cudaSuccess) e = split_run(f.s4a, f.s4b, (int)(ml * d1 * d2), (int)mr, 1, &out, nullptr, pr, st);
  (void)x2;
  return e;
}

// ---------------------------------------------------------------- fused split 1-site matvec
// The 2-site chain without its middle stage:
//   S1  T1 = L . psi      N order (k, e): e runs along S2's K = (b, e)
//   S2  T2 = Wt . T1[a]   written as S3's A ([re | im] along K = (f, k))
//   S3  y  = T2 . R^T     FP64 output
struct Fused1 {
  SplitPacked s1a, s1b, s2a, s2b, s3a, s3b;
  size_t bytes;
};

static bool fused1_eligible(const reno_heff_desc* d) {
  if (d->nsite != 1 || d->prec == RENO_PREC_FP64 || d->mpo_dtype != RENO_F64) return false;
  const bool allc = d->env_dtype == RENO_C128 && d->psi_dtype == RENO_C128;
  const bool allr = d->env_dtype == RENO_F64 && d->psi_dtype == RENO_F64;
  return allc || allr;
}

static Fused1 fused1_layout(const reno_heff_desc* d, char* base) {
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wr = d->wr, dd = d->d1;
  const bool c = d->env_dtype == RENO_C128;
  const int pr = d->prec;
  const int64_t x2 = c ? 2 : 1;
  struct Spec { int64_t rows, kext, nb; int mode; };
  const Spec s1a{x2 * ml * wl, x2 * ml, 1, c ? SPLIT_DBL_CPLX : SPLIT_REAL};
  const Spec s1b{dd * mr, x2 * ml, 1, c ? SPLIT_CAT : SPLIT_REAL};
  const Spec s2a{dd * wr, wl * dd, 1, SPLIT_REAL};
  const Spec s2b{x2 * mr, wl * dd, ml, c ? SPLIT_DBL_SPLIT : SPLIT_REAL};
  const Spec s3a{ml * dd, x2 * wr * mr, 1, c ? SPLIT_CAT : SPLIT_REAL};
  const Spec s3b{x2 * mr, x2 * wr * mr, 1, c ? SPLIT_DBL_CPLX : SPLIT_REAL};
  auto sz = [&](const Spec& q) { return split_packed_bytes(q.rows, q.kext, q.nb, pr); };
  auto at = [&](size_t off, const Spec& q) {
    return split_packed_at(base ? base + off : nullptr, q.rows, q.kext, q.nb, q.mode, pr);
  };
  Fused1 f{};
  size_t off = 0;
  f.s1a = at(off, s1a);
  off = align256(off + sz(s1a));
  f.s2a = at(off, s2a);
  off = align256(off + sz(s2a));
  f.s3b = at(off, s3b);
  off = align256(off + sz(s3b));
  // region P: psi packed (S1's B), later S3's A; region Q: S2's B
  const size_t P = off;
  off = align256(off + std::max(sz(s1b), sz(s3a)));
  const size_t Q = off;
  off = align256(off + sz(s2b));
  f.s1b = at(P, s1b);
  f.s3a = at(P, s3a);
  f.s2b = at(Q, s2b);
  f.bytes = off;
  return f;
}

static cudaError_t fused1_run(const reno_heff_desc* d, const Fused1& f, const void* L, const void* Wt,
                              const void* R, const void* psi, void* y, cudaStream_t st) {
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wr = d->wr, dd = d->d1;
  const int ev = d->env_dtype, pv = d->psi_dtype, pr = d->prec;
  const int64_t x2 = ev == RENO_C128 ? 2 : 1;
  cudaError_t e = split_pack(opnd(L, ev, ml, 1), (int)(ml * wl), (int)ml, 1, SplitRows{}, f.s1a, pr, st);
  // psi rows in (k, e) order: e at stride mr, k at 1; K = c at dd*mr
  SplitRows ke;
  ke.D0 = (int)dd;
  ke.D1 = (int)mr;
  ke.s_r1 = 1;
  ke.s_r2 = 0;
  if (e == cudaSuccess) e = split_pack(opnd(psi, pv, mr, dd * mr), (int)(dd * mr), (int)ml, 1, ke, f.s1b, pr, st);
  if (e == cudaSuccess)
    e = split_pack(opnd(Wt, RENO_F64, wl * dd, 1), (int)(dd * wr), (int)(wl * dd), 1, SplitRows{}, f.s2a, pr, st);
  if (e == cudaSuccess)
    e = split_pack(opnd(R, ev, wr * mr, 1), (int)mr, (int)(wr * mr), 1, SplitRows{}, f.s3b, pr, st);
  if (e != cudaSuccess) return e;
  // S1: rows (a, b) of L, columns (k, e) -> S2's B[a][k re/im][(b, e)]
  SplitPackOut o1{f.s2b.hi, f.s2b.lo, 0, f.s2b.rows * f.s2b.pitch, dd, x2 * f.s2b.pitch, 1, f.s2b.pitch,
                  (int)wl, (int)dd};
  e = split_run(f.s1a, f.s1b, (int)(ml * wl), (int)(dd * mr), 1, nullptr, &o1, pr, st);
  // S2 (batch a): rows (d', f), columns k -> S3's A[(a, d')][re/im | (f, k)]
  SplitPackOut o2{f.s3a.hi, f.s3a.lo, dd * f.s3a.pitch, f.s3a.pitch, mr, 0, 1, wr * mr, (int)wr, (int)mr};
  if (e == cudaSuccess) e = split_run(f.s2a, f.s2b, (int)(dd * wr), (int)mr, (int)ml, nullptr, &o2, pr, st);
  // S3: y[(a, d'), l] = T2 . R^T
  GemmParams out;
  out.C = y;
  out.sCm = mr;
  out.sCn = 1;
  if (e == cudaSuccess) e = split_run(f.s3a, f.s3b, (int)(ml * dd), (int)mr, 1, &out, nullptr, pr, st);
  return e;
}

static size_t heff_total(const reno_heff_desc* d) {
  const HeffLayout lay = heff_layout(d);
  if (fused2_eligible(d)) return lay.off_t1 + fused2_layout(d, nullptr).bytes;
  if (fused1_eligible(d)) return lay.off_t1 + fused1_layout(d, nullptr).bytes;
  char* nul = nullptr;
  return lay.off_split + align256(split_need(heff_stages(d, lay, nul, nullptr, nullptr, nullptr, nullptr)));
}

}  // namespace reno

using namespace reno;

extern "C" int reno_heff_workspace_bytes(const reno_heff_desc* d, size_t* bytes) {
  if (validate_heff(d) != RENO_OK || !bytes) return RENO_ERR_INVALID;
  *bytes = heff_total(d);
  return RENO_OK;
}

extern "C" int reno_heff_apply(reno_ctx* ctx, const reno_heff_desc* d, const void* L, const void* W1,
                               const void* W2, const void* R, const void* psi, void* y, void* ws,
                               size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (validate_heff(d) != RENO_OK) return set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply: invalid descriptor");
  if (!L || !R || !psi || !y || (d->nsite >= 1 && !W1) || (d->nsite == 2 && !W2))
    return set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply: null tensor pointer");
  const HeffLayout lay = heff_layout(d);
  char* w = static_cast<char*>(ws);
  if (fused1_eligible(d)) {
    const Fused1 f = fused1_layout(d, w ? w + lay.off_t1 : nullptr);
    if (ws_bytes < lay.off_t1 + f.bytes || !ws)
      return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heff_apply: workspace too small");
    cudaStream_t st = ctx->stream;
    cudaError_t e = launch_wt(W1, w + lay.off_wt1, d->mpo_dtype, d->wl, d->d1, d->wr, 0, st);
    if (e == cudaSuccess) e = fused1_run(d, f, L, w + lay.off_wt1, R, psi, y, st);
    return check_cuda(ctx, e, "reno_heff_apply");
  }
  if (fused2_eligible(d)) {
    const Fused2 f = fused2_layout(d, w ? w + lay.off_t1 : nullptr);
    if (ws_bytes < lay.off_t1 + f.bytes || !ws)
      return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heff_apply: workspace too small");
    cudaStream_t st = ctx->stream;
    cudaError_t e = launch_wt(W1, w + lay.off_wt1, d->mpo_dtype, d->wl, d->d1, d->wm, 0, st);
    if (e == cudaSuccess) e = launch_wt(W2, w + lay.off_wt2, d->mpo_dtype, d->wm, d->d2, d->wr, 0, st);
    if (e == cudaSuccess) e = fused2_run(d, f, L, w + lay.off_wt1, w + lay.off_wt2, R, psi, y, st);
    return check_cuda(ctx, e, "reno_heff_apply");
  }
  const std::vector<Stage> stages = heff_stages(d, lay, w, L, R, psi, y);
  const size_t need_split = split_need(stages);
  if (ws_bytes < lay.off_split + need_split || !ws)
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heff_apply: workspace too small");
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (d->nsite == 1) e = launch_wt(W1, w + lay.off_wt1, d->mpo_dtype, d->wl, d->d1, d->wr, 0, st);
  if (d->nsite == 2) {
    e = launch_wt(W1, w + lay.off_wt1, d->mpo_dtype, d->wl, d->d1, d->wm, 0, st);
    if (e == cudaSuccess) e = launch_wt(W2, w + lay.off_wt2, d->mpo_dtype, d->wm, d->d2, d->wr, 0, st);
  }
  for (const Stage& s : stages) {
    if (e != cudaSuccess) break;
    e = run_stage(s, w + lay.off_split, need_split, st);
  }
  return check_cuda(ctx, e, "reno_heff_apply");
}

// ---------------------------------------------------------------- grouped FP64 matvec
// Many independent local problems (static-disorder realisations, each with
// its own bond dimensions) advanced together: one launch transposes every
// problem's MPO tensors, then each stage of the contraction chain is one
// grouped GEMM launch over all problems.  Every problem's arithmetic is that
// of its own reno_heff_apply at FP64 (same stages, same tiles).
namespace reno {
constexpr int MAX_WT = 2 * fp64gemm::MAX_GROUP;
struct WtGroup {
  int count = 0;
  const void* W[MAX_WT] = {};
  void* Wt[MAX_WT] = {};
  int nc[MAX_WT] = {}, d[MAX_WT] = {}, nr[MAX_WT] = {};
};

template <typename T>
__global__ void wt_grouped_kernel(const __grid_constant__ WtGroup g) {
  const int i = blockIdx.y;
  const T* __restrict__ W = static_cast<const T*>(g.W[i]);
  T* __restrict__ Wt = static_cast<T*>(g.Wt[i]);
  const int nc = g.nc[i], d = g.d[i], nr = g.nr[i];
  const int64_t total = (int64_t)d * nr * nc * d;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int e = idx % d;
    const int c = (idx / d) % nc;
    const int r = (idx / ((int64_t)d * nc)) % nr;
    const int dd = idx / ((int64_t)d * nc * nr);
    Wt[idx] = W[(((int64_t)c * d + dd) * d + e) * nr + r];
  }
}

static int validate_group(int32_t count, const reno_heff_desc* descs) {
  if (count < 1 || count > fp64gemm::MAX_GROUP || !descs) return RENO_ERR_INVALID;
  for (int i = 0; i < count; ++i) {
    const reno_heff_desc* d = descs + i;
    if (validate_heff(d) != RENO_OK || d->prec != RENO_PREC_FP64) return RENO_ERR_INVALID;
    if (d->nsite != descs[0].nsite || d->psi_dtype != descs[0].psi_dtype || d->env_dtype != descs[0].env_dtype ||
        d->mpo_dtype != descs[0].mpo_dtype)
      return RENO_ERR_INVALID;
  }
  return RENO_OK;
}
}  // namespace reno

extern "C" int reno_heff_grouped_workspace_bytes(int32_t count, const reno_heff_desc* descs, size_t* bytes) {
  if (!bytes || validate_group(count, descs) != RENO_OK) return RENO_ERR_INVALID;
  size_t total = 0;
  for (int i = 0; i < count; ++i) total += align256(heff_layout(descs + i).off_split);
  *bytes = total;
  return RENO_OK;
}

extern "C" int reno_heff_apply_grouped(reno_ctx* ctx, int32_t count, const reno_heff_desc* descs,
                                       const void* const* L, const void* const* W1, const void* const* W2,
                                       const void* const* R, const void* const* psi, void* const* y, void* ws,
                                       size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (validate_group(count, descs) != RENO_OK)
    return set_error(ctx, RENO_ERR_INVALID,
                     "reno_heff_apply_grouped: 1..128 valid FP64 descriptors with the same nsite and dtypes");
  if (!L || !R || !psi || !y || (descs[0].nsite >= 1 && !W1) || (descs[0].nsite == 2 && !W2))
    return set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply_grouped: null pointer array");
  size_t need = 0;
  reno_heff_grouped_workspace_bytes(count, descs, &need);
  if (!ws || ws_bytes < need) return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heff_apply_grouped: workspace too small");
  const int nsite = descs[0].nsite;
  cudaStream_t st = ctx->stream;
  std::vector<std::vector<Stage>> stages(count);
  std::unique_ptr<WtGroup> wg(new WtGroup());
  int64_t max_wt = 0;
  size_t off = 0;
  for (int i = 0; i < count; ++i) {
    const reno_heff_desc* d = descs + i;
    if (!L[i] || !R[i] || !psi[i] || !y[i] || (nsite >= 1 && !W1[i]) || (nsite == 2 && !W2[i]))
      return set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply_grouped: null tensor pointer");
    const HeffLayout lay = heff_layout(d);
    char* w = static_cast<char*>(ws) + off;
    off += align256(lay.off_split);
    if (nsite >= 1) {
      const int k = wg->count++;
      wg->W[k] = W1[i];
      wg->Wt[k] = w + lay.off_wt1;
      wg->nc[k] = d->wl;
      wg->d[k] = d->d1;
      wg->nr[k] = nsite == 2 ? d->wm : d->wr;
      max_wt = std::max(max_wt, (int64_t)d->d1 * d->d1 * d->wl * wg->nr[k]);
    }
    if (nsite == 2) {
      const int k = wg->count++;
      wg->W[k] = W2[i];
      wg->Wt[k] = w + lay.off_wt2;
      wg->nc[k] = d->wm;
      wg->d[k] = d->d2;
      wg->nr[k] = d->wr;
      max_wt = std::max(max_wt, (int64_t)d->d2 * d->d2 * d->wm * d->wr);
    }
    stages[i] = heff_stages(d, lay, w, L[i], R[i], psi[i], y[i]);
    if (stages[i].size() != stages[0].size())
      return set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply_grouped: mixed contraction chains");
  }
  if (wg->count > 0) {
    const dim3 grid((unsigned)std::min<int64_t>(ceil_div(max_wt, 256), 64), (unsigned)wg->count);
    count_launch();
    if (descs[0].mpo_dtype == RENO_C128)
      wt_grouped_kernel<double2><<<grid, 256, 0, st>>>(*wg);
    else
      wt_grouped_kernel<double><<<grid, 256, 0, st>>>(*wg);
    RENO_LAUNCH_CHECK(ctx, "reno_heff_apply_grouped: MPO transposes");
  }
  std::unique_ptr<fp64gemm::GemmGroup> g(new fp64gemm::GemmGroup());
  for (size_t s = 0; s < stages[0].size(); ++s) {
    g->count = count;
    for (int i = 0; i < count; ++i) g->p[i] = stages[i][s].p;
    const int rc = check_cuda(ctx, gemm_fp64_grouped(*g, st), "reno_heff_apply_grouped: stage");
    if (rc != RENO_OK) return rc;
  }
  return RENO_OK;
}

// ---------------------------------------------------------------- env update
namespace reno {
struct EnvLayout {
  int dt_T1, dt_T2, dt_out, t32;
  size_t off_ketT, off_braT, off_wt, off_t1, off_t2, off_split;
};

static int validate_env(const reno_env_desc* d) {
  if (!d) return RENO_ERR_INVALID;
  if (d->side != 0 && d->side != 1) return RENO_ERR_INVALID;
  if (d->d <= 0 || d->w_in <= 0 || d->w_out <= 0 || d->mk_in <= 0 || d->mk_out <= 0 || d->mb_in <= 0 ||
      d->mb_out <= 0)
    return RENO_ERR_INVALID;
  for (int t : {d->env_dtype, d->ket_dtype, d->bra_dtype, d->mpo_dtype})
    if (t != RENO_F64 && t != RENO_C128) return RENO_ERR_INVALID;
  if (d->prec < RENO_PREC_FP64 || d->prec > RENO_PREC_TF32X3) return RENO_ERR_INVALID;
  return RENO_OK;
}

static EnvLayout env_layout(const reno_env_desc* d) {
  EnvLayout p{};
  const int64_t dd = d->d, wi = d->w_in, wo = d->w_out, ki = d->mk_in, ko = d->mk_out, bi = d->mb_in,
                bo = d->mb_out;
  p.dt_T1 = promote(d->env_dtype, d->ket_dtype);
  p.dt_T2 = promote(p.dt_T1, d->mpo_dtype);
  p.dt_out = promote(p.dt_T2, d->bra_dtype);
  p.t32 = d->prec != RENO_PREC_FP64;
  const int64_t div = p.t32 ? 2 : 1;
  size_t off = 0;
  p.off_ketT = off;
  if (d->side == 1) off = align256(off + ki * dd * ko * esz(d->ket_dtype));
  p.off_braT = off;
  if (d->side == 1) off = align256(off + bi * dd * bo * esz(d->bra_dtype));
  p.off_wt = off;
  off = align256(off + dd * wo * wi * dd * esz(d->mpo_dtype));
  p.off_t1 = off;
  off = align256(off + bi * wi * dd * ko * esz(p.dt_T1) / div);
  p.off_t2 = off;
  off = align256(off + bi * dd * wo * ko * esz(p.dt_T2) / div);
  p.off_split = off;
  return p;
}

// lib.py:200-205 stage order on (possibly mirrored) bra/ket
static std::vector<Stage> env_stages(const reno_env_desc* d, const EnvLayout& lay, char* w, const void* E,
                                     const void* k_op, const void* b_op, int bra_dt, int conj_bra, void* out) {
  const int64_t dd = d->d, wi = d->w_in, wo = d->w_out, ki = d->mk_in, ko = d->mk_out, bi = d->mb_in,
                bo = d->mb_out;
  void* Wt = w + lay.off_wt;
  void* T1 = w + lay.off_t1;
  void* T2 = w + lay.off_t2;
  const int pr = d->prec, f = lay.t32;
  std::vector<Stage> s;
  s.push_back({to_f32(gp(bi * wi, dd * ko, ki, 1, opnd(E, d->env_dtype, ki, 1), opnd(k_op, d->ket_dtype, 1, dd * ko),
                         T1, dd * ko, 1),
                      f),
               pr});
  s.push_back({to_f32(gp(dd * wo, ko, wi * dd, bi, opnd(Wt, d->mpo_dtype, wi * dd, 1),
                         iopnd(T1, lay.dt_T1, f, 1, ko, wi * dd * ko), T2, ko, 1, dd * wo * ko),
                      f),
               pr});
  s.push_back({gp(bo, wo * ko, bi * dd, 1, opnd(b_op, bra_dt, 1, bo, 0, conj_bra), iopnd(T2, lay.dt_T2, f, 1, wo * ko),
                  out, wo * ko, 1),
               pr});
  return s;
}

static size_t env_total(const reno_env_desc* d) {
  const EnvLayout lay = env_layout(d);
  char* nul = nullptr;
  return lay.off_split +
         align256(split_need(env_stages(d, lay, nul, nullptr, nullptr, nullptr, d->bra_dtype, 0, nullptr)));
}
}  // namespace reno

extern "C" int reno_env_workspace_bytes(const reno_env_desc* d, size_t* bytes) {
  if (validate_env(d) != RENO_OK || !bytes) return RENO_ERR_INVALID;
  *bytes = env_total(d);
  return RENO_OK;
}

extern "C" int reno_env_update(reno_ctx* ctx, const reno_env_desc* d, const void* E, const void* W,
                               const void* ket, const void* bra, void* out, void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (validate_env(d) != RENO_OK) return set_error(ctx, RENO_ERR_INVALID, "reno_env_update: invalid descriptor");
  if (!E || !W || !ket || !out) return set_error(ctx, RENO_ERR_INVALID, "reno_env_update: null tensor pointer");
  if (!bra && (d->mb_in != d->mk_in || d->mb_out != d->mk_out))
    return set_error(ctx, RENO_ERR_INVALID, "reno_env_update: bra == NULL needs bra dims == ket dims");
  const EnvLayout lay = env_layout(d);
  char* w = static_cast<char*>(ws);
  cudaStream_t st = ctx->stream;
  const int64_t dd = d->d, wi = d->w_in, wo = d->w_out, ki = d->mk_in, ko = d->mk_out, bi = d->mb_in,
                bo = d->mb_out;
  const void* k_op = ket;
  const void* b_op = bra;
  const int bra_dt = bra ? d->bra_dtype : d->ket_dtype;
  if (d->side == 1) {
    k_op = w + lay.off_ketT;
    if (bra) b_op = w + lay.off_braT;
  }
  const int conj_bra = bra ? 0 : 1;
  if (!bra) b_op = k_op;
  const std::vector<Stage> stages = env_stages(d, lay, w, E, k_op, b_op, bra_dt, conj_bra, out);
  const size_t need_split = split_need(stages);
  if (ws_bytes < lay.off_split + need_split || !ws)
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_env_update: workspace too small");
  cudaError_t e = cudaSuccess;
  if (d->side == 1) {
    // mirror: ketT[c,e,h] = ket[h,e,c], braT[a,d,f] = bra[f,d,a]
    e = launch_swap13(ket, w + lay.off_ketT, d->ket_dtype, (int)ko, (int)dd, (int)ki, st);
    if (e == cudaSuccess && bra) e = launch_swap13(bra, w + lay.off_braT, d->bra_dtype, (int)bo, (int)dd, (int)bi, st);
  }
  if (e == cudaSuccess) e = launch_wt(W, w + lay.off_wt, d->mpo_dtype, (int)wi, (int)dd, (int)wo, d->side == 1 ? 1 : 0, st);
  for (const Stage& s : stages) {
    if (e != cudaSuccess) break;
    e = run_stage(s, w + lay.off_split, need_split, st);
  }
  return check_cuda(ctx, e, "reno_env_update");
}

// ---------------------------------------------------------------- hdiag
namespace reno {
__device__ __forceinline__ double real_of(double v) { return v; }
__device__ __forceinline__ double real_of(double2 v) { return v.x; }

// hdiag[a, c, (dd,) f] = Re sum L[a,b,a] W1[b,c,c,e] (W2[e,dd,dd,g]) R[f,g,f]
// Real part only: the reference forms it from real DMRG tensors (gs.py:419-445).
template <typename TE, typename TW>
__global__ void hdiag_kernel(const TE* L, const TW* W1, const TW* W2, const TE* R, double* out, int nsite, int ml,
                             int mr, int wl, int wm, int wr, int d1, int d2) {
  const int dd2 = nsite == 2 ? d2 : 1;
  const int64_t total = (int64_t)ml * d1 * dd2 * mr;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int f = idx % mr;
    const int dd = (idx / mr) % dd2;
    const int c = (idx / ((int64_t)mr * dd2)) % d1;
    const int a = idx / ((int64_t)mr * dd2 * d1);
    double acc = 0.0;
    if (nsite == 1) {
      for (int b = 0; b < wl; ++b) {
        const double lv = real_of(L[((int64_t)a * wl + b) * ml + a]);
        if (lv == 0.0) continue;
        for (int g = 0; g < wr; ++g) {
          const double wv = real_of(W1[(((int64_t)b * d1 + c) * d1 + c) * wr + g]);
          if (wv == 0.0) continue;
          acc += lv * wv * real_of(R[((int64_t)f * wr + g) * mr + f]);
        }
      }
    } else {
      for (int b = 0; b < wl; ++b) {
        const double lv = real_of(L[((int64_t)a * wl + b) * ml + a]);
        if (lv == 0.0) continue;
        for (int e = 0; e < wm; ++e) {
          const double w1 = real_of(W1[(((int64_t)b * d1 + c) * d1 + c) * wm + e]);
          if (w1 == 0.0) continue;
          for (int g = 0; g < wr; ++g) {
            const double w2 = real_of(W2[(((int64_t)e * d2 + dd) * d2 + dd) * wr + g]);
            if (w2 == 0.0) continue;
            acc += lv * w1 * w2 * real_of(R[((int64_t)f * wr + g) * mr + f]);
          }
        }
      }
    }
    out[idx] = acc;
  }
}
}  // namespace reno

extern "C" int reno_heff_diag(reno_ctx* ctx, const reno_heff_desc* d, const void* L, const void* W1, const void* W2,
                              const void* R, double* hdiag) {
  if (!ctx) return RENO_ERR_INVALID;
  if (validate_heff(d) != RENO_OK || d->nsite < 1)
    return set_error(ctx, RENO_ERR_INVALID, "reno_heff_diag: invalid descriptor");
  if (!L || !W1 || !R || !hdiag || (d->nsite == 2 && !W2))
    return set_error(ctx, RENO_ERR_INVALID, "reno_heff_diag: null pointer");
  const int64_t total = (int64_t)d->ml * d->d1 * (d->nsite == 2 ? d->d2 : 1) * d->mr;
  const int g = grid_for(total);
  const bool ec = d->env_dtype == RENO_C128, wc = d->mpo_dtype == RENO_C128;
  count_launch();
#define HD(TE, TW)                                                                                         \
  hdiag_kernel<TE, TW><<<g, 256, 0, ctx->stream>>>((const TE*)L, (const TW*)W1, (const TW*)W2, (const TE*)R, \
                                                    hdiag, d->nsite, d->ml, d->mr, d->wl, d->wm, d->wr, d->d1,   \
                                                    d->d2)
  if (ec && wc)
    HD(double2, double2);
  else if (ec)
    HD(double2, double);
  else if (wc)
    HD(double, double2);
  else
    HD(double, double);
#undef HD
  return check_cuda(ctx, cudaGetLastError(), "reno_heff_diag");
}

// ---------------------------------------------------------------- plain GEMM
static GemmParams plain_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t a_dtype, int64_t a_rs,
                             int64_t a_cs, int32_t a_conj, const void* B, int32_t b_dtype, int64_t b_rs, int64_t b_cs,
                             int32_t b_conj, void* C, int64_t c_rs) {
  return gp(M, N, K, 1, opnd(A, a_dtype, a_rs, a_cs, 0, a_conj), opnd(B, b_dtype, b_cs, b_rs, 0, b_conj), C, c_rs, 1);
}

extern "C" int reno_gemm_workspace_bytes(int32_t M, int32_t N, int32_t K, int32_t a_dtype, int32_t b_dtype,
                                         int32_t prec, size_t* bytes) {
  if (!bytes || M < 0 || N < 0 || K < 0 || prec < RENO_PREC_FP64 || prec > RENO_PREC_TF32X3) return RENO_ERR_INVALID;
  const char* dummy = reinterpret_cast<const char*>(256);
  GemmParams p = plain_gemm(M, N, K, dummy, a_dtype, K, 1, 0, dummy, b_dtype, N, 1, 0, (void*)dummy, N);
  *bytes = split_gemm_required_bytes(p, prec);
  return RENO_OK;
}

extern "C" int reno_gemm(reno_ctx* ctx, int32_t M, int32_t N, int32_t K, const void* A, int32_t a_dtype,
                         int64_t a_rs, int64_t a_cs, int32_t a_conj, const void* B, int32_t b_dtype, int64_t b_rs,
                         int64_t b_cs, int32_t b_conj, void* C, int64_t c_rs, int32_t prec, void* ws,
                         size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (M < 0 || N < 0 || K < 0 || !A || !B || !C || (a_dtype != RENO_F64 && a_dtype != RENO_C128) ||
      (b_dtype != RENO_F64 && b_dtype != RENO_C128) || c_rs < N || prec < RENO_PREC_FP64 || prec > RENO_PREC_TF32X3)
    return set_error(ctx, RENO_ERR_INVALID, "reno_gemm: bad arguments");
  GemmParams p = plain_gemm(M, N, K, A, a_dtype, a_rs, a_cs, a_conj, B, b_dtype, b_rs, b_cs, b_conj, C, c_rs);
  if (prec == RENO_PREC_FP64) return check_cuda(ctx, gemm_fp64(p, ctx->stream), "reno_gemm");
  if (ws_bytes < split_gemm_required_bytes(p, prec) || !ws)
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_gemm: workspace too small");
  return check_cuda(ctx, split_gemm(p, prec, ws, ws_bytes, ctx->stream), "reno_gemm");
}

extern "C" int reno_device_error(reno_ctx* ctx, int32_t* code) {
  if (!ctx || !code) return RENO_ERR_INVALID;
  *code = split_gemm_take_error();
  return RENO_OK;
}
