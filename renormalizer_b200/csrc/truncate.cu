// reno_qn_svd_truncate: the QN-blocked truncation of one two-site (or
// one-site) coefficient, svd_qn.py:99-240 + select_basis lib.py:253-322 +
// compute_m_trunc configs.py:196-219 as used by the sweeps (mp.py:693-778),
// behind one C call so that a host without Python can run the truncation.
//
// Per QN sector (block X, m x n): the Gram matrix of the smaller side, its
// leading eigenpairs on the device eigensolver (reno_heev_top_batched, all
// blocks in one reduction launch), the eigenvectors ordered by decreasing
// eigenvalue and orthonormalised by Householder QR (reno_qr_blocks), a
// residual check, the back-transformation, then the kept basis K and the
// complementary factor P: the singular values are the norms of the projected
// rows (columns) of P.  When the kept side is the larger one, K is the
// Householder QR of the projected vectors.  The singular values come to the
// host, which selects the kept triplets like the reference (all blocks'
// values in block order, a stable descending sort, the count from the
// truncation rule), and the selected columns are scattered into the outputs.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <vector>
#include "reno_common.cuh"
#include "gemm_fp64.cuh"

using namespace reno;

namespace {

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void real_to_c128_kernel(const double* __restrict__ x, double2* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = make_double2(x[i], 0.0);
}

__global__ void c128_real_kernel(const double2* __restrict__ x, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i].x;
}

__global__ void conj_kernel(const double2* __restrict__ x, double2* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = make_double2(x[i].x, -x[i].y);
}

// Zd[i, j] = Z[i, kt - 1 - j]: eigenvectors by decreasing eigenvalue
__global__ void flip_cols_kernel(const double* __restrict__ Z, double* __restrict__ Zd, int n, int kt) {
  const int64_t tot = (int64_t)n * kt;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / kt, c = i % kt;
    Zd[i] = Z[r * kt + (kt - 1 - c)];
  }
}

// out[0] = max_j ||T q_j - rho_j q_j||_inf / max |w| for the orthonormal
// columns q_j of Q (n x kt); one block, deterministic
__global__ void __launch_bounds__(256) residual_kernel(const double* __restrict__ d, const double* __restrict__ e,
                                                      const double* __restrict__ w, const double* __restrict__ Q,
                                                      int n, int kt, double* __restrict__ out) {
  __shared__ double red[256];
  double worst = 0.0, wmax = 0.0;
  for (int j = 0; j < kt; ++j) wmax = fmax(wmax, fabs(w[j]));
  for (int j = threadIdx.x; j < kt; j += blockDim.x) {
    double rho = 0.0;
    for (int i = 0; i < n; ++i) {
      double tq = d[i] * Q[(int64_t)i * kt + j];
      if (i > 0) tq += e[i - 1] * Q[(int64_t)(i - 1) * kt + j];
      if (i < n - 1) tq += e[i] * Q[(int64_t)(i + 1) * kt + j];
      rho += Q[(int64_t)i * kt + j] * tq;
    }
    for (int i = 0; i < n; ++i) {
      double tq = d[i] * Q[(int64_t)i * kt + j];
      if (i > 0) tq += e[i - 1] * Q[(int64_t)(i - 1) * kt + j];
      if (i < n - 1) tq += e[i] * Q[(int64_t)(i + 1) * kt + j];
      const double r = fabs(tq - rho * Q[(int64_t)i * kt + j]);
      worst = (r > worst || r != r) ? r : worst;
    }
  }
  red[threadIdx.x] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) m = (red[t] > m || red[t] != red[t]) ? red[t] : m;
    out[0] = m / fmax(wmax, 2.2250738585072014e-308);
  }
}

// 2-norms of the rows (by_row) or columns of a rows x cols matrix
template <bool C>
__global__ void norms_kernel(const void* __restrict__ X, int rows, int cols, int by_row, double* __restrict__ out) {
  const int count = by_row ? rows : cols, len = by_row ? cols : rows;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < count; v += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int t = 0; t < len; ++t) {
      const int64_t idx = by_row ? (int64_t)v * cols + t : (int64_t)t * cols + v;
      if constexpr (C) {
        const double2 x = reinterpret_cast<const double2*>(X)[idx];
        s += x.x * x.x + x.y * x.y;
      } else {
        const double x = reinterpret_cast<const double*>(X)[idx];
        s += x * x;
      }
    }
    out[v] = sqrt(s);
  }
}

unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096)); }

struct Block {
  std::vector<int32_t> nl, nr;
  std::vector<int64_t> lset, rset;
  int m = 0, n = 0, s = 0, kt = 0;
  bool left_gram = true;  // Gram of the row side (X X^H)
  bool need_qr = false;   // the kept side is the larger one
  // workspace offsets
  size_t o_l, o_r, o_x, o_g, o_gr, o_d, o_e, o_tau, o_w, o_z, o_zd, o_q, o_qr, o_k, o_e2, o_p, o_v, o_kq, o_kqr, o_s,
      o_sel;
};

struct Plan {
  std::vector<Block> blocks;
  size_t heev_off = 0, heev_bytes = 0, qr_off = 0, qr_bytes = 0, chk_off = 0, total = 0;
};

bool label_eq(const int32_t* a, const int32_t* b, int qs) {
  for (int i = 0; i < qs; ++i)
    if (a[i] != b[i]) return false;
  return true;
}

int make_plan(const reno_trunc_desc* D, Plan& P, std::string& why) {
  const int qs = D->qn_size;
  if (D->rows < 1 || D->cols < 1 || qs < 1 || !D->qn_rows || !D->qn_cols || !D->qntot ||
      (D->dtype != RENO_F64 && D->dtype != RENO_C128) || D->mode < 0 || D->mode > 2 ||
      (D->mode != RENO_TRUNC_THRESHOLD && D->m_max < 1) ||
      (D->mode != RENO_TRUNC_FIXED && !(D->threshold > 0.0 && D->threshold < 1.0)) || D->nsectors < 0 ||
      (D->nsectors > 0 && !D->sectors)) {
    why = "reno_qn_svd_truncate: invalid descriptor";
    return RENO_ERR_INVALID;
  }
  // sector order: the caller's list, or first appearance among the rows
  std::vector<std::vector<int32_t>> order;
  if (D->nsectors > 0) {
    for (int i = 0; i < D->nsectors; ++i) order.emplace_back(D->sectors + (size_t)i * qs, D->sectors + (size_t)(i + 1) * qs);
  } else {
    for (int r = 0; r < D->rows; ++r) {
      const int32_t* q = D->qn_rows + (size_t)r * qs;
      bool seen = false;
      for (auto& o : order) seen = seen || label_eq(o.data(), q, qs);
      if (!seen) order.emplace_back(q, q + qs);
    }
  }
  for (auto& nl : order) {
    Block b;
    b.nl = nl;
    b.nr.resize(qs);
    for (int i = 0; i < qs; ++i) b.nr[i] = D->qntot[i] - nl[i];
    for (int r = 0; r < D->rows; ++r)
      if (label_eq(D->qn_rows + (size_t)r * qs, nl.data(), qs)) b.lset.push_back(r);
    for (int c = 0; c < D->cols; ++c)
      if (label_eq(D->qn_cols + (size_t)c * qs, b.nr.data(), qs)) b.rset.push_back(c);
    if (b.lset.empty() || b.rset.empty()) continue;
    b.m = (int)b.lset.size();
    b.n = (int)b.rset.size();
    b.s = std::min(b.m, b.n);
    if (b.s > 4096) {
      why = "reno_qn_svd_truncate: a QN block's smaller side exceeds 4096";
      return RENO_ERR_UNSUPPORTED;
    }
    // a fixed cap needs at most m_max triplets of any block; a threshold reads
    // the norm of every singular value
    b.kt = D->mode == RENO_TRUNC_FIXED ? std::min(b.s, (int)D->m_max) : b.s;
    b.left_gram = b.m < b.n || (b.m == b.n && D->keep_left);
    b.need_qr = (bool)D->keep_left != b.left_gram;
    P.blocks.push_back(std::move(b));
  }
  if (P.blocks.empty()) {
    why = "reno_qn_svd_truncate: Invalid quantum number (no block)";
    return RENO_ERR_INVALID;
  }
  if ((int)P.blocks.size() > RENO_HEEV_MAX_BATCH) {
    why = "reno_qn_svd_truncate: more than " + std::to_string(RENO_HEEV_MAX_BATCH) + " QN blocks";
    return RENO_ERR_UNSUPPORTED;
  }
  const size_t es = D->dtype == RENO_C128 ? 16 : 8;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = al256(o + std::max<size_t>(bytes, 1));
    return at;
  };
  std::vector<reno_heev_problem> hp;
  std::vector<reno_qr_block> q1, q2;
  for (auto& b : P.blocks) {
    const size_t s = b.s, kt = b.kt, m = b.m, n = b.n;
    b.o_l = take(m * 8);
    b.o_r = take(n * 8);
    b.o_x = take(m * n * es);
    b.o_g = take(s * s * 16);   // complex Gram (the reduction overwrites it)
    b.o_gr = take(D->dtype == RENO_C128 ? 1 : s * s * 8);
    b.o_d = take(s * 8);
    b.o_e = take(s * 8);
    b.o_tau = take(s * 16);
    b.o_w = take(kt * 8);
    b.o_z = take(s * kt * 8);
    b.o_zd = take(s * kt * 8);
    b.o_q = take(s * kt * 8);
    b.o_qr = take(kt * kt * 8);
    b.o_k = take(s * kt * 16);
    b.o_e2 = take(s * kt * es);   // eigenvectors in the block's dtype
    const size_t big = b.left_gram ? n : m;  // the larger side's length
    b.o_v = take(big * kt * es);            // projected vectors (need_qr)
    b.o_kq = take(big * kt * es);           // their QR (the kept basis)
    b.o_kqr = take(kt * kt * es);
    b.o_p = take(std::max(m, n) * kt * es); // complementary factor
    b.o_s = take(kt * 8);
    b.o_sel = take(3 * std::max<size_t>(kt, std::max(m, n)) * 8);
    hp.push_back(reno_heev_problem{(int32_t)s, (int32_t)kt, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                   nullptr});
    q1.push_back(reno_qr_block{(int32_t)s, (int32_t)kt, RENO_F64, 0, nullptr, nullptr, nullptr});
    q2.push_back(reno_qr_block{(int32_t)big, (int32_t)kt, D->dtype, 0, nullptr, nullptr, nullptr});
  }
  P.chk_off = take(P.blocks.size() * 8 * 4);
  if (reno_heev_batched_workspace_bytes((int32_t)hp.size(), hp.data(), &P.heev_bytes) != RENO_OK) {
    why = "reno_qn_svd_truncate: eigensolver workspace";
    return RENO_ERR_INVALID;
  }
  P.heev_off = take(P.heev_bytes);
  size_t b1 = 0, b2 = 0;
  if (reno_qr_workspace_bytes((int32_t)q1.size(), q1.data(), &b1) != RENO_OK ||
      reno_qr_workspace_bytes((int32_t)q2.size(), q2.data(), &b2) != RENO_OK) {
    why = "reno_qn_svd_truncate: QR workspace";
    return RENO_ERR_UNSUPPORTED;
  }
  P.qr_bytes = std::max(b1, b2);
  P.qr_off = take(P.qr_bytes);
  P.total = o;
  return RENO_OK;
}

GemmOperand gop(const void* p, int64_t s_outer, int64_t s_k, bool cplx, bool conj = false) {
  GemmOperand g;
  g.ptr = p;
  g.s_outer = s_outer;
  g.s_k = s_k;
  g.is_complex = cplx;
  g.conj = conj;
  return g;
}

// C (M x N, row-major) = opA(A) opB(B) with element strides
int gemm(reno_ctx* ctx, int M, int N, int K, GemmOperand A, GemmOperand B, void* C, const char* what) {
  GemmParams p;
  p.M = M;
  p.N = N;
  p.K = K;
  p.A = A;
  p.B = B;
  p.C = C;
  p.sCm = N;
  p.sCn = 1;
  count_launch();
  return check_cuda(ctx, gemm_fp64(p, ctx->stream), what);
}

}  // namespace

extern "C" int reno_qn_svd_truncate_workspace_bytes(const reno_trunc_desc* desc, size_t* bytes) {
  if (!desc || !bytes) return RENO_ERR_INVALID;
  Plan P;
  std::string why;
  const int rc = make_plan(desc, P, why);
  if (rc != RENO_OK) return rc;
  *bytes = P.total;
  return RENO_OK;
}

extern "C" int reno_qn_svd_truncate(reno_ctx* ctx, const reno_trunc_desc* D, const void* coef, void* left,
                                    void* right, int32_t ldm, double* sigma, int32_t* qn_out, int32_t* out_m,
                                    void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!D || !coef || !left || !right || !sigma || !qn_out || !out_m || !ws || ldm < 1)
    return set_error(ctx, RENO_ERR_INVALID, "reno_qn_svd_truncate: null argument");
  Plan P;
  std::string why;
  int rc = make_plan(D, P, why);
  if (rc != RENO_OK) return set_error(ctx, rc, why);
  if (ws_bytes < P.total) return set_error(ctx, RENO_ERR_WORKSPACE, "reno_qn_svd_truncate: workspace too small");
  cudaStream_t st = ctx->stream;
  char* base = static_cast<char*>(ws);
  const bool cplx = D->dtype == RENO_C128;
  const int32_t dt = D->dtype;
  const int qs = D->qn_size;
  const int nb = (int)P.blocks.size();
#define TR_TRY(call)              \
  do {                            \
    rc = (call);                  \
    if (rc != RENO_OK) return rc; \
  } while (0)
  auto at = [&](size_t off) { return static_cast<void*>(base + off); };
  // ---- gather, Gram
  for (auto& b : P.blocks) {
    TR_TRY(check_cuda(ctx, cudaMemcpyAsync(at(b.o_l), b.lset.data(), b.lset.size() * 8, cudaMemcpyHostToDevice, st),
                      "reno_qn_svd_truncate: rows"));
    TR_TRY(check_cuda(ctx, cudaMemcpyAsync(at(b.o_r), b.rset.data(), b.rset.size() * 8, cudaMemcpyHostToDevice, st),
                      "reno_qn_svd_truncate: cols"));
    TR_TRY(reno_qn_gather(ctx, dt, coef, D->cols, (const int64_t*)at(b.o_l), b.m, (const int64_t*)at(b.o_r), b.n,
                          at(b.o_x)));
    const int64_t ss = (int64_t)b.s * b.s;
    void* g = cplx ? at(b.o_g) : at(b.o_gr);  // a real Gram is widened to complex afterwards
    if (b.left_gram)  // X X^H (s = m)
      TR_TRY(gemm(ctx, b.s, b.s, b.n, gop(at(b.o_x), b.n, 1, cplx), gop(at(b.o_x), b.n, 1, cplx, true), g,
                  "reno_qn_svd_truncate: Gram"));
    else              // X^H X (s = n)
      TR_TRY(gemm(ctx, b.s, b.s, b.m, gop(at(b.o_x), 1, b.n, cplx, true), gop(at(b.o_x), 1, b.n, cplx), g,
                  "reno_qn_svd_truncate: Gram"));
    if (!cplx) {
      count_launch();
      real_to_c128_kernel<<<grid_for(ss), 256, 0, st>>>((const double*)at(b.o_gr), (double2*)at(b.o_g), ss);
      RENO_LAUNCH_CHECK(ctx, "reno_qn_svd_truncate: Gram to complex");
    }
  }
  // ---- eigenpairs of every Gram block (one batched reduction)
  std::vector<reno_heev_problem> hp;
  for (auto& b : P.blocks)
    hp.push_back(reno_heev_problem{b.s, b.kt, at(b.o_g), (double*)at(b.o_d), (double*)at(b.o_e), at(b.o_tau),
                                   (double*)at(b.o_w), (double*)at(b.o_z), at(b.o_k)});
  int32_t* status = (int32_t*)at(P.chk_off);
  double* chk = (double*)at(P.chk_off) + 2 * nb;
  TR_TRY(reno_heev_top_batched(ctx, nb, hp.data(), status, at(P.heev_off), P.heev_bytes));
  std::vector<reno_qr_block> qb;
  for (auto& b : P.blocks) {
    count_launch();
    flip_cols_kernel<<<grid_for((int64_t)b.s * b.kt), 256, 0, st>>>((const double*)at(b.o_z), (double*)at(b.o_zd),
                                                                     b.s, b.kt);
    RENO_LAUNCH_CHECK(ctx, "reno_qn_svd_truncate: order");
    qb.push_back(reno_qr_block{b.s, b.kt, RENO_F64, 0, at(b.o_zd), at(b.o_q), at(b.o_qr)});
  }
  TR_TRY(reno_qr_blocks(ctx, nb, qb.data(), at(P.qr_off), P.qr_bytes));
  for (int i = 0; i < nb; ++i) {
    auto& b = P.blocks[i];
    count_launch(2);
    residual_kernel<<<1, 256, 0, st>>>((const double*)at(b.o_d), (const double*)at(b.o_e), (const double*)at(b.o_w),
                                       (const double*)at(b.o_q), b.s, b.kt, chk + i);
    real_to_c128_kernel<<<grid_for((int64_t)b.s * b.kt), 256, 0, st>>>((const double*)at(b.o_q),
                                                                        (double2*)at(b.o_k), (int64_t)b.s * b.kt);
    RENO_LAUNCH_CHECK(ctx, "reno_qn_svd_truncate: residual");
  }
  TR_TRY(reno_heev_backtransform_batched(ctx, nb, hp.data(), at(P.heev_off), P.heev_bytes));
  // ---- kept basis, complementary factor, singular values
  std::vector<reno_qr_block> q2;
  for (auto& b : P.blocks) {
    void* E = at(b.o_k);
    if (!cplx) {
      count_launch();
      c128_real_kernel<<<grid_for((int64_t)b.s * b.kt), 256, 0, st>>>((const double2*)at(b.o_k), (double*)at(b.o_e2),
                                                                       (int64_t)b.s * b.kt);
      RENO_LAUNCH_CHECK(ctx, "reno_qn_svd_truncate: real eigenvectors");
      E = at(b.o_e2);
    }
    const int m = b.m, n = b.n, kt = b.kt;
    if (!b.need_qr) {
      if (D->keep_left) {  // K = E (m x kt), P = K^H X (kt x n), S = row norms
        TR_TRY(gemm(ctx, kt, n, m, gop(E, 1, kt, cplx, true), gop(at(b.o_x), 1, n, cplx), at(b.o_p),
                    "reno_qn_svd_truncate: projection"));
      } else {             // K = E (n x kt), P = X K (m x kt), S = column norms
        TR_TRY(gemm(ctx, m, kt, n, gop(at(b.o_x), n, 1, cplx), gop(E, 1, kt, cplx), at(b.o_p),
                    "reno_qn_svd_truncate: projection"));
      }
      b.o_kq = (size_t)((char*)E - base);
    } else {
      if (D->keep_left)    // Us = X E (m x kt)
        TR_TRY(gemm(ctx, m, kt, n, gop(at(b.o_x), n, 1, cplx), gop(E, 1, kt, cplx), at(b.o_v),
                    "reno_qn_svd_truncate: U sigma"));
      else                 // Vs = X^H E (n x kt)
        TR_TRY(gemm(ctx, n, kt, m, gop(at(b.o_x), 1, n, cplx, true), gop(E, 1, kt, cplx), at(b.o_v),
                    "reno_qn_svd_truncate: sigma V"));
      q2.push_back(reno_qr_block{D->keep_left ? m : n, kt, dt, 0, at(b.o_v), at(b.o_kq), at(b.o_kqr)});
    }
    // singular values: norms of P's rows (keep left) / columns, or of the projected vectors' columns
    count_launch();
    const void* src = b.need_qr ? at(b.o_v) : at(b.o_p);
    const int rows = b.need_qr ? (D->keep_left ? m : n) : (D->keep_left ? kt : m);
    const int by_row = (!b.need_qr && D->keep_left) ? 1 : 0;
    if (cplx) norms_kernel<true><<<grid_for(kt), 256, 0, st>>>(src, rows, by_row ? n : kt, by_row, (double*)at(b.o_s));
    else norms_kernel<false><<<grid_for(kt), 256, 0, st>>>(src, rows, by_row ? n : kt, by_row, (double*)at(b.o_s));
    RENO_LAUNCH_CHECK(ctx, "reno_qn_svd_truncate: sigma");
  }
  if (!q2.empty()) {
    TR_TRY(reno_qr_blocks(ctx, (int32_t)q2.size(), q2.data(), at(P.qr_off), P.qr_bytes));
    for (auto& b : P.blocks) {
      if (!b.need_qr) continue;
      const int m = b.m, n = b.n, kt = b.kt;
      if (D->keep_left)    // P = K^H X (kt x n)
        TR_TRY(gemm(ctx, kt, n, m, gop(at(b.o_kq), 1, kt, cplx, true), gop(at(b.o_x), 1, n, cplx), at(b.o_p),
                    "reno_qn_svd_truncate: projection"));
      else                 // P = X K (m x kt)
        TR_TRY(gemm(ctx, m, kt, n, gop(at(b.o_x), n, 1, cplx), gop(at(b.o_kq), 1, kt, cplx), at(b.o_p),
                    "reno_qn_svd_truncate: projection"));
    }
  }
  // ---- singular values and checks to the host
  std::vector<std::vector<double>> S(nb);
  std::vector<int32_t> hstatus(nb);
  std::vector<double> hchk(nb);
  for (int i = 0; i < nb; ++i) {
    S[i].resize(P.blocks[i].kt);
    TR_TRY(check_cuda(ctx, cudaMemcpyAsync(S[i].data(), at(P.blocks[i].o_s), S[i].size() * 8, cudaMemcpyDeviceToHost,
                                           st), "reno_qn_svd_truncate: sigma"));
  }
  TR_TRY(check_cuda(ctx, cudaMemcpyAsync(hstatus.data(), status, nb * 4, cudaMemcpyDeviceToHost, st),
                    "reno_qn_svd_truncate: status"));
  TR_TRY(check_cuda(ctx, cudaMemcpyAsync(hchk.data(), chk, nb * 8, cudaMemcpyDeviceToHost, st),
                    "reno_qn_svd_truncate: check"));
  TR_TRY(check_cuda(ctx, cudaStreamSynchronize(st), "reno_qn_svd_truncate: sync"));
  for (int i = 0; i < nb; ++i)
    if (hstatus[i] != 0 || !(hchk[i] <= 1e-12))
      return set_error(ctx, RENO_ERR_UNSUPPORTED,
                       "reno_qn_svd_truncate: the device eigensolver's check failed on QN block " + std::to_string(i) +
                           " (status " + std::to_string(hstatus[i]) + ", residual " + std::to_string(hchk[i]) + ")");
  // ---- selection: block order, stable descending sort, the truncation rule
  std::vector<double> sig;
  std::vector<int> blk, pos;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < P.blocks[i].kt; ++j) {
      sig.push_back(S[i][j]);
      blk.push_back(i);
      pos.push_back(j);
    }
  std::vector<int> idx(sig.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return sig[a] > sig[b]; });
  int64_t m_keep = (int64_t)sig.size();
  if (D->mode != RENO_TRUNC_THRESHOLD) m_keep = std::min<int64_t>(m_keep, D->m_max);
  if (D->mode != RENO_TRUNC_FIXED) {
    // sigma / ||sigma|| > threshold, ||sigma|| over every computed value
    double nrm = 0.0;
    for (double x : sig) nrm += x * x;
    nrm = std::sqrt(nrm);
    int64_t cnt = 0;
    for (double x : sig) cnt += (x / nrm > D->threshold) ? 1 : 0;
    m_keep = std::min(m_keep, cnt);
  }
  if (m_keep > ldm)
    return set_error(ctx, RENO_ERR_INVALID, "reno_qn_svd_truncate: " + std::to_string(m_keep) +
                                                " kept columns exceed ldm = " + std::to_string(ldm));
  *out_m = (int32_t)m_keep;
  const size_t es = cplx ? 16 : 8;
  TR_TRY(check_cuda(ctx, cudaMemsetAsync(left, 0, (size_t)D->rows * ldm * es, st), "reno_qn_svd_truncate: memset"));
  TR_TRY(check_cuda(ctx, cudaMemsetAsync(right, 0, (size_t)ldm * D->cols * es, st), "reno_qn_svd_truncate: memset"));
  std::vector<std::vector<int64_t>> scol(nb), dcol(nb);
  for (int64_t o = 0; o < m_keep; ++o) {
    const int e = idx[o];
    sigma[o] = sig[e];
    scol[blk[e]].push_back(pos[e]);
    dcol[blk[e]].push_back(o);
    const Block& b = P.blocks[blk[e]];
    for (int q = 0; q < qs; ++q) qn_out[o * qs + q] = D->keep_left ? b.nl[q] : b.nr[q];
  }
  for (int i = 0; i < nb; ++i) {
    Block& b = P.blocks[i];
    const int64_t nc = (int64_t)scol[i].size();
    if (nc == 0) continue;
    int64_t* dsc = (int64_t*)at(b.o_sel);
    int64_t* ddc = dsc + nc;
    TR_TRY(check_cuda(ctx, cudaMemcpyAsync(dsc, scol[i].data(), nc * 8, cudaMemcpyHostToDevice, st),
                      "reno_qn_svd_truncate: selection"));
    TR_TRY(check_cuda(ctx, cudaMemcpyAsync(ddc, dcol[i].data(), nc * 8, cudaMemcpyHostToDevice, st),
                      "reno_qn_svd_truncate: selection"));
    const int kt = b.kt;
    const void* K = at(b.o_kq);
    const int64_t* L = (const int64_t*)at(b.o_l);
    const int64_t* R = (const int64_t*)at(b.o_r);
    if (D->keep_left) {
      // left[lset[i], o] = K[i, j]; right[o, rset[i]] = P[j, i]
      TR_TRY(reno_qn_scatter(ctx, dt, K, kt, 1, L, b.m, dsc, ddc, nc, nullptr, left, ldm, 1));
      TR_TRY(reno_qn_scatter(ctx, dt, at(b.o_p), 1, b.n, R, b.n, dsc, ddc, nc, nullptr, right, 1, D->cols));
    } else {
      // right[o, rset[i]] = conj(K[i, j]); left[lset[i], o] = P[i, j]
      const void* Kc = K;
      if (cplx) {
        count_launch();
        conj_kernel<<<grid_for((int64_t)b.n * kt), 256, 0, st>>>((const double2*)K, (double2*)at(b.o_v),
                                                                 (int64_t)b.n * kt);
        RENO_LAUNCH_CHECK(ctx, "reno_qn_svd_truncate: conj");
        Kc = at(b.o_v);
      }
      TR_TRY(reno_qn_scatter(ctx, dt, Kc, kt, 1, R, b.n, dsc, ddc, nc, nullptr, right, 1, D->cols));
      TR_TRY(reno_qn_scatter(ctx, dt, at(b.o_p), kt, 1, L, b.m, dsc, ddc, nc, nullptr, left, ldm, 1));
    }
  }
#undef TR_TRY
  return RENO_OK;
}
