// Householder QR of a batch of independent matrices (the QN blocks of one
// site tensor), with LAPACK's conventions so that Q and R agree with
// scipy.linalg.qr(mode="economic") -- zgeqrf / dgeqrf + zungqr / dorgqr --
// including the signs: reflector j is H_j = I - tau_j v_j v_j^H with
// v_j[j] = 1, beta_j = -sign(Re alpha_j) |(alpha_j, x_j)| on the diagonal of R
// (zlarfg / dlarfg), and Q = H_0 H_1 ... H_{kq-1} [I; 0].
//
// Blocked right-looking algorithm, panels of nb columns:
//   qr_panel_kernel  one 8-CTA thread-block cluster per matrix factorises the
//                    panel: the panel's rows are split over the cluster's
//                    shared memories, the column norms and the w = v^H A
//                    products are reduced through distributed shared memory
//                    (every CTA sums the 8 partials in the same order, so the
//                    Householder scalars agree bit for bit), two cluster
//                    barriers per column.  It writes R's rows and the
//                    reflectors back, the explicit unit-lower V of the panel
//                    and the panel's triangular factor T (H_p0 ... H_p0+nb-1
//                    = I - V T V^H, LAPACK's forward columnwise zlarft).
//   trailing update  A[p0:, p0+nb:] -= V (T^H (V^H A[p0:, p0+nb:])): three
//                    grouped FP64 GEMMs over every matrix of the batch.
//   Q                Q = [I; 0], then for the panels from last to first
//                    Q[p0:, p0:] += V ((-T) (V^H Q[p0:, p0:])).
//
// Matrices are row-major (leading dimension = columns).  The input is
// overwritten.  Workspace comes from the caller (reno_qr_workspace_bytes).
#include <algorithm>
#include <cooperative_groups.h>
#include "reno_common.cuh"
#include "gemm_fp64.cuh"

namespace cg = cooperative_groups;

namespace reno {
namespace qr {

constexpr int QCL = 8;               // CTAs per cluster
constexpr int QT = 256;              // threads per CTA
constexpr int QW = QT / 32;
constexpr int NBMAX = 32;            // largest panel width
constexpr int PANEL_ELEMS = 10240;   // panel entries per CTA (160 KB of complex128)
constexpr int MAXB = RENO_QR_MAX_BLOCKS;

struct Prob {
  void* a;       // m x k, row-major, overwritten
  void* q;       // m x kq
  void* r;       // kq x k
  void* v;       // m x kq explicit unit-lower reflectors
  void* t;       // npan x nb x nb: T of each panel
  void* nt;      // npan x nb x nb: -T
  void* nth;     // npan x nb x nb: -T^H
  void* w1;      // nb x max(k, kq)
  void* w2;      // nb x max(k, kq)
  int m, k, kq;
};

struct Table {
  int count;
  Prob p[MAXB];
};

template <bool C>
struct Elem;
template <>
struct Elem<true> {
  using T = double2;
  static __device__ __forceinline__ T zero() { return make_double2(0.0, 0.0); }
  static __device__ __forceinline__ T one() { return make_double2(1.0, 0.0); }
  static __device__ __forceinline__ T add(T a, T b) { return make_double2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ T sub(T a, T b) { return make_double2(a.x - b.x, a.y - b.y); }
  static __device__ __forceinline__ T mul(T a, T b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  static __device__ __forceinline__ T conj(T a) { return make_double2(a.x, -a.y); }
  static __device__ __forceinline__ T neg(T a) { return make_double2(-a.x, -a.y); }
  static __device__ __forceinline__ double abs2(T a) { return a.x * a.x + a.y * a.y; }
  static __device__ __forceinline__ T shfl_xor(T v, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
  }
};
template <>
struct Elem<false> {
  using T = double;
  static __device__ __forceinline__ T zero() { return 0.0; }
  static __device__ __forceinline__ T one() { return 1.0; }
  static __device__ __forceinline__ T add(T a, T b) { return a + b; }
  static __device__ __forceinline__ T sub(T a, T b) { return a - b; }
  static __device__ __forceinline__ T mul(T a, T b) { return a * b; }
  static __device__ __forceinline__ T conj(T a) { return a; }
  static __device__ __forceinline__ T neg(T a) { return -a; }
  static __device__ __forceinline__ double abs2(T a) { return a * a; }
  static __device__ __forceinline__ T shfl_xor(T v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
};

template <bool C>
__device__ __forceinline__ typename Elem<C>::T warp_sum(typename Elem<C>::T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = Elem<C>::add(v, Elem<C>::shfl_xor(v, o));
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// zlarfg / dlarfg on (alpha, ||x||^2): beta, tau and the scale 1 / (alpha - beta)
// of x; tau = 0 (H = I) when x = 0 and alpha is real.
template <bool C>
__device__ __forceinline__ void householder(typename Elem<C>::T alpha, double xnorm2, double& beta,
                                            typename Elem<C>::T& tau, typename Elem<C>::T& scale) {
  if constexpr (C) {
    if (xnorm2 == 0.0 && alpha.y == 0.0) {
      beta = alpha.x;
      tau = make_double2(0.0, 0.0);
      scale = make_double2(0.0, 0.0);
      return;
    }
    beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
    tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
    const double2 den = make_double2(alpha.x - beta, alpha.y);
    const double d2 = den.x * den.x + den.y * den.y;
    scale = make_double2(den.x / d2, -den.y / d2);
  } else {
    if (xnorm2 == 0.0) {
      beta = alpha;
      tau = 0.0;
      scale = 0.0;
      return;
    }
    beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
    tau = (beta - alpha) / beta;
    scale = 1.0 / (alpha - beta);
  }
}

// Panel p0 .. p0+nbp-1 of matrix blockIdx.y (nbp = min(nb, kq - p0)).  The
// rows p0 .. m-1 are split in QCL contiguous chunks, one per CTA, held in
// shared memory as panel[(r - r0) * nb + jj].
template <bool C>
__global__ void __cluster_dims__(QCL, 1, 1) __launch_bounds__(QT, 1)
    qr_panel_kernel(const __grid_constant__ Table tab, int p0, int nb) {
  using E = Elem<C>;
  using T = typename E::T;
  cg::cluster_group cluster = cg::this_cluster();
  const Prob& P = tab.p[blockIdx.y];
  if (p0 >= P.kq) return;  // every CTA of this cluster returns here together
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nbp = min(nb, P.kq - p0);
  const int mr = P.m - p0;
  const int chunk = (mr + QCL - 1) / QCL;
  const int r0 = min(mr, rank * chunk), r1 = min(mr, r0 + chunk);
  const int nr = r1 - r0;
  T* A = reinterpret_cast<T*>(P.a);
  const int lda = P.k;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* panel = reinterpret_cast<T*>(smem_raw);               // nr x nb
  T* wpart = panel + (size_t)chunk * nb;                   // 2 x NBMAX: this CTA's partial v^H A
  T* wfull = wpart + 2 * NBMAX;                            // NBMAX: the summed w
  T* gram = wfull + NBMAX;                                 // NBMAX x NBMAX partial V^H V
  T* stau = gram + NBMAX * NBMAX;                          // NBMAX
  T* tsm = stau + NBMAX;                                   // NBMAX x NBMAX: T of the panel (CTA 0)
  T* xs = tsm + NBMAX * NBMAX;                             // NBMAX: one column's -tau_i (V^H V)[:, i]
  __shared__ double npart[2];                              // this CTA's partial ||x||^2 by column parity
  __shared__ T apart[2];                                   // alpha, written by its owner
  __shared__ double redd[QW];
  __shared__ T redt[QW];

  for (int idx = tid; idx < nr * nbp; idx += QT) {
    const int rl = idx / nbp, jj = idx % nbp;
    panel[(size_t)rl * nb + jj] = A[(size_t)(p0 + r0 + rl) * lda + p0 + jj];
  }
  __syncthreads();

  for (int jj = 0; jj < nbp; ++jj) {
    const int par = jj & 1;
    // ---- partial ||x||^2 over own rows below the pivot; the owner publishes alpha
    double s = 0.0;
    for (int rl = tid; rl < nr; rl += QT)
      if (r0 + rl > jj) s += E::abs2(panel[(size_t)rl * nb + jj]);
    s = warp_sum_d(s);
    if (lane == 0) redd[warp] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < QW; ++w) t += redd[w];
      npart[par] = t;
      if (jj >= r0 && jj < r1) apart[par] = panel[(size_t)(jj - r0) * nb + jj];
    }
    cluster.sync();
    double xn2 = 0.0;
    for (int c = 0; c < QCL; ++c) xn2 += cluster.map_shared_rank(npart, c)[par];
    const int owner = jj / chunk;
    const T alpha = cluster.map_shared_rank(apart, owner)[par];
    double beta;
    T tau, scale;
    householder<C>(alpha, xn2, beta, tau, scale);
    // ---- v below the pivot, beta on the diagonal
    for (int rl = tid; rl < nr; rl += QT) {
      const int r = r0 + rl;
      if (r > jj) panel[(size_t)rl * nb + jj] = E::mul(panel[(size_t)rl * nb + jj], scale);
      else if (r == jj) {
        if constexpr (C) panel[(size_t)rl * nb + jj] = make_double2(beta, 0.0);
        else panel[(size_t)rl * nb + jj] = beta;
      }
    }
    if (tid == 0) stau[jj] = tau;
    __syncthreads();
    if (jj + 1 < nbp) {
      // ---- w_c = sum_r conj(v_r) A[r, c] over own rows r >= jj, columns c > jj
      for (int c = jj + 1 + warp; c < nbp; c += QW) {
        T acc = E::zero();
        for (int rl = lane; rl < nr; rl += 32) {
          const int r = r0 + rl;
          if (r < jj) continue;
          const T v = (r == jj) ? E::one() : panel[(size_t)rl * nb + jj];
          acc = E::add(acc, E::mul(E::conj(v), panel[(size_t)rl * nb + c]));
        }
        acc = warp_sum<C>(acc);
        if (lane == 0) wpart[par * NBMAX + c] = acc;
      }
      cluster.sync();
      for (int c = jj + 1 + tid; c < nbp; c += QT) {
        T acc = E::zero();
        for (int q = 0; q < QCL; ++q) acc = E::add(acc, cluster.map_shared_rank(wpart, q)[par * NBMAX + c]);
        wfull[c] = acc;
      }
      __syncthreads();
      // ---- A[r, c] -= conj(tau) v_r w_c  (H^H applied from the left)
      const T ct = E::conj(tau);
      const int ncol = nbp - jj - 1;
      for (int idx = tid; idx < nr * ncol; idx += QT) {
        const int rl = idx / ncol, c = jj + 1 + idx % ncol;
        const int r = r0 + rl;
        if (r < jj) continue;
        const T v = (r == jj) ? E::one() : panel[(size_t)rl * nb + jj];
        panel[(size_t)rl * nb + c] = E::sub(panel[(size_t)rl * nb + c], E::mul(ct, E::mul(v, wfull[c])));
      }
      __syncthreads();
    }
  }

  // ---- V^H V over own rows, summed over the cluster by CTA 0
  for (int e = warp; e < nbp * nbp; e += QW) {
    const int i = e / nbp, j = e % nbp;
    T acc = E::zero();
    if (i < j) {
      for (int rl = lane; rl < nr; rl += 32) {
        const int r = r0 + rl;
        if (r < j) continue;
        const T vi = (r == i) ? E::one() : (r > i ? panel[(size_t)rl * nb + i] : E::zero());
        const T vj = (r == j) ? E::one() : panel[(size_t)rl * nb + j];
        acc = E::add(acc, E::mul(E::conj(vi), vj));
      }
      acc = warp_sum<C>(acc);
    }
    if (lane == 0) gram[i * NBMAX + j] = acc;
  }
  // ---- write back R rows / reflectors and the explicit V of this panel
  T* V = reinterpret_cast<T*>(P.v);
  for (int idx = tid; idx < nr * nbp; idx += QT) {
    const int rl = idx / nbp, jj = idx % nbp;
    const int r = r0 + rl;
    const T x = panel[(size_t)rl * nb + jj];
    A[(size_t)(p0 + r) * lda + p0 + jj] = x;
    V[(size_t)(p0 + r) * P.kq + p0 + jj] = (r == jj) ? E::one() : (r > jj ? x : E::zero());
  }
  cluster.sync();
  if (rank == 0) {
    // the cluster's V^H V: every entry summed over the CTAs (in rank order)
    // by one thread of CTA 0, in place in CTA 0's partial
    for (int e = tid; e < nbp * nbp; e += QT) {
      const int i = e / nbp, j = e % nbp;
      T g = E::zero();
      for (int q = 0; q < QCL; ++q) g = E::add(g, cluster.map_shared_rank(gram, q)[i * NBMAX + j]);
      gram[i * NBMAX + j] = g;
    }
    for (int e = tid; e < NBMAX * NBMAX; e += QT) tsm[e] = E::zero();
    __syncthreads();
    // zlarft (forward, columnwise): T[0:i, i] = -tau_i T[0:i, 0:i] (V^H V)[0:i, i];
    // lane l owns row l of T (nb <= 32), columns in order
    if (warp == 0) {
      for (int i = 0; i < nbp; ++i) {
        const T ti = stau[i];
        if (lane < i) xs[lane] = E::mul(E::neg(ti), gram[lane * NBMAX + i]);
        __syncwarp();
        if (lane < i) {
          T acc = E::zero();
          for (int c = lane; c < i; ++c) acc = E::add(acc, E::mul(tsm[lane * NBMAX + c], xs[c]));
          tsm[lane * NBMAX + i] = acc;
        } else if (lane == i) {
          tsm[i * NBMAX + i] = ti;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    const int pi = p0 / nb;
    T* Tm = reinterpret_cast<T*>(P.t) + (size_t)pi * nb * nb;
    T* NT = reinterpret_cast<T*>(P.nt) + (size_t)pi * nb * nb;
    T* NTH = reinterpret_cast<T*>(P.nth) + (size_t)pi * nb * nb;
    for (int e = tid; e < nb * nb; e += QT) {
      const int i = e / nb, j = e % nb;
      const T t = tsm[i * NBMAX + j];
      Tm[e] = t;
      NT[e] = E::neg(t);
      NTH[e] = E::neg(E::conj(tsm[j * NBMAX + i]));
    }
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// Q = [I; 0] (m x kq) for every matrix of the table
template <bool C>
__global__ void qr_init_q_kernel(const __grid_constant__ Table tab) {
  using E = Elem<C>;
  const Prob& P = tab.p[blockIdx.y];
  typename E::T* Q = reinterpret_cast<typename E::T*>(P.q);
  const size_t n = (size_t)P.m * P.kq;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / P.kq, c = i % P.kq;
    Q[i] = (r == c) ? E::one() : E::zero();
  }
}

// R = the upper trapezoid of the first kq rows of the factored A
template <bool C>
__global__ void qr_extract_r_kernel(const __grid_constant__ Table tab) {
  using E = Elem<C>;
  const Prob& P = tab.p[blockIdx.y];
  const typename E::T* A = reinterpret_cast<const typename E::T*>(P.a);
  typename E::T* R = reinterpret_cast<typename E::T*>(P.r);
  const size_t n = (size_t)P.kq * P.k;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / P.k, c = i % P.k;
    R[i] = (c >= r) ? A[i] : E::zero();
  }
}

}  // namespace qr
}  // namespace reno

using namespace reno;

namespace {

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// panel width: the largest power of two <= 32 whose panel rows fit a CTA
int panel_width(int mmax) {
  const int rows = (mmax + qr::QCL - 1) / qr::QCL;
  int nb = qr::NBMAX;
  while (nb > 1 && (size_t)rows * nb > (size_t)qr::PANEL_ELEMS) nb >>= 1;
  return (size_t)rows * nb <= (size_t)qr::PANEL_ELEMS ? nb : 0;
}

struct Layout {
  size_t off[RENO_QR_MAX_BLOCKS][7];
  size_t split = 0, split_bytes = 0;  // split-K partials of the V^H products
  size_t total = 0;
  int nb = 0;
};

int plan(int32_t count, const reno_qr_block* b, Layout& L, std::string& why) {
  if (count < 1 || count > RENO_QR_MAX_BLOCKS) {
    why = "reno_qr_blocks: count must be 1.." + std::to_string(RENO_QR_MAX_BLOCKS);
    return RENO_ERR_INVALID;
  }
  int mmax = 1;
  for (int i = 0; i < count; ++i) {
    if (b[i].m < 0 || b[i].k < 0 || (b[i].dtype != RENO_F64 && b[i].dtype != RENO_C128) ||
        b[i].dtype != b[0].dtype) {
      why = "reno_qr_blocks: invalid block " + std::to_string(i) + " (negative size or mixed/unknown dtype)";
      return RENO_ERR_INVALID;
    }
    mmax = std::max(mmax, (int)b[i].m);
  }
  L.nb = panel_width(mmax);
  if (L.nb == 0) {
    why = "reno_qr_blocks: " + std::to_string(mmax) + " rows exceed the panel capacity";
    return RENO_ERR_UNSUPPORTED;
  }
  const size_t es = b[0].dtype == RENO_C128 ? 16 : 8;
  size_t o = 0;
  for (int i = 0; i < count; ++i) {
    const size_t m = b[i].m, k = b[i].k, kq = std::min(m, k);
    const size_t npan = (kq + L.nb - 1) / L.nb;
    const size_t wcols = std::max<size_t>(std::max(k, kq), 1);
    const size_t sz[7] = {m * kq, npan * L.nb * L.nb, npan * L.nb * L.nb, npan * L.nb * L.nb,
                          (size_t)L.nb * wcols, (size_t)L.nb * wcols, 0};
    for (int s = 0; s < 6; ++s) {
      L.off[i][s] = o;
      o = al256(o + std::max<size_t>(sz[s], 1) * es);
    }
  }
  size_t wmax = 1;
  for (int i = 0; i < count; ++i)
    wmax = std::max<size_t>(wmax, std::max<size_t>(std::max(b[i].k, std::min(b[i].m, b[i].k)), 1));
  L.split = o;
  L.split_bytes = fp64gemm::splitk_bytes_bound(count, (int64_t)L.nb * (int64_t)wmax, es == 16);
  o = al256(o + L.split_bytes);
  L.total = o;
  return RENO_OK;
}

GemmOperand op(const void* p, int64_t s_outer, int64_t s_k, bool cplx, bool conj = false) {
  GemmOperand g;
  g.ptr = p;
  g.s_outer = s_outer;
  g.s_k = s_k;
  g.is_complex = cplx;
  g.conj = conj;
  return g;
}

}  // namespace

extern "C" int reno_qr_workspace_bytes(int32_t count, const reno_qr_block* blocks, size_t* bytes) {
  if (!blocks || !bytes) return RENO_ERR_INVALID;
  Layout L;
  std::string why;
  const int rc = plan(count, blocks, L, why);
  if (rc != RENO_OK) return rc;
  *bytes = L.total;
  return RENO_OK;
}

extern "C" int reno_qr_blocks(reno_ctx* ctx, int32_t count, const reno_qr_block* blocks, void* workspace,
                              size_t ws_bytes) {
  if (!ctx || !blocks) return RENO_ERR_INVALID;
  Layout L;
  std::string why;
  int rc = plan(count, blocks, L, why);
  if (rc != RENO_OK) return set_error(ctx, rc, why);
  if (ws_bytes < L.total)
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_qr_blocks: workspace of " + std::to_string(ws_bytes) +
                                                  " bytes, needs " + std::to_string(L.total));
  const bool cplx = blocks[0].dtype == RENO_C128;
  const size_t es = cplx ? 16 : 8;
  const int nb = L.nb;
  cudaStream_t st = ctx->stream;
  char* ws = reinterpret_cast<char*>(workspace);
  qr::Table tab{};
  tab.count = count;
  int kqmax = 0, nmax = 0;
  for (int i = 0; i < count; ++i) {
    const reno_qr_block& b = blocks[i];
    qr::Prob& P = tab.p[i];
    P.a = b.a;
    P.q = b.q;
    P.r = b.r;
    P.m = b.m;
    P.k = b.k;
    P.kq = std::min(b.m, b.k);
    P.v = ws + L.off[i][0];
    P.t = ws + L.off[i][1];
    P.nt = ws + L.off[i][2];
    P.nth = ws + L.off[i][3];
    P.w1 = ws + L.off[i][4];
    P.w2 = ws + L.off[i][5];
    if ((P.m > 0 && P.k > 0) && (!P.a || !P.q || !P.r))
      return set_error(ctx, RENO_ERR_INVALID, "reno_qr_blocks: null matrix pointer in block " + std::to_string(i));
    kqmax = std::max(kqmax, P.kq);
    nmax = std::max(nmax, P.m);
  }
  const int rows = (nmax + qr::QCL - 1) / qr::QCL;
  const size_t smem =
      ((size_t)rows * nb + 2 * qr::NBMAX + qr::NBMAX + 2 * qr::NBMAX * qr::NBMAX + 2 * qr::NBMAX) * es;
  // the opt-in is made once per device, so it covers the largest panel any call can use
  const int smem_max = (int)(((size_t)qr::PANEL_ELEMS + 5 * qr::NBMAX + 2 * qr::NBMAX * qr::NBMAX) * 16);
  static std::atomic<unsigned long long> set_c{0}, set_r{0};
  cudaError_t e = cplx ? smem_optin_once(qr::qr_panel_kernel<true>, smem_max, set_c)
                       : smem_optin_once(qr::qr_panel_kernel<false>, smem_max, set_r);
  if (e != cudaSuccess) return check_cuda(ctx, e, "reno_qr_blocks: shared-memory opt-in");

  // ---- factorisation, panel by panel
  for (int p0 = 0; p0 < kqmax; p0 += nb) {
    count_launch();
    if (cplx) qr::qr_panel_kernel<true><<<dim3(qr::QCL, count), qr::QT, smem, st>>>(tab, p0, nb);
    else qr::qr_panel_kernel<false><<<dim3(qr::QCL, count), qr::QT, smem, st>>>(tab, p0, nb);
    RENO_LAUNCH_CHECK(ctx, "reno_qr_blocks: panel");
    fp64gemm::GemmGroup g1, g2, g3;
    for (int i = 0; i < count; ++i) {
      const qr::Prob& P = tab.p[i];
      if (p0 >= P.kq) continue;
      const int nbp = std::min(nb, P.kq - p0);
      const int nc = P.k - p0 - nbp;
      if (nc <= 0) continue;
      const int mr = P.m - p0;
      const int pi = p0 / nb;
      const char* Vp = reinterpret_cast<const char*>(P.v) + ((size_t)p0 * P.kq + p0) * es;
      const char* Cp = reinterpret_cast<const char*>(P.a) + ((size_t)p0 * P.k + p0 + nbp) * es;
      const char* NTHp = reinterpret_cast<const char*>(P.nth) + (size_t)pi * nb * nb * es;
      GemmParams a;  // W1 = V^H C : (nbp x mr) (mr x nc)
      a.M = nbp; a.N = nc; a.K = mr;
      a.A = op(Vp, 1, P.kq, cplx, true);
      a.B = op(Cp, 1, P.k, cplx);
      a.C = P.w1; a.sCm = nc; a.sCn = 1;
      GemmParams b2;  // W2 = (-T^H) W1
      b2.M = nbp; b2.N = nc; b2.K = nbp;
      b2.A = op(NTHp, nb, 1, cplx);
      b2.B = op(P.w1, 1, nc, cplx);
      b2.C = P.w2; b2.sCm = nc; b2.sCn = 1;
      GemmParams c3;  // C += V W2
      c3.M = mr; c3.N = nc; c3.K = nbp;
      c3.A = op(Vp, P.kq, 1, cplx);
      c3.B = op(P.w2, 1, nc, cplx);
      c3.C = const_cast<char*>(Cp); c3.sCm = P.k; c3.sCn = 1; c3.accumulate = 1;
      g1.p[g1.count++] = a;
      g2.p[g2.count++] = b2;
      g3.p[g3.count++] = c3;
    }
    if (g1.count) {
      rc = check_cuda(ctx, gemm_fp64_grouped_splitk(g1, ws + L.split, L.split_bytes, st), "reno_qr_blocks: V^H C");
      if (rc == RENO_OK) rc = check_cuda(ctx, gemm_fp64_grouped(g2, st), "reno_qr_blocks: T^H W");
      if (rc == RENO_OK) rc = check_cuda(ctx, gemm_fp64_grouped(g3, st), "reno_qr_blocks: C += V W");
      if (rc != RENO_OK) return rc;
    }
  }
  // ---- R, then Q from the reflectors (last panel first)
  const int fill_blocks = 4 * sm_count_current_device() / std::max(count, 1) + 1;
  count_launch(2);
  if (cplx) {
    qr::qr_extract_r_kernel<true><<<dim3(fill_blocks, count), 256, 0, st>>>(tab);
    qr::qr_init_q_kernel<true><<<dim3(fill_blocks, count), 256, 0, st>>>(tab);
  } else {
    qr::qr_extract_r_kernel<false><<<dim3(fill_blocks, count), 256, 0, st>>>(tab);
    qr::qr_init_q_kernel<false><<<dim3(fill_blocks, count), 256, 0, st>>>(tab);
  }
  RENO_LAUNCH_CHECK(ctx, "reno_qr_blocks: R / Q init");
  const int npan_max = (kqmax + nb - 1) / nb;
  for (int pi = npan_max - 1; pi >= 0; --pi) {
    const int p0 = pi * nb;
    fp64gemm::GemmGroup g1, g2, g3;
    for (int i = 0; i < count; ++i) {
      const qr::Prob& P = tab.p[i];
      if (p0 >= P.kq) continue;
      const int nbp = std::min(nb, P.kq - p0);
      const int mr = P.m - p0, nc = P.kq - p0;
      const char* Vp = reinterpret_cast<const char*>(P.v) + ((size_t)p0 * P.kq + p0) * es;
      const char* Qp = reinterpret_cast<const char*>(P.q) + ((size_t)p0 * P.kq + p0) * es;
      const char* NTp = reinterpret_cast<const char*>(P.nt) + (size_t)pi * nb * nb * es;
      GemmParams a;  // W1 = V^H Qsub
      a.M = nbp; a.N = nc; a.K = mr;
      a.A = op(Vp, 1, P.kq, cplx, true);
      a.B = op(Qp, 1, P.kq, cplx);
      a.C = P.w1; a.sCm = nc; a.sCn = 1;
      GemmParams b2;  // W2 = (-T) W1
      b2.M = nbp; b2.N = nc; b2.K = nbp;
      b2.A = op(NTp, nb, 1, cplx);
      b2.B = op(P.w1, 1, nc, cplx);
      b2.C = P.w2; b2.sCm = nc; b2.sCn = 1;
      GemmParams c3;  // Qsub += V W2
      c3.M = mr; c3.N = nc; c3.K = nbp;
      c3.A = op(Vp, P.kq, 1, cplx);
      c3.B = op(P.w2, 1, nc, cplx);
      c3.C = const_cast<char*>(Qp); c3.sCm = P.kq; c3.sCn = 1; c3.accumulate = 1;
      g1.p[g1.count++] = a;
      g2.p[g2.count++] = b2;
      g3.p[g3.count++] = c3;
    }
    if (!g1.count) continue;
    rc = check_cuda(ctx, gemm_fp64_grouped_splitk(g1, ws + L.split, L.split_bytes, st), "reno_qr_blocks: V^H Q");
    if (rc == RENO_OK) rc = check_cuda(ctx, gemm_fp64_grouped(g2, st), "reno_qr_blocks: T W");
    if (rc == RENO_OK) rc = check_cuda(ctx, gemm_fp64_grouped(g3, st), "reno_qr_blocks: Q += V W");
    if (rc != RENO_OK) return rc;
  }
  return RENO_OK;
}
