// Hermitian eigensolver for the truncation's Gram blocks: the leading kt
// eigenpairs of an n x n Hermitian matrix G (the QN-block Gram matrices of
// svd_qn.py:12-49 / mp.py:693-778, which the reference factorises with
// LAPACK gesdd), entirely on the device.
//
//   1. hetrd_kernel   Householder reduction G = Q T Q^H to a real symmetric
//                     tridiagonal T (d, e), one persistent cooperative launch.
//                     Step k forms reflector k from row k of the trailing
//                     matrix, then every CTA streams its rows of the trailing
//                     matrix once: it applies the rank-2 update of step k-1
//                     (lagged by one step) and accumulates y = A v_k in the
//                     same pass.  The only inter-CTA dependency per column is
//                     the sum of y^H v_k, so there is one grid barrier per
//                     column; each CTA recomputes v_k and w_k itself from
//                     row k and y (bitwise identical in every CTA: same data,
//                     same reduction order).  Reflector k is stored in row k.
//   2. bisect_kernel  eigenvalues of T by Sturm-count multisection, one warp
//                     per eigenvalue, 32 points per round.
//   3. inviter_kernel eigenvectors of T by inverse iteration, one thread per
//                     eigenvalue: LU of T - lambda I with partial pivoting,
//                     three solves from a hashed start vector.  The host
//                     orthonormalises the block (CholeskyQR2) and checks the
//                     residuals ||T z - lambda z||.
//   4. back-transformation K = Q Z in blocks of 64 reflectors (compact WY
//                     form, three FP64 GEMMs per block, last block first).
//
// Every grid-barrier wait is bounded (2 s of wall clock by default, see
// reno_set_wait_limit_ns): on timeout the
// CTA raises the abort flag and a status word in the caller's workspace and
// returns; the others return at their next barrier.
#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <vector>
#include <cstddef>
#include "reno_common.cuh"
#include "gemm_fp64.cuh"
#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace reno {
namespace heev {

constexpr int THREADS = 256, WARPS = THREADS / 32;
constexpr int MAX_N = 4096;

struct Sync {
  unsigned count, gen;
  int abort, status;
};

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 conjg(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block sum in a fixed order (shuffle tree, then warps 0..NW-1); every
// thread gets the result
template <int NW>
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NW; ++w) s += red[w];
  return s;
}

// grid barrier over the nblocks CTAs that share `s`: a monotonic arrival
// counter (no reset between columns), released by each CTA's thread 0 after
// a CTA barrier and acquired by polling, the ordering pattern of CUTLASS's
// generic barrier.  false when this or another CTA gave up (abort raised).
// skip_arrival (test hook only): this CTA does not arrive, so every wait of
// this barrier runs out after wait_ns.
__device__ bool grid_sync(Sync* s, unsigned nblocks, unsigned& epoch, int* ok_sh, uint64_t wait_ns,
                          bool skip_arrival) {
  __syncthreads();
  if (threadIdx.x == 0) {
    epoch += 1u;
    const unsigned target = epoch * nblocks;
    bool good = true;
    if (!skip_arrival) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&s->count) : "memory");
    volatile int* va = &s->abort;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0;; ++it) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&s->count) : "memory");
      if (v >= target) break;
      if ((it & 63u) == 63u) {
        if (*va) {
          good = false;
          break;
        }
        if (global_ns() - t0 > wait_ns) {
          atomicExch(&s->abort, 1);
          atomicCAS(&s->status, 0, 1);
          good = false;
          break;
        }
      }
    }
    *ok_sh = good && !*va;
  }
  __syncthreads();
  return *ok_sh != 0;
}

constexpr int HT = 512, HW = HT / 32;  // reduction kernel: 16 warps, one CTA per SM
constexpr int U1 = 4;                  // loads in flight per thread (rows k, y)
constexpr int U2 = 6;                  // loads in flight per lane per item (trailing rows)
constexpr int MAXM = 32;               // matrices per batched launch

// One matrix of a batched reduction: CTAs first .. first + nblk - 1 of the
// cooperative grid work on it, with their own barrier word and buffers.
struct HetrdProb {
  double2* A;
  int n;
  double* d;
  double* e;
  double2* tau;
  double2* Y;
  double2* P;
  Sync* sync;
  int first, nblk;
  double2* YP;  // lower-triangle reduction: YP_G x n partial sums of y (nullptr: not available)
};
// One matrix of the batched small-matrix reduction and of the batched
// eigenvalue / eigenvector stages (blockIdx.y = entry).
struct EigProb {
  double2* a;
  double2* tau;
  double* d;
  double* e;
  int n, kt;
  double* w;
  double* z;
  double* bnd;
  double* scr;
};
struct EigTable {
  int count;
  EigProb p[MAXM];
};

struct HetrdTable {
  int count;
  int skip_column;      // test hook: CTA 0 of matrix 0 skips its arrival after this column (-1: none)
  uint64_t wait_ns;     // limit of every grid-barrier wait
  HetrdProb p[MAXM];
};

// A: n x n row-major Hermitian (both triangles), overwritten: row k holds
// reflector k from column k+1 on.  Y: 2n, P: 2 * nblk scratch.  Every
// matrix of the table is reduced by its own share of the grid.
//
// Per column k (lagged: update k-1 is applied while column k is processed):
//   phase 1 (every CTA)  row k with update k-1 applied, reflector k;
//   phase 2              the trailing rows r > k are dealt round-robin to the
//                        matrix's CTAs (r = k + 1 + bid + j G); each CTA splits
//                        its rows into chunks of HCH columns and spreads the
//                        (row, chunk) items over its warps, two items in
//                        flight per warp: update k-1 applied and stored, the
//                        chunk's share of y_r = (A v_k)_r kept in shared
//                        memory and summed per row in chunk order;
//   grid barrier;
//   phase 3 (every CTA)  w_k from y and the CTA partials of y^H v_k, issued
//                        together with the loads of row k+1 for the next
//                        phase 1 (one round trip to L2 for both).
constexpr int HCH = 32 * U2;    // columns per phase-2 item
constexpr int PARTS = 1024;     // per-CTA (row, chunk) partial sums held at once

// one phase-2 item: update k-1 on U2 x 32 entries of a row (a: their loaded
// values), stored back; returns the lane's share of the row's y
__device__ __forceinline__ double2 hetrd_item(double2* __restrict__ row, int cbase, int n, double2 vpr, double2 wpr,
                                              const double2* vp, const double2* wp, const double2* vc,
                                              const double2 (&a)[U2]) {
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int u = 0; u < U2; ++u) {
    const int c = cbase + 32 * u;
    if (c < n) {
      const double2 x = csub(csub(a[u], cmulc(vpr, wp[c])), cmulc(wpr, vp[c]));
      __stcg(&row[c], x);
      acc = cadd(acc, cmul(x, vc[c]));
    }
  }
  return acc;
}

__global__ void __launch_bounds__(HT, 1) hetrd_kernel(const __grid_constant__ HetrdTable tab) {
  int pi = 0;
  while (pi + 1 < tab.count && (int)blockIdx.x >= tab.p[pi + 1].first) ++pi;
  const HetrdProb& PR = tab.p[pi];
  double2* __restrict__ A = PR.A;
  const int n = PR.n;
  double* __restrict__ d = PR.d;
  double* __restrict__ e = PR.e;
  double2* __restrict__ tau = PR.tau;
  double2* __restrict__ Y = PR.Y;
  double2* __restrict__ P = PR.P;
  Sync* sync = PR.sync;
  const int bid = (int)blockIdx.x - PR.first;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* vp = reinterpret_cast<double2*>(smem_raw);  // v of step k-1 (pending update)
  double2* wp = vp + n;                                // w of step k-1
  double2* vc = wp + n;                                // v of step k
  double2* parts = vc + n;                             // PARTS (row, chunk) partial sums of y
  __shared__ double red[HW];
  __shared__ double2 redc[HW];
  __shared__ double s_akk;
  __shared__ int s_ok;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = PR.nblk;
  unsigned gen = 0;
  for (int i = tid; i < n; i += HT) {
    vp[i] = make_double2(0.0, 0.0);
    wp[i] = make_double2(0.0, 0.0);
    vc[i] = make_double2(0.0, 0.0);
  }
  // row 0, the part phase 1 reads in its first pass (c = tid + u HT)
  double2 pre[U1];
#pragma unroll
  for (int u = 0; u < U1; ++u) {
    const int c = tid + u * HT;
    pre[u] = c < n ? __ldcg(&A[c]) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  // Shared-memory discipline: in phases 1 and 3 thread t owns the entries
  // c = k + t + j HT of vc (phase 1 of column k) and c = k + 1 + t + j HT of
  // vp, wp (phase 3 of column k), i.e. the same entries as phase 1 of column
  // k + 1, so those phases need no block barrier between them; every thread
  // recomputes the scalars that more than one thread needs (the Householder
  // scalars, the dot y^H v and the pending pivot entries v_{k-1}[k] = 1,
  // w_{k-1}[k]) with the same operations, so they agree bit for bit.
  double2 tk_prev = make_double2(0.0, 0.0), alph_prev = make_double2(0.0, 0.0), yk_prev = make_double2(0.0, 0.0);
  for (int k = 0; k < n - 1; ++k) {
    // ---- phase 1 (every CTA): row k with update k-1 applied, reflector k
    double2 vpk = make_double2(0.0, 0.0), wpk = make_double2(0.0, 0.0);
    if (k > 0) {
      vpk = make_double2(1.0, 0.0);
      wpk = cadd(cmul(tk_prev, yk_prev), cmul(alph_prev, vpk));
    }
    const double2* rowk = A + (size_t)k * n;
    double ss = 0.0;
    for (int base = k + tid; base < n; base += U1 * HT) {
      double2 a[U1];
      if (base == k + tid) {
#pragma unroll
        for (int u = 0; u < U1; ++u) a[u] = pre[u];
      } else {
#pragma unroll
        for (int u = 0; u < U1; ++u) {
          const int c = base + u * HT;
          a[u] = c < n ? __ldcg(&rowk[c]) : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int c = base + u * HT;
        if (c < n) {
          const double2 x = csub(csub(a[u], cmulc(vpk, wp[c])), cmulc(wpk, vp[c]));
          if (c == k) {
            s_akk = x.x;
          } else {
            const double2 xc = conjg(x);  // column k below the diagonal
            vc[c] = xc;
            if (c >= k + 2) ss += xc.x * xc.x + xc.y * xc.y;
          }
        }
      }
    }
    // block sum of ss; alpha = vc[k+1] is read by every thread between the two
    // barriers, before its writer can rescale it below
    ss = warp_sum(ss);
    __syncthreads();
    if (lane == 0) red[warp] = ss;
    const double2 alpha = vc[k + 1];
    __syncthreads();
    ss = 0.0;
#pragma unroll
    for (int w = 0; w < HW; ++w) ss += red[w];
    double beta;
    double2 tk, sc;
    if (ss == 0.0 && alpha.y == 0.0) {
      tk = make_double2(0.0, 0.0);
      sc = make_double2(0.0, 0.0);
      beta = alpha.x;
    } else {
      beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
      tk = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
      const double2 den = make_double2(alpha.x - beta, alpha.y);
      const double m2 = den.x * den.x + den.y * den.y;
      sc = make_double2(den.x / m2, -den.y / m2);
    }
    if (bid == 0 && tid == 0) {
      d[k] = s_akk;
      e[k] = beta;
      tau[k] = tk;
    }
    // own entries of vc: v_k; reflector k-1 (own entries of vp) into row k-1,
    // which no CTA reads any more
    for (int c = k + tid; c < n; c += HT) {
      if (c > k) vc[c] = (c == k + 1) ? make_double2(1.0, 0.0) : cmul(vc[c], sc);
      if (bid == 0 && k > 0) __stcg(&A[(size_t)(k - 1) * n + c], vp[c]);
    }
    __syncthreads();

    // ---- phase 2: update k-1 on this CTA's trailing rows, y = A v_k
    const int nrow = n - k - 1;
    const int nr_c = nrow > bid ? (nrow - bid + G - 1) / G : 0;
    const int nch = (nrow + HCH - 1) / HCH;
    const int rb = max(1, PARTS / nch);
    double2 pdot = make_double2(0.0, 0.0);
    for (int j0 = 0; j0 < nr_c; j0 += rb) {
      const int jn = min(rb, nr_c - j0);
      const int nit = jn * nch;
      for (int it = warp; it < nit; it += 2 * HW) {
        const int it2 = it + HW;
        const int jl1 = it / nch, ch1 = it - jl1 * nch;
        const int r1 = k + 1 + bid + (j0 + jl1) * G;
        const int cb1 = k + 1 + ch1 * HCH + lane;
        double2* row1 = A + (size_t)r1 * n;
        double2 a1[U2], a2[U2];
#pragma unroll
        for (int u = 0; u < U2; ++u) {
          const int c = cb1 + 32 * u;
          a1[u] = c < n ? __ldcg(&row1[c]) : make_double2(0.0, 0.0);
        }
        int jl2 = 0, ch2 = 0, r2 = 0, cb2 = 0;
        double2* row2 = row1;
        if (it2 < nit) {
          jl2 = it2 / nch;
          ch2 = it2 - jl2 * nch;
          r2 = k + 1 + bid + (j0 + jl2) * G;
          cb2 = k + 1 + ch2 * HCH + lane;
          row2 = A + (size_t)r2 * n;
#pragma unroll
          for (int u = 0; u < U2; ++u) {
            const int c = cb2 + 32 * u;
            a2[u] = c < n ? __ldcg(&row2[c]) : make_double2(0.0, 0.0);
          }
        }
        double2 acc = hetrd_item(row1, cb1, n, vp[r1], wp[r1], vp, wp, vc, a1);
        acc = warp_sum(acc);
        if (lane == 0) parts[jl1 * nch + ch1] = acc;
        if (it2 < nit) {
          acc = hetrd_item(row2, cb2, n, vp[r2], wp[r2], vp, wp, vc, a2);
          acc = warp_sum(acc);
          if (lane == 0) parts[jl2 * nch + ch2] = acc;
        }
      }
      __syncthreads();
      for (int jl = tid; jl < jn; jl += HT) {
        double2 y = make_double2(0.0, 0.0);
        for (int ch = 0; ch < nch; ++ch) y = cadd(y, parts[jl * nch + ch]);
        const int r = k + 1 + bid + (j0 + jl) * G;
        __stcg(&Y[(size_t)(k & 1) * n + r], y);
        pdot = cadd(pdot, cmulc(vc[r], y));  // v_r conj(y_r)
      }
      __syncthreads();  // parts is refilled by the next row group
    }
    pdot = warp_sum(pdot);
    if (lane == 0) redc[warp] = pdot;
    __syncthreads();
    if (tid == 0) {
      double2 s = make_double2(0.0, 0.0);
      for (int w = 0; w < HW; ++w) s = cadd(s, redc[w]);
      __stcg(&P[(size_t)(k & 1) * G + bid], s);
    }
    if (!grid_sync(sync, (unsigned)G, gen, &s_ok, tab.wait_ns, pi == 0 && bid == 0 && k == tab.skip_column)) return;

    // ---- phase 3 (every CTA): w_k = tau y - (|tau|^2 / 2)(y^H v) v; every
    // warp sums the CTA partials itself.  The loads of y, of the partials, of
    // y_{k+1} and of row k+1 (phase 1 of the next column) go out together.
    const bool next = k + 2 < n;
    const double2* rown = A + (size_t)(k + 1) * n;
    double2 yv[U1];
#pragma unroll
    for (int u = 0; u < U1; ++u) {
      const int c = k + 1 + tid + u * HT;
      yv[u] = c < n ? __ldcg(&Y[(size_t)(k & 1) * n + c]) : make_double2(0.0, 0.0);
      pre[u] = (next && c < n) ? __ldcg(&rown[c]) : make_double2(0.0, 0.0);
    }
    const double2 yk1 = __ldcg(&Y[(size_t)(k & 1) * n + k + 1]);
    double2 dot = make_double2(0.0, 0.0);
    for (int base = lane; base < G; base += 32 * U1) {
      double2 pp[U1];
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int b = base + 32 * u;
        pp[u] = b < G ? __ldcg(&P[(size_t)(k & 1) * G + b]) : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < U1; ++u) dot = cadd(dot, pp[u]);
    }
    dot = warp_sum(dot);
    const double t2 = tk.x * tk.x + tk.y * tk.y;
    const double2 alph = make_double2(-0.5 * t2 * dot.x, -0.5 * t2 * dot.y);
    for (int base = k + 1 + tid; base < n; base += U1 * HT) {
      double2 y[U1];
      if (base == k + 1 + tid) {
#pragma unroll
        for (int u = 0; u < U1; ++u) y[u] = yv[u];
      } else {
#pragma unroll
        for (int u = 0; u < U1; ++u) {
          const int c = base + u * HT;
          y[u] = c < n ? __ldcg(&Y[(size_t)(k & 1) * n + c]) : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int c = base + u * HT;
        if (c < n) {
          const double2 v = vc[c];
          wp[c] = cadd(cmul(tk, y[u]), cmul(alph, v));
          vp[c] = v;
        }
      }
    }
    tk_prev = tk;
    alph_prev = alph;
    yk_prev = yk1;
  }
  if (bid == 0 && tid == 0) {
    if (n == 1) {
      d[0] = __ldcg(&A[0]).x;
    } else {
      double2 a = __ldcg(&A[(size_t)(n - 1) * n + (n - 1)]);
      a = csub(csub(a, cmulc(vp[n - 1], wp[n - 1])), cmulc(wp[n - 1], vp[n - 1]));
      d[n - 1] = a.x;
      __stcg(&A[(size_t)(n - 2) * n + (n - 1)], vp[n - 1]);
    }
  }
}

// ---------------------------------------------------------------- large matrices (n >= 3072), lower triangle
// The same lagged one-column-at-a-time reduction for large n, reading and
// updating only the lower triangle of A: half the bytes per column, and a
// 3584^2 complex matrix (205 MB in full) then stays in the 126 MB L2 instead
// of streaming from HBM twice per column.  Element (r, c), c < r, adds
// x v_c to y_r and conj(x) v_r to y_c; the diagonal adds x v_r to y_r.
//   phase 1 (every CTA)  "row" k is column k of the lower triangle (strided
//                        loads), update k-1 applied, reflector k;
//   phase 2              the trailing rows dealt round-robin to the CTAs; each
//                        warp owns column chunks of LCH columns (assigned in a
//                        snake order for balance) and walks the CTA's rows
//                        through them, two rows in flight: update k-1 stored,
//                        the row's chunk share of y kept in shared memory and
//                        the column contributions in the lanes' registers;
//                        the CTA writes its partial y (columns, plus its rows'
//                        sums in chunk order) to YP[bid][.];
//   grid barrier;
//   phase 2b             CTA b sums YP[0..G-1][i] for its slice of i (one warp
//                        per entry, lanes over the CTAs, fixed shuffle tree),
//                        writes y and its share of y^H v;
//   grid barrier;
//   phase 3 (every CTA)  w_k as before, with column k+1 loaded for phase 1.
// Every reduction has a fixed order, so the result is the same on every run.
constexpr int LU2 = 4;                 // loads in flight per lane per row of a chunk
constexpr int LCH = 32 * LU2;          // columns per chunk
constexpr int LPARTS = 2048;           // (row, chunk) partial sums per CTA
constexpr int YP_G = 256;              // largest CTA count per matrix (YP rows)
constexpr int LOWER_MIN_N = 3072;      // the lower-triangle kernel runs when the batch's largest n reaches this

// one row of a phase-2 chunk: update k-1 on its lower-triangle entries
// (a: their loaded values), stored back; the row's y share (warp-summed) is
// returned and the column contributions added to col
__device__ __forceinline__ double2 lower_row(double2* __restrict__ A, int r, int cs, int lane, int n,
                                             const double2* vp, const double2* wp, const double2* vc,
                                             const double2 (&a)[LU2], double2 (&col)[LU2]) {
  const double2 vpr = vp[r], wpr = wp[r], vr = vc[r];
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int u = 0; u < LU2; ++u) {
    const int c = cs + lane + 32 * u;
    if (c <= r && c < n) {
      const double2 x = csub(csub(a[u], cmulc(vpr, wp[c])), cmulc(wpr, vp[c]));
      __stcg(&A[(size_t)r * n + c], x);
      acc = cadd(acc, cmul(x, vc[c]));
      if (c < r) col[u] = cadd(col[u], cmul(conjg(x), vr));
    }
  }
  return warp_sum(acc);
}

__global__ void __launch_bounds__(HT, 1) hetrd_lower_kernel(const __grid_constant__ HetrdTable tab) {
  int pi = 0;
  while (pi + 1 < tab.count && (int)blockIdx.x >= tab.p[pi + 1].first) ++pi;
  const HetrdProb& PR = tab.p[pi];
  double2* __restrict__ A = PR.A;
  const int n = PR.n;
  double* __restrict__ d = PR.d;
  double* __restrict__ e = PR.e;
  double2* __restrict__ tau = PR.tau;
  double2* __restrict__ Y = PR.Y;
  double2* __restrict__ P = PR.P;
  double2* __restrict__ YP = PR.YP;
  Sync* sync = PR.sync;
  const int bid = (int)blockIdx.x - PR.first;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* vp = reinterpret_cast<double2*>(smem_raw);  // v of step k-1 (pending update)
  double2* wp = vp + n;                                // w of step k-1
  double2* vc = wp + n;                                // v of step k
  double2* parts = vc + n;                             // LPARTS (row, chunk) partial sums of y
  __shared__ double red[HW];
  __shared__ double2 redc[HW];
  __shared__ double s_akk;
  __shared__ int s_ok;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = PR.nblk;
  unsigned gen = 0;
  for (int i = tid; i < n; i += HT) {
    vp[i] = make_double2(0.0, 0.0);
    wp[i] = make_double2(0.0, 0.0);
    vc[i] = make_double2(0.0, 0.0);
  }
  // column 0 of the lower triangle, the part phase 1 reads in its first pass
  double2 pre[U1];
#pragma unroll
  for (int u = 0; u < U1; ++u) {
    const int c = tid + u * HT;
    pre[u] = c < n ? conjg(__ldcg(&A[(size_t)c * n])) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2 tk_prev = make_double2(0.0, 0.0), alph_prev = make_double2(0.0, 0.0), yk_prev = make_double2(0.0, 0.0);
  for (int k = 0; k < n - 1; ++k) {
    // ---- phase 1 (every CTA): row k = conj(column k) with update k-1, reflector k
    double2 vpk = make_double2(0.0, 0.0), wpk = make_double2(0.0, 0.0);
    if (k > 0) {
      vpk = make_double2(1.0, 0.0);
      wpk = cadd(cmul(tk_prev, yk_prev), cmul(alph_prev, vpk));
    }
    double ss = 0.0;
    for (int base = k + tid; base < n; base += U1 * HT) {
      double2 a[U1];
      if (base == k + tid) {
#pragma unroll
        for (int u = 0; u < U1; ++u) a[u] = pre[u];
      } else {
#pragma unroll
        for (int u = 0; u < U1; ++u) {
          const int c = base + u * HT;
          a[u] = c < n ? conjg(__ldcg(&A[(size_t)c * n + k])) : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int c = base + u * HT;
        if (c < n) {
          const double2 x = csub(csub(a[u], cmulc(vpk, wp[c])), cmulc(wpk, vp[c]));
          if (c == k) {
            s_akk = x.x;
          } else {
            const double2 xc = conjg(x);
            vc[c] = xc;
            if (c >= k + 2) ss += xc.x * xc.x + xc.y * xc.y;
          }
        }
      }
    }
    ss = warp_sum(ss);
    __syncthreads();
    if (lane == 0) red[warp] = ss;
    const double2 alpha = vc[k + 1];
    __syncthreads();
    ss = 0.0;
#pragma unroll
    for (int w = 0; w < HW; ++w) ss += red[w];
    double beta;
    double2 tk, sc;
    if (ss == 0.0 && alpha.y == 0.0) {
      tk = make_double2(0.0, 0.0);
      sc = make_double2(0.0, 0.0);
      beta = alpha.x;
    } else {
      beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
      tk = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
      const double2 den = make_double2(alpha.x - beta, alpha.y);
      const double m2 = den.x * den.x + den.y * den.y;
      sc = make_double2(den.x / m2, -den.y / m2);
    }
    if (bid == 0 && tid == 0) {
      d[k] = s_akk;
      e[k] = beta;
      tau[k] = tk;
    }
    // own entries of vc: v_k; reflector k-1 into row k-1 (upper triangle, which
    // this kernel never reads)
    for (int c = k + tid; c < n; c += HT) {
      if (c > k) vc[c] = (c == k + 1) ? make_double2(1.0, 0.0) : cmul(vc[c], sc);
      if (bid == 0 && k > 0) __stcg(&A[(size_t)(k - 1) * n + c], vp[c]);
    }
    __syncthreads();

    // ---- phase 2: update k-1 on the lower triangle of this CTA's rows; partial y
    const int nrow = n - k - 1;
    const int nr_c = nrow > bid ? (nrow - bid + G - 1) / G : 0;
    const int nch = (nrow + LCH - 1) / LCH;
    double2* yp = YP + (size_t)bid * n;
    // chunk ch of warp w: ch = w + 2 HW t or 2 HW - 1 - w + 2 HW t
    for (int t = 0; 2 * HW * t + warp < nch; ++t) {
#pragma unroll 1
      for (int q = 0; q < 2; ++q) {
        const int ch = q == 0 ? 2 * HW * t + warp : 2 * HW * t + 2 * HW - 1 - warp;
        if (ch >= nch) continue;
        const int cs = k + 1 + ch * LCH;
        double2 col[LU2];
#pragma unroll
        for (int u = 0; u < LU2; ++u) col[u] = make_double2(0.0, 0.0);
        // first own row reaching this chunk: r_j >= cs
        const int j0 = cs - (k + 1 + bid) > 0 ? (cs - (k + 1 + bid) + G - 1) / G : 0;
        for (int j = j0; j < nr_c; j += 2) {
          const int r1 = k + 1 + bid + j * G;
          const bool two = j + 1 < nr_c;
          const int r2 = two ? r1 + G : r1;
          double2 a1[LU2], a2[LU2];
#pragma unroll
          for (int u = 0; u < LU2; ++u) {
            const int c = cs + lane + 32 * u;
            a1[u] = (c <= r1 && c < n) ? __ldcg(&A[(size_t)r1 * n + c]) : make_double2(0.0, 0.0);
            a2[u] = (two && c <= r2 && c < n) ? __ldcg(&A[(size_t)r2 * n + c]) : make_double2(0.0, 0.0);
          }
          double2 acc = lower_row(A, r1, cs, lane, n, vp, wp, vc, a1, col);
          if (lane == 0) parts[j * nch + ch] = acc;
          if (two) {
            acc = lower_row(A, r2, cs, lane, n, vp, wp, vc, a2, col);
            if (lane == 0) parts[(j + 1) * nch + ch] = acc;
          }
        }
#pragma unroll
        for (int u = 0; u < LU2; ++u) {
          const int c = cs + lane + 32 * u;
          if (c < n) __stcg(&yp[c], col[u]);
        }
      }
    }
    __syncthreads();
    // this CTA's rows: add their sums over the chunks they reach, in chunk order
    for (int j = tid; j < nr_c; j += HT) {
      const int r = k + 1 + bid + j * G;
      const int chmax = (r - k - 1) / LCH;
      double2 s = __ldcg(&yp[r]);
      double2 rs = make_double2(0.0, 0.0);
      for (int ch = 0; ch <= chmax; ++ch) rs = cadd(rs, parts[j * nch + ch]);
      __stcg(&yp[r], cadd(s, rs));
    }
    if (!grid_sync(sync, (unsigned)G, gen, &s_ok, tab.wait_ns, pi == 0 && bid == 0 && k == tab.skip_column)) return;

    // ---- phase 2b: y_i = sum over the CTAs' partials, one warp per entry of this CTA's slice
    const int sl = (nrow + G - 1) / G;
    const int i0 = k + 1 + bid * sl, i1 = min(n, i0 + sl);
    double2 pdot = make_double2(0.0, 0.0);
    for (int i = i0 + warp; i < i1; i += HW) {
      // G <= YP_G = 8 x 32: every lane's partials are loaded before any is summed
      double2 part[YP_G / 32];
#pragma unroll
      for (int u = 0; u < YP_G / 32; ++u) {
        const int b = lane + 32 * u;
        part[u] = b < G ? __ldcg(&YP[(size_t)b * n + i]) : make_double2(0.0, 0.0);
      }
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int u = 0; u < YP_G / 32; ++u) acc = cadd(acc, part[u]);
      acc = warp_sum(acc);
      if (lane == 0) {
        __stcg(&Y[(size_t)(k & 1) * n + i], acc);
        pdot = cadd(pdot, cmulc(vc[i], acc));
      }
    }
    if (lane == 0) redc[warp] = pdot;
    __syncthreads();
    if (tid == 0) {
      double2 sum = make_double2(0.0, 0.0);
      for (int w = 0; w < HW; ++w) sum = cadd(sum, redc[w]);
      __stcg(&P[(size_t)(k & 1) * G + bid], sum);
    }
    if (!grid_sync(sync, (unsigned)G, gen, &s_ok, tab.wait_ns, false)) return;

    // ---- phase 3 (every CTA): w_k; column k+1 loaded for the next phase 1
    const bool next = k + 2 < n;
    double2 yv[U1];
#pragma unroll
    for (int u = 0; u < U1; ++u) {
      const int c = k + 1 + tid + u * HT;
      yv[u] = c < n ? __ldcg(&Y[(size_t)(k & 1) * n + c]) : make_double2(0.0, 0.0);
      pre[u] = (next && c < n) ? conjg(__ldcg(&A[(size_t)c * n + k + 1])) : make_double2(0.0, 0.0);
    }
    const double2 yk1 = __ldcg(&Y[(size_t)(k & 1) * n + k + 1]);
    double2 dot = make_double2(0.0, 0.0);
    for (int base = lane; base < G; base += 32 * U1) {
      double2 pp[U1];
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int b = base + 32 * u;
        pp[u] = b < G ? __ldcg(&P[(size_t)(k & 1) * G + b]) : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < U1; ++u) dot = cadd(dot, pp[u]);
    }
    dot = warp_sum(dot);
    const double t2 = tk.x * tk.x + tk.y * tk.y;
    const double2 alph = make_double2(-0.5 * t2 * dot.x, -0.5 * t2 * dot.y);
    for (int base = k + 1 + tid; base < n; base += U1 * HT) {
      double2 y[U1];
      if (base == k + 1 + tid) {
#pragma unroll
        for (int u = 0; u < U1; ++u) y[u] = yv[u];
      } else {
#pragma unroll
        for (int u = 0; u < U1; ++u) {
          const int c = base + u * HT;
          y[u] = c < n ? __ldcg(&Y[(size_t)(k & 1) * n + c]) : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int c = base + u * HT;
        if (c < n) {
          const double2 v = vc[c];
          wp[c] = cadd(cmul(tk, y[u]), cmul(alph, v));
          vp[c] = v;
        }
      }
    }
    tk_prev = tk;
    alph_prev = alph;
    yk_prev = yk1;
  }
  if (bid == 0 && tid == 0) {
    if (n == 1) {
      d[0] = __ldcg(&A[0]).x;
    } else {
      double2 a = __ldcg(&A[(size_t)(n - 1) * n + (n - 1)]);
      a = csub(csub(a, cmulc(vp[n - 1], wp[n - 1])), cmulc(wp[n - 1], vp[n - 1]));
      d[n - 1] = a.x;
      __stcg(&A[(size_t)(n - 2) * n + (n - 1)], vp[n - 1]);
    }
  }
}

// ---------------------------------------------------------------- small matrices
// n <= 256: the same lagged one-barrier-per-column reduction on one
// thread-block cluster of CL CTAs whose shared memories hold the matrix
// (row r in CTA r % CL, slot r / CL).  Row k is read from its owner through
// distributed shared memory, y_r and the partial dots are pushed to every CTA
// (double-buffered by column parity, so a CTA that runs ahead never
// overwrites a buffer another is still reading), and the hardware cluster
// barrier, which every CTA executes the same number of times, separates the
// columns.  Reflector k is written to row k of Aout (which may alias Gin: all
// of Gin is read before the first barrier).  blockIdx.y = matrix.
constexpr int CL = 8, CT = 256, CW = CT / 32, NMAX_C = 256, RL = NMAX_C / CL;

inline size_t cluster_smem_bytes(int n) {
  return ((size_t)RL * n + 5 * (size_t)n + 2 * CL) * sizeof(double2);
}

__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(CT, 1)
    hetrd_cluster_kernel(const __grid_constant__ EigTable tab) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const EigProb& PR = tab.p[blockIdx.y];
  const double2* __restrict__ Gin = PR.a;
  double2* Aout = PR.a;
  const int n = PR.n;
  double* __restrict__ d = PR.d;
  double* __restrict__ e = PR.e;
  double2* __restrict__ tau = PR.tau;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* rows = reinterpret_cast<double2*>(smem_raw);  // RL x n
  double2* vp = rows + (size_t)RL * n;
  double2* wp = vp + n;
  double2* vc = wp + n;
  double2* yb = vc + n;      // 2 x n
  double2* pb = yb + 2 * n;  // 2 x CL
  __shared__ double red[CW];
  __shared__ double2 redc[CW];
  __shared__ double2 s_scale, s_tau;
  __shared__ double s_akk;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int sl = 0; sl < RL; ++sl) {
    const int r = sl * CL + rank;
    if (r < n)
      for (int c = tid; c < n; c += CT) rows[(size_t)sl * n + c] = Gin[(size_t)r * n + c];
  }
  for (int i = tid; i < n; i += CT) {
    vp[i] = make_double2(0.0, 0.0);
    wp[i] = make_double2(0.0, 0.0);
    vc[i] = make_double2(0.0, 0.0);
  }
  cluster.sync();
  for (int k = 0; k < n - 1; ++k) {
    const int par = k & 1;
    // ---- phase 1: row k from its owner, update k-1 applied, reflector k
    const double2* rk = cluster.map_shared_rank(rows + (size_t)(k / CL) * n, k % CL);
    const double2 vpk = vp[k], wpk = wp[k];
    double ss = 0.0;
    for (int c = k + tid; c < n; c += CT) {
      const double2 x = csub(csub(rk[c], cmulc(vpk, wp[c])), cmulc(wpk, vp[c]));
      if (c == k) {
        s_akk = x.x;
      } else {
        const double2 xc = conjg(x);
        vc[c] = xc;
        if (c >= k + 2) ss += xc.x * xc.x + xc.y * xc.y;
      }
    }
    ss = block_sum<CW>(ss, red);
    if (tid == 0) {
      const double2 alpha = vc[k + 1];
      double beta;
      if (ss == 0.0 && alpha.y == 0.0) {
        s_tau = make_double2(0.0, 0.0);
        s_scale = make_double2(0.0, 0.0);
        beta = alpha.x;
      } else {
        beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
        s_tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
        const double2 den = make_double2(alpha.x - beta, alpha.y);
        const double m2 = den.x * den.x + den.y * den.y;
        s_scale = make_double2(den.x / m2, -den.y / m2);
      }
      if (rank == 0) {
        d[k] = s_akk;
        e[k] = beta;
        tau[k] = s_tau;
      }
    }
    __syncthreads();
    const double2 sc = s_scale, tk = s_tau;
    for (int c = k + 1 + tid; c < n; c += CT) {
      const double2 v = (c == k + 1) ? make_double2(1.0, 0.0) : cmul(vc[c], sc);
      vc[c] = v;
      if (rank == 0) Aout[(size_t)k * n + c] = v;
    }
    __syncthreads();
    // ---- phase 2: owned rows r >= k+1: update k-1, y_r = row . v_k, pushed to every CTA
    double2 pdot = make_double2(0.0, 0.0);
    for (int sl = warp; sl < RL; sl += CW) {
      const int r = sl * CL + rank;
      if (r <= k || r >= n) continue;
      double2* row = rows + (size_t)sl * n;
      const double2 vpr = vp[r], wpr = wp[r];
      double2 acc = make_double2(0.0, 0.0);
      for (int c = k + 1 + lane; c < n; c += 32) {
        const double2 x = csub(csub(row[c], cmulc(vpr, wp[c])), cmulc(wpr, vp[c]));
        row[c] = x;
        acc = cadd(acc, cmul(x, vc[c]));
      }
      acc = warp_sum(acc);
      if (lane < CL) cluster.map_shared_rank(yb + (size_t)par * n, lane)[r] = acc;
      if (lane == 0) pdot = cadd(pdot, cmulc(vc[r], acc));
    }
    if (lane == 0) redc[warp] = pdot;
    __syncthreads();
    if (tid < CL) {
      double2 sum = make_double2(0.0, 0.0);
      for (int w = 0; w < CW; ++w) sum = cadd(sum, redc[w]);
      cluster.map_shared_rank(pb + par * CL, tid)[rank] = sum;
    }
    cluster.sync();
    // ---- phase 3: w_k = tau y - (|tau|^2 / 2)(y^H v) v
    double2 dot = make_double2(0.0, 0.0);
    for (int q = 0; q < CL; ++q) dot = cadd(dot, pb[par * CL + q]);
    const double t2 = tk.x * tk.x + tk.y * tk.y;
    const double2 alph = make_double2(-0.5 * t2 * dot.x, -0.5 * t2 * dot.y);
    for (int c = k + 1 + tid; c < n; c += CT) {
      const double2 v = vc[c];
      wp[c] = cadd(cmul(tk, yb[(size_t)par * n + c]), cmul(alph, v));
      vp[c] = v;
    }
    __syncthreads();
  }
  if (rank == 0 && tid == 0) {
    if (n == 1) {
      d[0] = rows[0].x;
    } else {
      const double2* rn = cluster.map_shared_rank(rows + (size_t)((n - 1) / CL) * n, (n - 1) % CL);
      const double2 a = csub(csub(rn[n - 1], cmulc(vp[n - 1], wp[n - 1])), cmulc(wp[n - 1], vp[n - 1]));
      d[n - 1] = a.x;
    }
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------- eigenvalues
// Number of eigenvalues of T below x (LDL^T pivots, LAPACK dstebz's guard
// |q| >= pivmin).
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int n, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int cnt = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// Gershgorin bounds and pivmin of T into out[0..2] (one block)
__global__ void __launch_bounds__(THREADS) bounds_kernel(const __grid_constant__ EigTable tab) {
  const EigProb& PR = tab.p[blockIdx.y];
  const double* __restrict__ d = PR.d;
  const double* __restrict__ e = PR.e;
  const int n = PR.n;
  double* __restrict__ out = PR.bnd;
  __shared__ double rmin[WARPS], rmax[WARPS], re2[WARPS];
  double lo = DBL_MAX, hi = -DBL_MAX, m2 = 0.0;
  for (int i = threadIdx.x; i < n; i += THREADS) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    if (i < n - 1) m2 = fmax(m2, e[i] * e[i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    rmin[warp] = lo;
    rmax[warp] = hi;
    re2[warp] = m2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < WARPS; ++w) {
      lo = fmin(lo, rmin[w]);
      hi = fmax(hi, rmax[w]);
      m2 = fmax(m2, re2[w]);
    }
    lo = fmin(lo, rmin[0]);
    hi = fmax(hi, rmax[0]);
    m2 = fmax(m2, re2[0]);
    const double tn = fmax(fabs(lo), fabs(hi));
    const double pivmin = DBL_MIN * fmax(1.0, m2);
    out[0] = lo - 2.0 * DBL_EPSILON * tn - 2.0 * pivmin;
    out[1] = hi + 2.0 * DBL_EPSILON * tn + 2.0 * pivmin;
    out[2] = pivmin;
  }
}

// eigenvalue i0 + j (ascending) of T for j < cnt, one warp each
__global__ void __launch_bounds__(THREADS) bisect_kernel(const __grid_constant__ EigTable tab) {
  const EigProb& PR = tab.p[blockIdx.y];
  const double* __restrict__ d = PR.d;
  const double* __restrict__ e = PR.e;
  const int n = PR.n, i0 = PR.n - PR.kt, cnt = PR.kt;
  const double* __restrict__ bnd = PR.bnd;
  double* __restrict__ w = PR.w;
  extern __shared__ double sh[];
  double* sd = sh;
  double* se2 = sh + n;
  for (int i = threadIdx.x; i < n; i += THREADS) {
    sd[i] = d[i];
    if (i < n - 1) se2[i] = e[i] * e[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * WARPS + (threadIdx.x >> 5);
  if (j >= cnt) return;
  const int idx = i0 + j;
  const double pivmin = bnd[2];
  double lo = bnd[0], hi = bnd[1];
  for (int round = 0; round < 40; ++round) {
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    const double x = lo + (hi - lo) * ((double)(lane + 1) / 33.0);
    const int c = sturm_count(sd, se2, n, x, pivmin);
    // count(x) > idx  <=>  eigenvalue idx < x
    const unsigned above = __ballot_sync(0xffffffffu, c > idx);
    const int first = above ? __ffs(above) - 1 : 32;
    const double xl = __shfl_sync(0xffffffffu, x, first > 0 ? first - 1 : 0);
    const double xh = __shfl_sync(0xffffffffu, x, first < 32 ? first : 31);
    const double nlo = first == 0 ? lo : xl;
    const double nhi = first == 32 ? hi : xh;
    if (nlo == lo && nhi == hi) break;
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) w[j] = 0.5 * (lo + hi);
}

// ---------------------------------------------------------------- eigenvectors
__device__ __forceinline__ double hash_unit(uint32_t a, uint32_t b) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  h *= 0x297A2D39u;
  h ^= h >> 15;
  return (double)h * (2.0 / 4294967296.0) - 1.0;
}

// column j of Z (n x cnt row-major) = eigenvector of T for w[j]; scratch:
// 4 * n * cnt doubles laid out [i * cnt + j] (coalesced across threads).
// d, e are staged in shared memory; every sequential loop loads the next CH
// steps' independent inputs before running their dependent chain.
constexpr int IV_THREADS = 128, CH = 8;
__global__ void __launch_bounds__(IV_THREADS) inviter_kernel(const __grid_constant__ EigTable tab) {
  const EigProb& PR = tab.p[blockIdx.y];
  const double* __restrict__ d = PR.d;
  const double* __restrict__ e = PR.e;
  const int n = PR.n, cnt = PR.kt;
  const double* __restrict__ w = PR.w;
  const double* __restrict__ bnd = PR.bnd;
  double* __restrict__ Z = PR.z;
  double* __restrict__ scr = PR.scr;
  extern __shared__ double sh_de[];
  double* sd = sh_de;
  double* se = sh_de + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sd[i] = d[i];
    se[i] = i < n - 1 ? e[i] : 0.0;
  }
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cnt) return;
  const size_t S = (size_t)cnt;
  double* ua = scr;                       // 1 / u_kk
  double* uc = scr + 1 * (size_t)n * S;   // u_{k,k+1}
  double* uc2 = scr + 2 * (size_t)n * S;  // u_{k,k+2}
  double* ml = scr + 3 * (size_t)n * S;   // multiplier (+4 when rows k, k+1 were swapped)
  const double lam = w[j];
  const double tn = fmax(fabs(bnd[0]), fabs(bnd[1]));
  const double tiny = DBL_EPSILON * fmax(tn, DBL_MIN);
  // LU of T - lam I with partial pivoting.  The current row k has entries
  // (ak, ck) at columns (k, k+1); the next original row is (bk, ak1, ck1) at
  // columns (k, k+1, k+2).  U row k is (ak, ck, 0) without a swap and
  // (bk, ak1, ck1) with one; |multiplier| <= 1 either way.
  double ak = sd[0] - lam;
  double ck = se[0];
  for (int k = 0; k < n - 1; ++k) {
    const double bk = se[k];
    const double ak1 = sd[k + 1] - lam;
    const double ck1 = se[k + 1];
    double u_kk, u_k1, u_k2, flagged;
    if (fabs(ak) >= fabs(bk)) {
      u_kk = ak == 0.0 ? tiny : ak;
      u_k1 = ck;
      u_k2 = 0.0;
      const double m = bk / u_kk;
      flagged = m;
      ak = ak1 - m * ck;
      ck = ck1;
    } else {
      u_kk = bk;
      u_k1 = ak1;
      u_k2 = ck1;
      const double m = ak / bk;
      flagged = m + 4.0;
      ak = ck - m * ak1;
      ck = -m * ck1;
    }
    if (fabs(u_kk) < tiny) u_kk = copysign(tiny, u_kk);
    ua[(size_t)k * S + j] = 1.0 / u_kk;
    uc[(size_t)k * S + j] = u_k1;
    uc2[(size_t)k * S + j] = u_k2;
    ml[(size_t)k * S + j] = flagged;
  }
  {
    double u = ak;
    if (fabs(u) < tiny) u = copysign(tiny, u == 0.0 ? 1.0 : u);
    ua[(size_t)(n - 1) * S + j] = 1.0 / u;
    uc[(size_t)(n - 1) * S + j] = 0.0;
    uc2[(size_t)(n - 1) * S + j] = 0.0;
  }
  double* z = Z;
#pragma unroll 8
  for (int i = 0; i < n; ++i) z[(size_t)i * S + j] = hash_unit((uint32_t)j + 1u, (uint32_t)i);
  for (int it = 0; it < 3; ++it) {
    // forward: L^-1 with the row swaps
    double zk = z[j];
    for (int k0 = 0; k0 < n - 1; k0 += CH) {
      double mm[CH], zn[CH];
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        const int k = k0 + u;
        mm[u] = k < n - 1 ? ml[(size_t)k * S + j] : 0.0;
        zn[u] = k < n - 1 ? z[(size_t)(k + 1) * S + j] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        const int k = k0 + u;
        if (k < n - 1) {
          if (mm[u] > 2.0) {  // rows k, k+1 swapped
            z[(size_t)k * S + j] = zn[u];
            zk = zk - (mm[u] - 4.0) * zn[u];
          } else {
            z[(size_t)k * S + j] = zk;
            zk = zn[u] - mm[u] * zk;
          }
        }
      }
    }
    z[(size_t)(n - 1) * S + j] = zk;
    // backward: U with two super-diagonals
    double z1 = 0.0, z2 = 0.0, nrm = 0.0;
    for (int k0 = n - 1; k0 >= 0; k0 -= CH) {
      double zz[CH], c1[CH], c2[CH], ia[CH];
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        const int k = k0 - u;
        const bool ok = k >= 0;
        zz[u] = ok ? z[(size_t)k * S + j] : 0.0;
        c1[u] = ok ? uc[(size_t)k * S + j] : 0.0;
        c2[u] = ok ? uc2[(size_t)k * S + j] : 0.0;
        ia[u] = ok ? ua[(size_t)k * S + j] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        const int k = k0 - u;
        if (k >= 0) {
          const double v = (zz[u] - c1[u] * z1 - c2[u] * z2) * ia[u];
          z[(size_t)k * S + j] = v;
          z2 = z1;
          z1 = v;
          nrm += v * v;
        }
      }
    }
    const double inv = nrm > 0.0 ? 1.0 / sqrt(nrm) : 0.0;
#pragma unroll 8
    for (int i = 0; i < n; ++i) z[(size_t)i * S + j] *= inv;
  }
}

// ---------------------------------------------------------------- back-transformation
// K = Q K with Q = H_0 ... H_{n-2} in blocks of NB reflectors (compact WY:
// H_k0 ... H_k0+kb-1 = I - V T V^H, LAPACK's forward columnwise larft), the
// blocks applied from the last to the first, each as three FP64 GEMMs.
constexpr int NB = 64;
constexpr int KCH = 256;  // row chunk of the split-K products V_b^H K

inline int nch_max(int n) { return (int)ceil_div(std::max(n - 1, 1), KCH); }

// rows 0..n-2 of A become the reflectors (0 before column k+1, 1 at k+1) and
// row n-1 becomes 0, so that every reflector row can be read over all n columns
__global__ void clean_v_kernel(double2* __restrict__ A, int n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n * n) return;
  const int k = (int)(idx / n), c = (int)(idx % n);
  if (k == n - 1 || c <= k) A[idx] = make_double2(0.0, 0.0);
  else if (c == k + 1) A[idx] = make_double2(1.0, 0.0);
}

// minus the NB x NB upper-triangular T of block b from S = V^H V and tau,
// written rep times side by side (row i of block b at
// Tg + (b NB + i) NB rep): the split-K partials of V^H K then sum inside the
// T product.  Thread i owns row i (written and read only by itself).
__global__ void __launch_bounds__(NB) larft_kernel(const double2* __restrict__ Sg, const double2* __restrict__ tau,
                                                   double2* __restrict__ Tg, int n, int rep) {
  __shared__ double2 x[NB];
  const int b = blockIdx.x, i = threadIdx.x;
  const int k0 = b * NB, kb = min(NB, n - 1 - k0);
  const double2* S = Sg + (size_t)b * NB * NB;
  double2* T = Tg + ((size_t)b * NB + i) * NB * rep;
  for (int c = 0; c < NB; ++c) T[c] = make_double2(0.0, 0.0);
  for (int j = 0; j < kb; ++j) {
    const double2 tj = tau[k0 + j];
    if (i < j) x[i] = cmul(make_double2(-tj.x, -tj.y), S[(size_t)i * NB + j]);
    __syncthreads();
    if (i < j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int l = i; l < j; ++l) acc = cadd(acc, cmul(T[l], x[l]));
      T[j] = acc;
    } else if (i == j) {
      T[j] = tj;
    }
    __syncthreads();
  }
  for (int c = 0; c < NB; ++c) {
    const double2 v = make_double2(-T[c].x, -T[c].y);
    for (int r = 0; r < rep; ++r) T[(size_t)r * NB + c] = v;
  }
}

}  // namespace heev
}  // namespace reno

using namespace reno;
using namespace reno::heev;

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

namespace {
struct HeevLayout {
  size_t sync, y, p, yp, bnd, scr, s, t, w1, w2, total;
};
HeevLayout heev_layout(int n, int kt) {
  HeevLayout L{};
  const size_t nblk = (size_t)ceil_div(std::max(n - 1, 1), NB);
  size_t off = 0;
  L.sync = off;
  off += align256(sizeof(Sync));
  L.y = off;
  off += align256(2 * (size_t)n * sizeof(double2));
  L.p = off;
  off += align256(2 * 1024 * sizeof(double2));
  L.yp = off;  // partial sums of the lower-triangle reduction (grid path only)
  off += n > NMAX_C ? align256((size_t)YP_G * n * sizeof(double2)) : 0;
  L.bnd = off;
  off += align256(4 * sizeof(double));
  L.scr = off;
  off += align256(4 * (size_t)n * kt * sizeof(double));
  L.s = off;
  off += align256(nblk * NB * NB * sizeof(double2));
  L.t = off;
  off += align256(nblk * NB * NB * nch_max(n) * sizeof(double2));
  L.w1 = off;
  off += align256((size_t)nch_max(n) * NB * kt * sizeof(double2));
  L.w2 = off;
  off += align256((size_t)NB * kt * sizeof(double2));
  L.total = off;
  return L;
}

GemmOperand op(const void* p, int64_t s_outer, int64_t s_k, int conj) {
  GemmOperand o;
  o.ptr = p;
  o.s_outer = s_outer;
  o.s_k = s_k;
  o.is_complex = 1;
  o.conj = conj;
  return o;
}
}  // namespace

// Cooperative launch of the reduction over the matrices of tab (n > NMAX_C):
// one CTA per SM, the SMs shared out in proportion to each matrix's n^2.  When
// the largest matrix has at least LOWER_MIN_N rows the lower-triangle kernel
// runs (each matrix then needs enough CTAs that its rows' (row, chunk)
// partials fit LPARTS, and at most YP_G); otherwise the full-row kernel.
static int launch_hetrd(reno_ctx* ctx, HetrdTable& tab, int nmax, const char* what) {
  static std::atomic<unsigned long long> hetrd_set{0}, lower_set{0};
  int rc = check_cuda(ctx, smem_optin_once(hetrd_kernel, (3 * MAX_N + PARTS) * 16, hetrd_set),
                      (std::string(what) + ": hetrd smem attribute").c_str());
  if (rc == RENO_OK)
    rc = check_cuda(ctx, smem_optin_once(hetrd_lower_kernel, (3 * MAX_N + LPARTS) * 16, lower_set),
                    (std::string(what) + ": hetrd smem attribute").c_str());
  if (rc != RENO_OK) return rc;
  const int G = std::min(sm_count_current_device(), 1024);
  if (tab.count > G) return set_error(ctx, RENO_ERR_INVALID, std::string(what) + ": more matrices than SMs");
  // CTAs a matrix needs under the lower-triangle kernel
  auto gmin_lower = [](int n) {
    const int nch = (int)ceil_div(n - 1, LCH);
    const int rows = std::max(1, LPARTS / std::max(nch, 1));
    return (int)ceil_div(n - 1, rows);
  };
  // RENO_HETRD_LOWER_MIN overrides the size from which the lower-triangle kernel runs
  static const int lower_min = [] {
    const char* e = std::getenv("RENO_HETRD_LOWER_MIN");
    return (e && std::atoi(e) > 0) ? std::atoi(e) : LOWER_MIN_N;
  }();
  bool lower = nmax >= lower_min;
  int need = 0;
  for (int i = 0; i < tab.count; ++i) {
    if (!tab.p[i].YP) lower = false;
    need += gmin_lower(tab.p[i].n);
  }
  if (need > G) lower = false;
  void* kfn = lower ? (void*)hetrd_lower_kernel : (void*)hetrd_kernel;
  const size_t smem = (3 * (size_t)nmax + (lower ? LPARTS : PARTS)) * sizeof(double2);
  int per_sm = 0;
  rc = check_cuda(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, HT, smem),
                  (std::string(what) + ": occupancy").c_str());
  if (rc != RENO_OK) return rc;
  if (per_sm < 1) return set_error(ctx, RENO_ERR_INVALID, std::string(what) + ": hetrd kernel does not fit on an SM");
  double work = 0.0;
  for (int i = 0; i < tab.count; ++i) work += (double)tab.p[i].n * tab.p[i].n;
  int used = 0, reserved = 0;
  if (lower)
    for (int i = 0; i < tab.count; ++i) reserved += gmin_lower(tab.p[i].n);
  for (int i = 0; i < tab.count; ++i) {
    const int left = tab.count - 1 - i;  // at least one CTA for every later matrix
    const int floor_i = lower ? gmin_lower(tab.p[i].n) : 1;
    if (lower) reserved -= floor_i;
    const int later = lower ? reserved : left;
    int nb = i == tab.count - 1 ? G - used
                                : (int)std::lround(G * (double)tab.p[i].n * tab.p[i].n / std::max(work, 1.0));
    nb = std::max(floor_i, std::min(nb, G - used - later));
    if (lower) nb = std::min(nb, YP_G);
    tab.p[i].first = used;
    tab.p[i].nblk = nb;
    used += nb;
  }
  tab.wait_ns = g_wait_ns.load(std::memory_order_relaxed);
  tab.skip_column = g_skip_hetrd_column.exchange(-1);
  void* args[] = {&tab};
  count_launch();
  return check_cuda(ctx, cudaLaunchCooperativeKernel(kfn, dim3(used), dim3(HT), args, smem, ctx->stream),
                    (std::string(what) + ": hetrd launch").c_str());
}

extern "C" int reno_heev_workspace_bytes(int32_t n, int32_t kt, size_t* bytes) {
  if (!bytes || n < 1 || n > MAX_N || kt < 1 || kt > n) return RENO_ERR_INVALID;
  *bytes = heev_layout(n, kt).total;
  return RENO_OK;
}

namespace {

int heev_attrs(reno_ctx* ctx) {
  static std::atomic<unsigned long long> bisect_set{0}, inviter_set{0}, cluster_set{0};
  int rc = check_cuda(ctx, smem_optin_once(bisect_kernel, 2 * MAX_N * (int)sizeof(double), bisect_set),
                      "reno_heev_top: bisect smem attribute");
  if (rc == RENO_OK)
    rc = check_cuda(ctx, smem_optin_once(inviter_kernel, 2 * MAX_N * (int)sizeof(double), inviter_set),
                    "reno_heev_top: inverse iteration smem attribute");
  if (rc == RENO_OK)
    rc = check_cuda(ctx, smem_optin_once(hetrd_cluster_kernel, (int)cluster_smem_bytes(NMAX_C), cluster_set),
                    "reno_heev_top: cluster smem attribute");
  return rc;
}

// tridiagonal reduction of small matrices (n <= NMAX_C): one thread-block
// cluster per matrix, all in one launch
int heev_reduce_small(reno_ctx* ctx, const EigTable& tab, int nmax) {
  if (tab.count == 0) return RENO_OK;
  count_launch();
  hetrd_cluster_kernel<<<dim3(CL, tab.count), CT, cluster_smem_bytes(nmax), ctx->stream>>>(tab);
  RENO_LAUNCH_CHECK(ctx, "reno_heev_top: cluster hetrd");
  return RENO_OK;
}

// eigenvalues n-kt .. n-1 of every T (ascending) and their inverse-iteration
// vectors: one launch per stage for all matrices of the table
int heev_eig(reno_ctx* ctx, const EigTable& tab) {
  if (tab.count == 0) return RENO_OK;
  int nmax = 1, ktmax = 1;
  for (int i = 0; i < tab.count; ++i) {
    nmax = std::max(nmax, tab.p[i].n);
    ktmax = std::max(ktmax, tab.p[i].kt);
  }
  cudaStream_t st = ctx->stream;
  count_launch();
  bounds_kernel<<<dim3(1, tab.count), THREADS, 0, st>>>(tab);
  RENO_LAUNCH_CHECK(ctx, "reno_heev_top: bounds");
  count_launch();
  bisect_kernel<<<dim3((unsigned)ceil_div(ktmax, WARPS), tab.count), THREADS, 2 * (size_t)nmax * sizeof(double),
                  st>>>(tab);
  RENO_LAUNCH_CHECK(ctx, "reno_heev_top: bisect");
  count_launch();
  inviter_kernel<<<dim3((unsigned)ceil_div(ktmax, IV_THREADS), tab.count), IV_THREADS,
                   2 * (size_t)nmax * sizeof(double), st>>>(tab);
  RENO_LAUNCH_CHECK(ctx, "reno_heev_top: inverse iteration");
  return RENO_OK;
}

bool heev_problem_ok(const reno_heev_problem& p) {
  return p.n >= 1 && p.n <= MAX_N && p.kt >= 1 && p.kt <= p.n && p.a && p.d && p.e && p.tau && p.w && p.z;
}

size_t batched_offset(int32_t count, const reno_heev_problem* probs, int upto) {
  size_t off = 0;
  for (int i = 0; i < upto && i < count; ++i) off += align256(heev_layout(probs[i].n, probs[i].kt).total);
  return off;
}

}  // namespace

// The reflector rows of v are written in place of the upper triangle of A,
// so A must be a private copy of G.
extern "C" int reno_heev_top(reno_ctx* ctx, int32_t n, int32_t kt, void* A, double* d, double* e, void* tau,
                             double* w, double* Z, void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (n < 1 || n > MAX_N || kt < 1 || kt > n)
    return set_error(ctx, RENO_ERR_INVALID, "reno_heev_top: need 1 <= kt <= n <= 4096");
  if (!A || !d || !e || !tau || !w || !Z || !ws) return set_error(ctx, RENO_ERR_INVALID, "reno_heev_top: null pointer");
  const HeevLayout L = heev_layout(n, kt);
  if (ws_bytes < L.total) return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heev_top: workspace too small");
  char* base = static_cast<char*>(ws);
  Sync* sync = reinterpret_cast<Sync*>(base + L.sync);
  double2* Y = reinterpret_cast<double2*>(base + L.y);
  double2* P = reinterpret_cast<double2*>(base + L.p);
  double* bnd = reinterpret_cast<double*>(base + L.bnd);
  double* scr = reinterpret_cast<double*>(base + L.scr);
  int rc = check_cuda(ctx, cudaMemsetAsync(sync, 0, sizeof(Sync), ctx->stream), "reno_heev_top: memset");
  if (rc == RENO_OK) rc = heev_attrs(ctx);
  if (rc != RENO_OK) return rc;
  EigTable et{};
  et.count = 1;
  et.p[0] = EigProb{static_cast<double2*>(A), static_cast<double2*>(tau), d, e, n, kt, w, Z, bnd, scr};
  if (n <= NMAX_C) {
    rc = heev_reduce_small(ctx, et, n);
  } else {
    HetrdTable tab{};
    tab.count = 1;
    tab.p[0] = HetrdProb{static_cast<double2*>(A), n, d, e, static_cast<double2*>(tau), Y, P, sync, 0, 0,
                         reinterpret_cast<double2*>(base + L.yp)};
    rc = launch_hetrd(ctx, tab, n, "reno_heev_top");
  }
  if (rc != RENO_OK) return rc;
  return heev_eig(ctx, et);
}

extern "C" int reno_heev_batched_workspace_bytes(int32_t count, const reno_heev_problem* probs, size_t* bytes) {
  if (!bytes || !probs || count < 1 || count > RENO_HEEV_MAX_BATCH) return RENO_ERR_INVALID;
  for (int i = 0; i < count; ++i)
    if (probs[i].n < 1 || probs[i].n > MAX_N || probs[i].kt < 1 || probs[i].kt > probs[i].n) return RENO_ERR_INVALID;
  *bytes = batched_offset(count, probs, count);
  return RENO_OK;
}

// reno_heev_top for several matrices: the matrices larger than the cluster
// path share one cooperative reduction launch (the grid split among them),
// so the QN blocks of one bond are reduced side by side.
extern "C" int reno_heev_top_batched(reno_ctx* ctx, int32_t count, const reno_heev_problem* probs, int32_t* status,
                                     void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!probs || !status || !ws || count < 1 || count > RENO_HEEV_MAX_BATCH)
    return set_error(ctx, RENO_ERR_INVALID, "reno_heev_top_batched: invalid batch");
  for (int i = 0; i < count; ++i)
    if (!heev_problem_ok(probs[i]))
      return set_error(ctx, RENO_ERR_INVALID, "reno_heev_top_batched: problem " + std::to_string(i) +
                                                  " needs 1 <= kt <= n <= 4096 and non-null pointers");
  if (ws_bytes < batched_offset(count, probs, count))
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heev_top_batched: workspace too small");
  int rc = heev_attrs(ctx);
  if (rc != RENO_OK) return rc;
  HetrdTable tab{};
  EigTable small{}, all{};
  int nmax = 0, nsmall = 1;
  for (int i = 0; i < count; ++i) {
    const reno_heev_problem& p = probs[i];
    char* base = static_cast<char*>(ws) + batched_offset(count, probs, i);
    const HeevLayout L = heev_layout(p.n, p.kt);
    Sync* sync = reinterpret_cast<Sync*>(base + L.sync);
    rc = check_cuda(ctx, cudaMemsetAsync(sync, 0, sizeof(Sync), ctx->stream), "reno_heev_top_batched: memset");
    if (rc != RENO_OK) return rc;
    const EigProb ep{static_cast<double2*>(p.a), static_cast<double2*>(p.tau), p.d, p.e, p.n, p.kt, p.w, p.z,
                     reinterpret_cast<double*>(base + L.bnd), reinterpret_cast<double*>(base + L.scr)};
    all.p[all.count++] = ep;
    if (p.n <= NMAX_C) {
      small.p[small.count++] = ep;
      nsmall = std::max(nsmall, (int)p.n);
    } else {
      tab.p[tab.count++] = HetrdProb{static_cast<double2*>(p.a), p.n, p.d, p.e, static_cast<double2*>(p.tau),
                                     reinterpret_cast<double2*>(base + L.y), reinterpret_cast<double2*>(base + L.p),
                                     sync, 0, 0, reinterpret_cast<double2*>(base + L.yp)};
      nmax = std::max(nmax, (int)p.n);
    }
  }
  rc = heev_reduce_small(ctx, small, nsmall);
  if (rc != RENO_OK) return rc;
  if (tab.count) {
    rc = launch_hetrd(ctx, tab, nmax, "reno_heev_top_batched");
    if (rc != RENO_OK) return rc;
  }
  rc = heev_eig(ctx, all);
  if (rc != RENO_OK) return rc;
  for (int i = 0; i < count; ++i) {
    char* base = static_cast<char*>(ws) + batched_offset(count, probs, i);
    const HeevLayout L = heev_layout(probs[i].n, probs[i].kt);
    rc = check_cuda(ctx, cudaMemcpyAsync(status + i, base + L.sync + offsetof(Sync, status), sizeof(int32_t),
                                         cudaMemcpyDeviceToDevice, ctx->stream),
                    "reno_heev_top_batched: status");
    if (rc != RENO_OK) return rc;
  }
  return RENO_OK;
}

// K (n x kt complex128, in: eigenvectors of T, out: Q K) after reno_heev_top
// on the same A, tau and workspace; A's reflector rows are cleaned in place.
extern "C" int reno_heev_backtransform(reno_ctx* ctx, int32_t n, int32_t kt, void* A, const void* tau, void* K,
                                       void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (n < 1 || n > MAX_N || kt < 1 || kt > n || !A || !tau || !K || !ws)
    return set_error(ctx, RENO_ERR_INVALID, "reno_heev_backtransform: invalid arguments");
  const HeevLayout L = heev_layout(n, kt);
  if (ws_bytes < L.total) return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heev_backtransform: workspace too small");
  if (n == 1) return RENO_OK;
  char* base = static_cast<char*>(ws);
  double2* Sg = reinterpret_cast<double2*>(base + L.s);
  double2* Tg = reinterpret_cast<double2*>(base + L.t);
  double2* W1 = reinterpret_cast<double2*>(base + L.w1);
  double2* W2 = reinterpret_cast<double2*>(base + L.w2);
  double2* V = static_cast<double2*>(A);
  double2* Kc = static_cast<double2*>(K);
  cudaStream_t st = ctx->stream;
  const int nblk = (int)ceil_div(n - 1, NB);
  const int rep = nch_max(n);
  const size_t nel = (size_t)n * n;
  count_launch();
  clean_v_kernel<<<(unsigned)ceil_div((int64_t)nel, 256), 256, 0, st>>>(V, n);
  RENO_LAUNCH_CHECK(ctx, "reno_heev_backtransform: clean");
  int rc = check_cuda(ctx, cudaMemsetAsync(Sg, 0, (size_t)nblk * NB * NB * sizeof(double2), st),
                      "reno_heev_backtransform: memset");
  if (rc != RENO_OK) return rc;
  // S_b = V_b^H V_b: the blocks of NB reflectors in one batched GEMM over all
  // n columns (zeros before each row's reflector), a partial last block apart
  const int nfull = (n - 1) / NB;
  if (nfull > 0) {
    GemmParams p;
    p.M = NB;
    p.N = NB;
    p.K = n;
    p.batch = nfull;
    p.A = op(V, n, 1, 1);
    p.A.s_batch = (int64_t)NB * n;
    p.B = op(V, n, 1, 0);
    p.B.s_batch = (int64_t)NB * n;
    p.C = Sg;
    p.sCm = NB;
    p.sCn = 1;
    p.sCb = (int64_t)NB * NB;
    count_launch();
    rc = check_cuda(ctx, gemm_fp64(p, st), "reno_heev_backtransform: gram");
    if (rc != RENO_OK) return rc;
  }
  if (nfull < nblk) {
    const int k0 = nfull * NB, kb = n - 1 - k0;
    GemmParams p;
    p.M = kb;
    p.N = kb;
    p.K = n;
    p.A = op(V + (size_t)k0 * n, n, 1, 1);
    p.B = op(V + (size_t)k0 * n, n, 1, 0);
    p.C = Sg + (size_t)nfull * NB * NB;
    p.sCm = NB;
    p.sCn = 1;
    count_launch();
    rc = check_cuda(ctx, gemm_fp64(p, st), "reno_heev_backtransform: gram (last block)");
    if (rc != RENO_OK) return rc;
  }
  count_launch();
  larft_kernel<<<nblk, NB, 0, st>>>(Sg, static_cast<const double2*>(tau), Tg, n, rep);
  RENO_LAUNCH_CHECK(ctx, "reno_heev_backtransform: larft");
  for (int b = nblk - 1; b >= 0; --b) {
    const int k0 = b * NB, kb = std::min(NB, n - 1 - k0);
    const int rows = n - k0 - 1;
    const int nfc = rows / KCH, rem = rows % KCH, nch = nfc + (rem > 0);
    const double2* Vb = V + (size_t)k0 * n + k0 + 1;
    double2* Kb = Kc + (size_t)(k0 + 1) * kt;
    if (kb < NB) {
      rc = check_cuda(ctx, cudaMemsetAsync(W1, 0, (size_t)nch * NB * kt * sizeof(double2), st),
                      "reno_heev_backtransform: memset W1");
      if (rc != RENO_OK) return rc;
    }
    // W1[s] = V_b^H K over row chunk s (split K: one batch entry per full chunk)
    if (nfc > 0) {
      GemmParams p1;
      p1.M = kb;
      p1.N = kt;
      p1.K = KCH;
      p1.batch = nfc;
      p1.A = op(Vb, n, 1, 1);
      p1.A.s_batch = KCH;
      p1.B = op(Kb, 1, kt, 0);
      p1.B.s_batch = (int64_t)KCH * kt;
      p1.C = W1;
      p1.sCm = kt;
      p1.sCn = 1;
      p1.sCb = (int64_t)NB * kt;
      count_launch();
      rc = check_cuda(ctx, gemm_fp64(p1, st), "reno_heev_backtransform: V^H K");
      if (rc != RENO_OK) return rc;
    }
    if (rem > 0) {
      GemmParams p1;
      p1.M = kb;
      p1.N = kt;
      p1.K = rem;
      p1.A = op(Vb + (size_t)nfc * KCH, n, 1, 1);
      p1.B = op(Kb + (size_t)nfc * KCH * kt, 1, kt, 0);
      p1.C = W1 + (size_t)nfc * NB * kt;
      p1.sCm = kt;
      p1.sCn = 1;
      count_launch();
      rc = check_cuda(ctx, gemm_fp64(p1, st), "reno_heev_backtransform: V^H K (last chunk)");
      if (rc != RENO_OK) return rc;
    }
    // W2 = (-T_b) sum_s W1[s]: -T_b replicated along K
    GemmParams p2;
    p2.M = kb;
    p2.N = kt;
    p2.K = NB * nch;
    p2.A = op(Tg + (size_t)b * NB * NB * rep, (int64_t)NB * rep, 1, 0);
    p2.B = op(W1, 1, kt, 0);
    p2.C = W2;
    p2.sCm = kt;
    p2.sCn = 1;
    // K[k0+1:] += V_b W2
    GemmParams p3;
    p3.M = rows;
    p3.N = kt;
    p3.K = kb;
    p3.A = op(Vb, 1, n, 0);
    p3.B = op(W2, 1, kt, 0);
    p3.C = Kb;
    p3.sCm = kt;
    p3.sCn = 1;
    p3.accumulate = 1;
    count_launch(2);
    rc = check_cuda(ctx, gemm_fp64(p2, st), "reno_heev_backtransform: T W");
    if (rc == RENO_OK) rc = check_cuda(ctx, gemm_fp64(p3, st), "reno_heev_backtransform: K += V W");
    if (rc != RENO_OK) return rc;
  }
  return RENO_OK;
}

// status word of the last reno_heev_top on a workspace: the int at this
// byte offset of ws (0 = ok, 1 = a grid barrier timed out)
extern "C" int reno_heev_status_offset(size_t* offset) {
  if (!offset) return RENO_ERR_INVALID;
  *offset = offsetof(Sync, status);
  return RENO_OK;
}

// reno_heev_backtransform for every problem of a reno_heev_top_batched call
// (same problems and workspace): K_i <- Q_i K_i.  The GEMMs of all problems
// run as grouped launches: the Grams of the reflector blocks in one launch,
// then, for the blocks of NB reflectors from the last, one launch each for
// V_b^H K, (-T_b) W1 and K += V_b W2 over every problem that has block b.
extern "C" int reno_heev_backtransform_batched(reno_ctx* ctx, int32_t count, const reno_heev_problem* probs,
                                               void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!probs || !ws || count < 1 || count > RENO_HEEV_MAX_BATCH)
    return set_error(ctx, RENO_ERR_INVALID, "reno_heev_backtransform_batched: invalid batch");
  if (ws_bytes < batched_offset(count, probs, count))
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heev_backtransform_batched: workspace too small");
  cudaStream_t st = ctx->stream;
  struct One {
    int n, kt, nblk, rep;
    double2 *V, *K, *Sg, *Tg, *W1, *W2;
    const double2* tau;
  };
  std::vector<One> P;
  int rc = RENO_OK;
  static_assert(2 * RENO_HEEV_MAX_BATCH < fp64gemm::MAX_GROUP, "one block step of a batch fits one group");
  auto flush = [&](fp64gemm::GemmGroup& g, const char* what) -> int {
    if (g.count == 0) return RENO_OK;
    const int r = check_cuda(ctx, gemm_fp64_grouped(g, st), what);
    g.count = 0;
    return r;
  };
  auto add = [&](fp64gemm::GemmGroup& g, const GemmParams& q, const char* what) -> int {
    g.p[g.count++] = q;
    return g.count == fp64gemm::MAX_GROUP ? flush(g, what) : RENO_OK;
  };
  for (int i = 0; i < count; ++i) {
    const reno_heev_problem& p = probs[i];
    if (!p.k || !p.a || !p.tau) return set_error(ctx, RENO_ERR_INVALID, "reno_heev_backtransform_batched: null");
    if (p.n < 2) continue;
    char* base = static_cast<char*>(ws) + batched_offset(count, probs, i);
    const HeevLayout L = heev_layout(p.n, p.kt);
    One o{p.n, p.kt, (int)ceil_div(p.n - 1, NB), nch_max(p.n), static_cast<double2*>(p.a),
          static_cast<double2*>(p.k), reinterpret_cast<double2*>(base + L.s), reinterpret_cast<double2*>(base + L.t),
          reinterpret_cast<double2*>(base + L.w1), reinterpret_cast<double2*>(base + L.w2),
          static_cast<const double2*>(p.tau)};
    count_launch();
    clean_v_kernel<<<(unsigned)ceil_div((int64_t)o.n * o.n, 256), 256, 0, st>>>(o.V, o.n);
    RENO_LAUNCH_CHECK(ctx, "reno_heev_backtransform_batched: clean");
    rc = check_cuda(ctx, cudaMemsetAsync(o.Sg, 0, (size_t)o.nblk * NB * NB * sizeof(double2), st),
                    "reno_heev_backtransform_batched: memset");
    if (rc != RENO_OK) return rc;
    P.push_back(o);
  }
  if (P.empty()) return RENO_OK;
  // S_b = V_b^H V_b of every problem (full blocks batched, the partial last block apart)
  fp64gemm::GemmGroup g1, g2, g3;
  for (const One& o : P) {
    const int nfull = (o.n - 1) / NB;
    if (nfull > 0) {
      GemmParams q;
      q.M = NB;
      q.N = NB;
      q.K = o.n;
      q.batch = nfull;
      q.A = op(o.V, o.n, 1, 1);
      q.A.s_batch = (int64_t)NB * o.n;
      q.B = op(o.V, o.n, 1, 0);
      q.B.s_batch = (int64_t)NB * o.n;
      q.C = o.Sg;
      q.sCm = NB;
      q.sCn = 1;
      q.sCb = (int64_t)NB * NB;
      if ((rc = add(g1, q, "reno_heev_backtransform_batched: gram")) != RENO_OK) return rc;
    }
    if (nfull < o.nblk) {
      const int k0 = nfull * NB, kb = o.n - 1 - k0;
      GemmParams q;
      q.M = kb;
      q.N = kb;
      q.K = o.n;
      q.A = op(o.V + (size_t)k0 * o.n, o.n, 1, 1);
      q.B = op(o.V + (size_t)k0 * o.n, o.n, 1, 0);
      q.C = o.Sg + (size_t)nfull * NB * NB;
      q.sCm = NB;
      q.sCn = 1;
      if ((rc = add(g1, q, "reno_heev_backtransform_batched: gram")) != RENO_OK) return rc;
    }
  }
  if ((rc = flush(g1, "reno_heev_backtransform_batched: gram")) != RENO_OK) return rc;
  int bmax = 0;
  for (const One& o : P) {
    count_launch();
    larft_kernel<<<o.nblk, NB, 0, st>>>(o.Sg, o.tau, o.Tg, o.n, o.rep);
    RENO_LAUNCH_CHECK(ctx, "reno_heev_backtransform_batched: larft");
    bmax = std::max(bmax, o.nblk);
  }
  // blocks of reflectors from the last: every problem with block b advances together
  for (int b = bmax - 1; b >= 0; --b) {
    for (const One& o : P) {
      if (b >= o.nblk) continue;
      const int k0 = b * NB, kb = std::min(NB, o.n - 1 - k0);
      const int rows = o.n - k0 - 1;
      const int nfc = rows / KCH, rem = rows % KCH, nch = nfc + (rem > 0);
      const double2* Vb = o.V + (size_t)k0 * o.n + k0 + 1;
      double2* Kb = o.K + (size_t)(k0 + 1) * o.kt;
      if (kb < NB) {
        rc = check_cuda(ctx, cudaMemsetAsync(o.W1, 0, (size_t)nch * NB * o.kt * sizeof(double2), st),
                        "reno_heev_backtransform_batched: memset W1");
        if (rc != RENO_OK) return rc;
      }
      if (nfc > 0) {  // W1[s] = V_b^H K over row chunk s
        GemmParams q;
        q.M = kb;
        q.N = o.kt;
        q.K = KCH;
        q.batch = nfc;
        q.A = op(Vb, o.n, 1, 1);
        q.A.s_batch = KCH;
        q.B = op(Kb, 1, o.kt, 0);
        q.B.s_batch = (int64_t)KCH * o.kt;
        q.C = o.W1;
        q.sCm = o.kt;
        q.sCn = 1;
        q.sCb = (int64_t)NB * o.kt;
        if ((rc = add(g1, q, "reno_heev_backtransform_batched: V^H K")) != RENO_OK) return rc;
      }
      if (rem > 0) {
        GemmParams q;
        q.M = kb;
        q.N = o.kt;
        q.K = rem;
        q.A = op(Vb + (size_t)nfc * KCH, o.n, 1, 1);
        q.B = op(Kb + (size_t)nfc * KCH * o.kt, 1, o.kt, 0);
        q.C = o.W1 + (size_t)nfc * NB * o.kt;
        q.sCm = o.kt;
        q.sCn = 1;
        if ((rc = add(g1, q, "reno_heev_backtransform_batched: V^H K")) != RENO_OK) return rc;
      }
      GemmParams q2;  // W2 = (-T_b) sum_s W1[s]
      q2.M = kb;
      q2.N = o.kt;
      q2.K = NB * nch;
      q2.A = op(o.Tg + (size_t)b * NB * NB * o.rep, (int64_t)NB * o.rep, 1, 0);
      q2.B = op(o.W1, 1, o.kt, 0);
      q2.C = o.W2;
      q2.sCm = o.kt;
      q2.sCn = 1;
      if ((rc = add(g2, q2, "reno_heev_backtransform_batched: T W")) != RENO_OK) return rc;
      GemmParams q3;  // K[k0+1:] += V_b W2
      q3.M = rows;
      q3.N = o.kt;
      q3.K = kb;
      q3.A = op(Vb, 1, o.n, 0);
      q3.B = op(o.W2, 1, o.kt, 0);
      q3.C = Kb;
      q3.sCm = o.kt;
      q3.sCn = 1;
      q3.accumulate = 1;
      if ((rc = add(g3, q3, "reno_heev_backtransform_batched: K += V W")) != RENO_OK) return rc;
    }
    if ((rc = flush(g1, "reno_heev_backtransform_batched: V^H K")) != RENO_OK) return rc;
    if ((rc = flush(g2, "reno_heev_backtransform_batched: T W")) != RENO_OK) return rc;
    if ((rc = flush(g3, "reno_heev_backtransform_batched: K += V W")) != RENO_OK) return rc;
  }
  return RENO_OK;
}
