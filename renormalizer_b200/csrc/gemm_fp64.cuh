// Strided batched FP64 GEMM on the sm_100a double-precision MMA pipe
// (mma.sync m8n8k4 .f64), complex handled as four real products.
//
//   C[b][m][n] (+)= sum_k opA(A)[b][m][k] * opB(B)[b][k][n]
//
// Every stage of the H_eff matvec and of the environment update is one call
// of this kernel with the strides of the reference's C-order tensors, so no
// operand is ever permuted in HBM (hop_expr.py:57-103, lib.py:200-237).
// Operands are staged global -> shared with cp.async (zero-filled tails) in a
// 3-stage ring; each warp owns a 32x32 output tile = 4x4 m8n8 fragments.
#pragma once
#include <algorithm>
#include <type_traits>
#include "reno_common.cuh"

namespace reno {

struct GemmOperand {
  const void* ptr = nullptr;
  int64_t s_outer = 0;  // stride of the M (A) or N (B) index, in elements
  int64_t s_k = 0;      // stride of the K index
  int64_t s_batch = 0;
  int is_complex = 0;
  int conj = 0;
  int is_f32 = 0;       // elements are float / float2 (split-precision intermediates only)
};

struct GemmParams {
  int M = 0, N = 0, K = 0, batch = 1;
  GemmOperand A, B;
  void* C = nullptr;
  int64_t sCm = 0, sCn = 0, sCb = 0;
  int accumulate = 0;
  int c_f32 = 0;        // C is float / float2 (split-precision intermediates only)
};

namespace fp64gemm {

constexpr int BM = 64, BN = 64, BK = 16, BKP = BK + 4, STAGES = 3, THREADS = 128;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* dst, const void* src, bool valid) {
  const int src_bytes = valid ? BYTES : 0;
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(src_bytes));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(src_bytes));
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Copy one BM(or BN) x BK tile of an operand into shared memory laid out
// [outer][k] with row pitch BKP.  Thread->element mapping follows whichever
// global index is unit-stride so that the global reads coalesce.
template <bool CPLX>
__device__ __forceinline__ void load_tile(void* smem, const GemmOperand& op, const char* base,
                                          int outer0, int outer_max, int k0, int K, int tid) {
  using T = typename std::conditional<CPLX, double2, double>::type;
  T* s = reinterpret_cast<T*>(smem);
  const T* g = reinterpret_cast<const T*>(base);
  constexpr int ELEMS = BM * BK / THREADS;
  const bool k_fast = (op.s_k == 1);
#pragma unroll
  for (int i = 0; i < ELEMS; ++i) {
    const int idx = tid + i * THREADS;
    int o, k;
    if (k_fast) {
      k = idx % BK;
      o = idx / BK;
    } else {
      o = idx % BM;
      k = idx / BM;
    }
    const int go = outer0 + o, gk = k0 + k;
    const bool valid = (go < outer_max) && (gk < K);
    const T* src = valid ? g + (int64_t)go * op.s_outer + (int64_t)gk * op.s_k : g;
    cp_async_zfill<sizeof(T)>(s + o * BKP + k, src, valid);
  }
}

// one BM x BN output tile (tile column bx, tile row by, batch entry bz) of p
template <bool AC, bool BC>
__device__ __forceinline__ void gemm_tile(const GemmParams& p, int bx, int by, int bz) {
  constexpr bool CC = AC || BC;
  using TA = typename std::conditional<AC, double2, double>::type;
  using TB = typename std::conditional<BC, double2, double>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TA* sA = reinterpret_cast<TA*>(smem_raw);
  TB* sB = reinterpret_cast<TB*>(smem_raw + STAGES * BM * BKP * sizeof(TA));

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp & 1) * 32, wn0 = (warp >> 1) * 32;
  const int m0 = by * BM, n0 = bx * BN;
  const int64_t b = bz;
  const char* baseA = reinterpret_cast<const char*>(p.A.ptr) + b * p.A.s_batch * sizeof(TA);
  const char* baseB = reinterpret_cast<const char*>(p.B.ptr) + b * p.B.s_batch * sizeof(TB);

  double accr[4][4][2], acci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      accr[i][j][0] = accr[i][j][1] = 0.0;
      acci[i][j][0] = acci[i][j][1] = 0.0;
    }

  const int nk = (int)ceil_div(p.K, BK);
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) {
      load_tile<AC>(sA + s * BM * BKP, p.A, baseA, m0, p.M, s * BK, p.K, tid);
      load_tile<BC>(sB + s * BN * BKP, p.B, baseB, n0, p.N, s * BK, p.K, tid);
    }
    cp_async_commit();
  }

  const double sgnA = p.A.conj ? -1.0 : 1.0, sgnB = p.B.conj ? -1.0 : 1.0;
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const TA* a_s = sA + (kt % STAGES) * BM * BKP;
    const TB* b_s = sB + (kt % STAGES) * BN * BKP;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[4], ai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const TA va = a_s[(wm0 + i * 8 + (lane >> 2)) * BKP + kk + (lane & 3)];
        if constexpr (AC) {
          ar[i] = va.x;
          ai[i] = sgnA * va.y;
        } else {
          ar[i] = va;
          ai[i] = 0.0;
        }
        const TB vb = b_s[(wn0 + i * 8 + (lane >> 2)) * BKP + kk + (lane & 3)];
        if constexpr (BC) {
          br[i] = vb.x;
          bi[i] = sgnB * vb.y;
        } else {
          br[i] = vb;
          bi[i] = 0.0;
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
          if constexpr (AC && BC) dmma(accr[i][j][0], accr[i][j][1], -ai[i], bi[j]);
          if constexpr (BC) dmma(acci[i][j][0], acci[i][j][1], ar[i], bi[j]);
          if constexpr (AC) dmma(acci[i][j][0], acci[i][j][1], ai[i], br[j]);
        }
      }
    }
    const int ks = kt + STAGES - 1;
    if (ks < nk) {
      load_tile<AC>(sA + (ks % STAGES) * BM * BKP, p.A, baseA, m0, p.M, ks * BK, p.K, tid);
      load_tile<BC>(sB + (ks % STAGES) * BN * BKP, p.B, baseB, n0, p.N, ks * BK, p.K, tid);
    }
    cp_async_commit();
  }
  cp_async_wait<0>();

  // epilogue: fragment (i,j) element e sits at row lane/4, column 2*(lane%4)+e
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + wm0 + i * 8 + (lane >> 2);
    if (m >= p.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int n = n0 + wn0 + j * 8 + (lane & 3) * 2 + e;
        if (n >= p.N) continue;
        const int64_t off = b * p.sCb + (int64_t)m * p.sCm + (int64_t)n * p.sCn;
        if constexpr (CC) {
          double2* c = reinterpret_cast<double2*>(p.C) + off;
          double2 v = make_double2(accr[i][j][e], acci[i][j][e]);
          if (p.accumulate) {
            const double2 o = *c;
            v.x += o.x;
            v.y += o.y;
          }
          *c = v;
        } else {
          double* c = reinterpret_cast<double*>(p.C) + off;
          double v = accr[i][j][e];
          if (p.accumulate) v += *c;
          *c = v;
        }
      }
    }
  }
}

template <bool AC, bool BC>
__global__ void __launch_bounds__(THREADS) gemm_kernel(GemmParams p) {
  gemm_tile<AC, BC>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Many independent GEMMs (same operand types) in one launch: CTA t runs tile
// t - first[i] of problem i, first[i] <= t < first[i + 1], tiles of a problem
// numbered like the single launch's grid (x fastest, then y, then batch).
constexpr int MAX_GROUP = 128;
struct GemmGroup {
  int count = 0;
  int first[MAX_GROUP + 1] = {};
  GemmParams p[MAX_GROUP];
};

template <bool AC, bool BC>
__global__ void __launch_bounds__(THREADS) gemm_grouped_kernel(const __grid_constant__ GemmGroup g) {
  const int t = blockIdx.x;
  int lo = 0, hi = g.count;  // first[lo] <= t < first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (g.first[mid] <= t) lo = mid;
    else hi = mid;
  }
  const GemmParams& p = g.p[lo];
  const int lt = t - g.first[lo];
  const int nx = (int)ceil_div(p.N, BN), ny = (int)ceil_div(p.M, BM);
  gemm_tile<AC, BC>(p, lt % nx, (lt / nx) % ny, lt / (nx * ny));
}

template <bool AC, bool BC>
inline size_t smem_bytes() {
  return STAGES * (BM * BKP * (AC ? 16 : 8) + BN * BKP * (BC ? 16 : 8));
}

template <bool AC, bool BC>
inline cudaError_t launch_t(const GemmParams& p, cudaStream_t st) {
  const size_t sm = smem_bytes<AC, BC>();
  static std::atomic<unsigned long long> smem_set{0};
  {
    cudaError_t e = smem_optin_once(gemm_kernel<AC, BC>, (int)sm, smem_set);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)ceil_div(p.N, BN), (unsigned)ceil_div(p.M, BM), (unsigned)p.batch);
  count_launch();
  gemm_kernel<AC, BC><<<grid, THREADS, sm, st>>>(p);
  return cudaGetLastError();
}

template <bool AC, bool BC>
inline cudaError_t launch_grouped_t(const GemmGroup& g, cudaStream_t st) {
  const size_t sm = smem_bytes<AC, BC>();
  static std::atomic<unsigned long long> smem_set{0};
  {
    cudaError_t e = smem_optin_once(gemm_grouped_kernel<AC, BC>, (int)sm, smem_set);
    if (e != cudaSuccess) return e;
  }
  if (g.first[g.count] == 0) return cudaSuccess;
  count_launch();
  gemm_grouped_kernel<AC, BC><<<g.first[g.count], THREADS, sm, st>>>(g);
  return cudaGetLastError();
}

}  // namespace fp64gemm

// Launch a group of FP64 GEMMs whose operands all have the same types (tile
// counts filled in here); returns a CUDA error code.
inline cudaError_t gemm_fp64_grouped(fp64gemm::GemmGroup& g, cudaStream_t st) {
  if (g.count < 1 || g.count > fp64gemm::MAX_GROUP) return cudaErrorInvalidValue;
  const bool ac = g.p[0].A.is_complex, bc = g.p[0].B.is_complex;
  g.first[0] = 0;
  for (int i = 0; i < g.count; ++i) {
    const GemmParams& p = g.p[i];
    if (p.A.is_f32 || p.B.is_f32 || p.c_f32 || (bool)p.A.is_complex != ac || (bool)p.B.is_complex != bc)
      return cudaErrorInvalidValue;
    const int64_t tiles = (p.M > 0 && p.N > 0 && p.batch > 0)
                              ? ceil_div(p.N, fp64gemm::BN) * ceil_div(p.M, fp64gemm::BM) * p.batch
                              : 0;
    if (g.first[i] + tiles > 0x7fffffff) return cudaErrorInvalidValue;
    g.first[i + 1] = g.first[i] + (int)tiles;
  }
  if (ac && bc) return fp64gemm::launch_grouped_t<true, true>(g, st);
  if (ac) return fp64gemm::launch_grouped_t<true, false>(g, st);
  if (bc) return fp64gemm::launch_grouped_t<false, true>(g, st);
  return fp64gemm::launch_grouped_t<false, false>(g, st);
}

namespace fp64gemm {

// Split-K for groups whose output tiles alone cannot fill the GPU (a few
// rows by a few hundred columns summed over thousands of rows, as in the
// V^H C products of blocked Householder QR): each such product is cut into
// S chunks of its K range, the chunks run as separate group entries into
// partial buffers, and one reduction launch sums the partials in chunk order
// (deterministic), adding the old C when the product accumulates.
constexpr int SPLITK_MAX = 16;
constexpr int SPLITK_CHUNK = 256;  // smallest K range of a chunk

struct SplitReduce {
  int count;
  struct Entry {
    void* C;
    const void* part;
    int M, N, batch, S;
    int64_t sCm, sCn, sCb;
    int accumulate;
  } e[MAX_GROUP];
};

template <bool CC>
__global__ void splitk_reduce_kernel(const __grid_constant__ SplitReduce r) {
  using T = typename std::conditional<CC, double2, double>::type;
  const SplitReduce::Entry& E = r.e[blockIdx.y];
  const int64_t n = (int64_t)E.M * E.N * E.batch;
  const T* part = reinterpret_cast<const T*>(E.part);
  T* C = reinterpret_cast<T*>(E.C);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int nn = (int)(i % E.N);
    const int64_t rest = i / E.N;
    const int m = (int)(rest % E.M);
    const int64_t b = rest / E.M;
    T acc = part[i];
    for (int s = 1; s < E.S; ++s) {
      const T x = part[(int64_t)s * n + i];
      if constexpr (CC) {
        acc.x += x.x;
        acc.y += x.y;
      } else {
        acc += x;
      }
    }
    T* c = C + b * E.sCb + (int64_t)m * E.sCm + (int64_t)nn * E.sCn;
    if (E.accumulate) {
      if constexpr (CC) {
        acc.x += c->x;
        acc.y += c->y;
      } else {
        acc += *c;
      }
    }
    *c = acc;
  }
}

// chunks per entry (1 = unsplit); returns the partial-buffer bytes
inline size_t splitk_plan(const GemmGroup& g, int target_ctas, int* S) {
  int64_t tiles = 0;
  for (int i = 0; i < g.count; ++i) {
    const GemmParams& p = g.p[i];
    tiles += (p.M > 0 && p.N > 0) ? ceil_div(p.N, BN) * ceil_div(p.M, BM) * p.batch : 0;
  }
  const int want = tiles > 0 ? (int)std::min<int64_t>(SPLITK_MAX, ceil_div(target_ctas, tiles)) : 1;
  for (int cap = want;; cap = std::max(1, cap / 2)) {
    int total = 0;
    for (int i = 0; i < g.count; ++i) {
      const GemmParams& p = g.p[i];
      S[i] = (p.M > 0 && p.N > 0 && tiles < target_ctas) ? std::max(1, std::min(cap, p.K / SPLITK_CHUNK)) : 1;
      total += S[i];
    }
    if (total <= MAX_GROUP || cap == 1) break;
  }
  size_t bytes = 0;
  for (int i = 0; i < g.count; ++i) {
    const GemmParams& p = g.p[i];
    const size_t es = (p.A.is_complex || p.B.is_complex) ? 16 : 8;
    if (S[i] > 1) bytes += (size_t)S[i] * p.M * p.N * p.batch * es;
  }
  return bytes;
}

// upper bound of splitk_plan's bytes for a group of `count` entries of at most
// M x N x batch outputs
inline size_t splitk_bytes_bound(int count, int64_t mn_batch, bool complex_out) {
  return (size_t)count * SPLITK_MAX * (size_t)mn_batch * (complex_out ? 16 : 8);
}

}  // namespace fp64gemm

// gemm_fp64_grouped with split-K where the group's output tiles are fewer
// than about two per SM; ws holds the partials (fp64gemm::splitk_plan bytes).
inline cudaError_t gemm_fp64_grouped_splitk(fp64gemm::GemmGroup& g, void* ws, size_t ws_bytes, cudaStream_t st) {
  using namespace fp64gemm;
  if (g.count < 1 || g.count > MAX_GROUP) return cudaErrorInvalidValue;
  int S[MAX_GROUP];
  const size_t need = splitk_plan(g, 2 * sm_count_current_device(), S);
  bool any = false;
  for (int i = 0; i < g.count; ++i) any = any || S[i] > 1;
  if (!any) return gemm_fp64_grouped(g, st);
  if (need > ws_bytes || !ws) return cudaErrorInvalidValue;
  GemmGroup x;
  SplitReduce red{};
  char* part = reinterpret_cast<char*>(ws);
  const bool cc = g.p[0].A.is_complex || g.p[0].B.is_complex;
  for (int i = 0; i < g.count; ++i) {
    const GemmParams& p = g.p[i];
    if (S[i] == 1) {
      x.p[x.count++] = p;
      continue;
    }
    const size_t esA = p.A.is_complex ? 16 : 8, esB = p.B.is_complex ? 16 : 8, esC = cc ? 16 : 8;
    const int kc = (int)ceil_div(p.K, S[i]);
    const int64_t n = (int64_t)p.M * p.N * p.batch;
    int used = 0;
    for (int s = 0; s < S[i]; ++s) {
      const int k0 = s * kc, k1 = std::min(p.K, k0 + kc);
      GemmParams q = p;
      q.K = std::max(0, k1 - k0);
      q.A.ptr = reinterpret_cast<const char*>(p.A.ptr) + (int64_t)k0 * p.A.s_k * (int64_t)esA;
      q.B.ptr = reinterpret_cast<const char*>(p.B.ptr) + (int64_t)k0 * p.B.s_k * (int64_t)esB;
      q.C = part + (size_t)s * n * esC;
      q.sCm = p.N;
      q.sCn = 1;
      q.sCb = (int64_t)p.M * p.N;
      q.accumulate = 0;
      x.p[x.count++] = q;
      ++used;
    }
    SplitReduce::Entry& e = red.e[red.count++];
    e.C = p.C;
    e.part = part;
    e.M = p.M;
    e.N = p.N;
    e.batch = p.batch;
    e.S = used;
    e.sCm = p.sCm;
    e.sCn = p.sCn;
    e.sCb = p.sCb;
    e.accumulate = p.accumulate;
    part += (size_t)used * n * esC;
  }
  cudaError_t err = gemm_fp64_grouped(x, st);
  if (err != cudaSuccess) return err;
  int64_t nmax = 1;
  for (int i = 0; i < red.count; ++i) nmax = std::max<int64_t>(nmax, (int64_t)red.e[i].M * red.e[i].N * red.e[i].batch);
  const unsigned bx = (unsigned)std::min<int64_t>(ceil_div(nmax, 256), 64);
  count_launch();
  if (cc) splitk_reduce_kernel<true><<<dim3(bx, red.count), 256, 0, st>>>(red);
  else splitk_reduce_kernel<false><<<dim3(bx, red.count), 256, 0, st>>>(red);
  return cudaGetLastError();
}

// Launch the FP64 GEMM; returns a CUDA error code.
inline cudaError_t gemm_fp64(const GemmParams& p, cudaStream_t st) {
  if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return cudaSuccess;
  // FP32 operands / outputs exist only between split-precision stages
  if (p.A.is_f32 || p.B.is_f32 || p.c_f32) return cudaErrorInvalidValue;
  const bool ac = p.A.is_complex, bc = p.B.is_complex;
  if (ac && bc) return fp64gemm::launch_t<true, true>(p, st);
  if (ac) return fp64gemm::launch_t<true, false>(p, st);
  if (bc) return fp64gemm::launch_t<false, true>(p, st);
  return fp64gemm::launch_t<false, false>(p, st);
}

}  // namespace reno
