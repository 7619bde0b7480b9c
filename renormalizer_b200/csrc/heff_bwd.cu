// Reverse mode of the effective-Hamiltonian matvec (hop_expr.py:57-103; the
// reference has no gradients) and the general strided tensordot it is built
// from.
//
// For y = H_eff(L, W1[, W2], R) psi, multilinear in its operands, the
// gradient (torch's convention for complex tensors: grad_x = J^H grad_y) with
// respect to each operand is the contraction of gy with the complex
// conjugates of the other operands:
//   d psi : the matvec itself with L'[c,b,a] = conj L[a,b,c],
//           W'[b,e,d,f] = conj W[b,d,e,f], R'[k,f,l] = conj R[l,f,k]
//           applied to gy (reno_heff_apply, any precision)
//   d L, d R, d W1, d W2 : fixed chains of pairwise contractions, each one
//           permute-copy per operand (conjugation folded in) followed by one
//           FP64 DMMA GEMM, and a final permute into the caller's layout.
// Intermediates live in the caller's workspace (bump allocation; the
// workspace query runs the same code without launching anything).
#include "reno_common.cuh"
#include "gemm_fp64.cuh"
#include <algorithm>
#include <vector>

extern "C" int reno_heff_workspace_bytes(const reno_heff_desc* d, size_t* bytes);
extern "C" int reno_heff_apply(reno_ctx* ctx, const reno_heff_desc* d, const void* L, const void* W1,
                               const void* W2, const void* R, const void* psi, void* y, void* ws, size_t ws_bytes);

namespace reno {
namespace bwd {

constexpr int MAXR = 6;

// a strided tensor view: element (i0..ir-1) at p[sum i_k s_k]
struct TView {
  const void* p = nullptr;
  int dt = RENO_F64;
  int r = 0;
  int64_t n[MAXR] = {};
  int64_t s[MAXR] = {};
  int conj = 0;
  int64_t size() const {
    int64_t t = 1;
    for (int k = 0; k < r; ++k) t *= n[k];
    return t;
  }
};

static TView contiguous(const void* p, int dt, std::initializer_list<int64_t> shape, int conj = 0) {
  TView v;
  v.p = p;
  v.dt = dt;
  v.conj = conj;
  for (int64_t x : shape) v.n[v.r++] = x;
  int64_t st = 1;
  for (int k = v.r - 1; k >= 0; --k) {
    v.s[k] = st;
    st *= v.n[k];
  }
  return v;
}

static TView conj_of(TView v) {
  v.conj ^= 1;
  return v;
}

static inline int64_t esz(int dt) { return dt == RENO_C128 ? 16 : 8; }

struct PermArgs {
  const void* src;
  void* dst;
  int src_c, dst_c, conj, r;
  int64_t total;
  int64_t n[MAXR];  // output extents, output axis order
  int64_t s[MAXR];  // source strides of those axes
};

// dst (contiguous, output axis order) = conj?(src permuted), promoted to dst's type
__global__ void permute_kernel(PermArgs a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t rem = i, off = 0;
    for (int k = a.r - 1; k >= 0; --k) {
      const int64_t c = rem % a.n[k];
      rem /= a.n[k];
      off += c * a.s[k];
    }
    double2 v;
    if (a.src_c) {
      v = reinterpret_cast<const double2*>(a.src)[off];
      if (a.conj) v.y = -v.y;
    } else {
      v = make_double2(reinterpret_cast<const double*>(a.src)[off], 0.0);
    }
    if (a.dst_c)
      reinterpret_cast<double2*>(a.dst)[i] = v;
    else
      reinterpret_cast<double*>(a.dst)[i] = v.x;
  }
}

// workspace bump allocator; a null base is the sizing pass
struct Bump {
  char* base;
  size_t off = 0;
  explicit Bump(void* b) : base(static_cast<char*>(b)) {}
  void* take(size_t bytes) {
    const size_t o = (off + 255) & ~size_t(255);
    off = o + bytes;
    return base ? base + o : nullptr;
  }
  bool dry() const { return base == nullptr; }
};

// out (contiguous, dtype out_dt) axis k = src axis perm[k]
static cudaError_t permute_to(const TView& src, const int* perm, void* out, int out_dt, cudaStream_t st) {
  PermArgs a{};
  a.src = src.p;
  a.dst = out;
  a.src_c = src.dt == RENO_C128;
  a.dst_c = out_dt == RENO_C128;
  a.conj = src.conj;
  a.r = src.r;
  a.total = src.size();
  for (int k = 0; k < src.r; ++k) {
    a.n[k] = src.n[perm[k]];
    a.s[k] = src.s[perm[k]];
  }
  if (a.total == 0) return cudaSuccess;
  int64_t g = ceil_div(a.total, 256);
  if (g > 148 * 16) g = 148 * 16;
  count_launch();
  permute_kernel<<<(unsigned)g, 256, 0, st>>>(a);
  return cudaGetLastError();
}

// c[fa..., fb...] = sum over a's axes ia paired with b's axes ib; contiguous
// output in ws, complex when either operand is
static cudaError_t tensordot(const TView& a, const TView& b, int na, const int* ia, const int* ib, TView& c, Bump& ws,
                             cudaStream_t st) {
  int fa[MAXR], fb[MAXR], nfa = 0, nfb = 0;
  for (int k = 0; k < a.r; ++k)
    if (std::find(ia, ia + na, k) == ia + na) fa[nfa++] = k;
  for (int k = 0; k < b.r; ++k)
    if (std::find(ib, ib + na, k) == ib + na) fb[nfb++] = k;
  int64_t M = 1, N = 1, K = 1;
  for (int k = 0; k < nfa; ++k) M *= a.n[fa[k]];
  for (int k = 0; k < nfb; ++k) N *= b.n[fb[k]];
  for (int k = 0; k < na; ++k) {
    if (a.n[ia[k]] != b.n[ib[k]]) return cudaErrorInvalidValue;
    K *= a.n[ia[k]];
  }
  int pa[MAXR], pb[MAXR];
  for (int k = 0; k < nfa; ++k) pa[k] = fa[k];
  for (int k = 0; k < na; ++k) pa[nfa + k] = ia[k];
  for (int k = 0; k < na; ++k) pb[k] = ib[k];
  for (int k = 0; k < nfb; ++k) pb[na + k] = fb[k];
  void* A = ws.take((size_t)(M * K) * esz(a.dt));
  void* B = ws.take((size_t)(K * N) * esz(b.dt));
  const int cdt = (a.dt == RENO_C128 || b.dt == RENO_C128) ? RENO_C128 : RENO_F64;
  void* C = ws.take((size_t)(M * N) * esz(cdt));
  c = TView{};
  c.p = C;
  c.dt = cdt;
  for (int k = 0; k < nfa; ++k) c.n[c.r++] = a.n[fa[k]];
  for (int k = 0; k < nfb; ++k) c.n[c.r++] = b.n[fb[k]];
  int64_t stc = 1;
  for (int k = c.r - 1; k >= 0; --k) {
    c.s[k] = stc;
    stc *= c.n[k];
  }
  if (ws.dry()) return cudaSuccess;
  cudaError_t e = permute_to(a, pa, A, a.dt, st);
  if (e == cudaSuccess) e = permute_to(b, pb, B, b.dt, st);
  if (e != cudaSuccess) return e;
  GemmParams p;
  p.M = (int)M;
  p.N = (int)N;
  p.K = (int)K;
  p.A.ptr = A;
  p.A.is_complex = a.dt == RENO_C128;
  p.A.s_outer = K;
  p.A.s_k = 1;
  p.B.ptr = B;
  p.B.is_complex = b.dt == RENO_C128;
  p.B.s_outer = 1;
  p.B.s_k = N;
  p.C = C;
  p.sCm = N;
  p.sCn = 1;
  return gemm_fp64(p, st);
}

// final permute of a chain result into the caller's buffer
static cudaError_t emit(const TView& src, std::initializer_list<int> perm, void* out, int out_dt, Bump& ws,
                        cudaStream_t st) {
  if (ws.dry() || !out) return cudaSuccess;
  std::vector<int> pv(perm);
  return permute_to(src, pv.data(), out, out_dt, st);
}

struct Ops {
  TView L, W1, W2, R, P, gy;
  int nsite;
};

static cudaError_t grad_L(const Ops& o, void* out, int odt, Bump& ws, cudaStream_t st) {
  TView t, u, v, g;
  const TView cL = conj_of(o.L), cR = conj_of(o.R), cP = conj_of(o.P), cW1 = conj_of(o.W1), cW2 = conj_of(o.W2);
  cudaError_t e;
  (void)cL;
  if (o.nsite == 0) {
    const int a0[] = {1}, b0[] = {2};
    if ((e = tensordot(cP, cR, 1, a0, b0, t, ws, st))) return e;                  // c l b
    const int a1[] = {1}, b1[] = {1};
    if ((e = tensordot(o.gy, t, 1, a1, b1, g, ws, st))) return e;                 // a c b
  } else if (o.nsite == 1) {
    const int a0[] = {2}, b0[] = {2};
    if ((e = tensordot(cP, cR, 1, a0, b0, t, ws, st))) return e;                  // c e l f
    const int a1[] = {1, 3}, b1[] = {2, 3};
    if ((e = tensordot(t, cW1, 2, a1, b1, u, ws, st))) return e;                  // c l b d
    const int a2[] = {1, 2}, b2[] = {3, 1};
    if ((e = tensordot(o.gy, u, 2, a2, b2, g, ws, st))) return e;                 // a c b
  } else {
    const int a0[] = {3}, b0[] = {2};
    if ((e = tensordot(cP, cR, 1, a0, b0, t, ws, st))) return e;                  // c e h l j
    const int a1[] = {2, 4}, b1[] = {2, 3};
    if ((e = tensordot(t, cW2, 2, a1, b1, u, ws, st))) return e;                  // c e l f g
    const int a2[] = {1, 3}, b2[] = {2, 3};
    if ((e = tensordot(u, cW1, 2, a2, b2, v, ws, st))) return e;                  // c l g b d
    const int a3[] = {1, 2, 3}, b3[] = {4, 2, 1};
    if ((e = tensordot(o.gy, v, 3, a3, b3, g, ws, st))) return e;                 // a c b
  }
  return emit(g, {0, 2, 1}, out, odt, ws, st);
}

static cudaError_t grad_R(const Ops& o, void* out, int odt, Bump& ws, cudaStream_t st) {
  TView t, u, v, g;
  const TView cL = conj_of(o.L), cP = conj_of(o.P), cW1 = conj_of(o.W1), cW2 = conj_of(o.W2);
  cudaError_t e;
  if (o.nsite == 0) {
    const int a0[] = {2}, b0[] = {0};
    if ((e = tensordot(cL, cP, 1, a0, b0, t, ws, st))) return e;                  // a b k
    const int a1[] = {0}, b1[] = {0};
    if ((e = tensordot(o.gy, t, 1, a1, b1, g, ws, st))) return e;                 // l b k
    return emit(g, {0, 1, 2}, out, odt, ws, st);
  }
  if (o.nsite == 1) {
    const int a0[] = {2}, b0[] = {0};
    if ((e = tensordot(cL, cP, 1, a0, b0, t, ws, st))) return e;                  // a b e k
    const int a1[] = {1, 2}, b1[] = {0, 2};
    if ((e = tensordot(t, cW1, 2, a1, b1, u, ws, st))) return e;                  // a k d f
    const int a2[] = {0, 1}, b2[] = {0, 2};
    if ((e = tensordot(o.gy, u, 2, a2, b2, g, ws, st))) return e;                 // l k f
  } else {
    const int a0[] = {2}, b0[] = {0};
    if ((e = tensordot(cL, cP, 1, a0, b0, t, ws, st))) return e;                  // a b e h k
    const int a1[] = {1, 2}, b1[] = {0, 2};
    if ((e = tensordot(t, cW1, 2, a1, b1, u, ws, st))) return e;                  // a h k d f
    const int a2[] = {4, 1}, b2[] = {0, 2};
    if ((e = tensordot(u, cW2, 2, a2, b2, v, ws, st))) return e;                  // a k d g j
    const int a3[] = {0, 1, 2}, b3[] = {0, 2, 3};
    if ((e = tensordot(o.gy, v, 3, a3, b3, g, ws, st))) return e;                 // l k j
  }
  return emit(g, {0, 2, 1}, out, odt, ws, st);
}

static cudaError_t grad_W1(const Ops& o, void* out, int odt, Bump& ws, cudaStream_t st) {
  TView t, u, v, g;
  const TView cL = conj_of(o.L), cR = conj_of(o.R), cP = conj_of(o.P), cW2 = conj_of(o.W2);
  cudaError_t e;
  if (o.nsite == 1) {
    const int a0[] = {2}, b0[] = {0};
    if ((e = tensordot(cL, cP, 1, a0, b0, t, ws, st))) return e;                  // a b e k
    const int a1[] = {3}, b1[] = {2};
    if ((e = tensordot(t, cR, 1, a1, b1, u, ws, st))) return e;                   // a b e l f
    const int a2[] = {0, 2}, b2[] = {0, 3};
    if ((e = tensordot(o.gy, u, 2, a2, b2, g, ws, st))) return e;                 // d b e f
    return emit(g, {1, 0, 2, 3}, out, odt, ws, st);
  }
  const int a0[] = {3}, b0[] = {2};
  if ((e = tensordot(cP, cR, 1, a0, b0, t, ws, st))) return e;                    // c e h l j
  const int a1[] = {2, 4}, b1[] = {2, 3};
  if ((e = tensordot(t, cW2, 2, a1, b1, u, ws, st))) return e;                    // c e l f g
  const int a2[] = {0}, b2[] = {2};
  if ((e = tensordot(u, cL, 1, a2, b2, v, ws, st))) return e;                     // e l f g a b
  const int a3[] = {0, 2, 3}, b3[] = {4, 3, 1};
  if ((e = tensordot(o.gy, v, 3, a3, b3, g, ws, st))) return e;                   // d e f b
  return emit(g, {3, 0, 1, 2}, out, odt, ws, st);
}

static cudaError_t grad_W2(const Ops& o, void* out, int odt, Bump& ws, cudaStream_t st) {
  TView t, u, v, g;
  const TView cL = conj_of(o.L), cR = conj_of(o.R), cP = conj_of(o.P), cW1 = conj_of(o.W1);
  cudaError_t e;
  const int a0[] = {2}, b0[] = {0};
  if ((e = tensordot(cL, cP, 1, a0, b0, t, ws, st))) return e;                    // a b e h k
  const int a1[] = {1, 2}, b1[] = {0, 2};
  if ((e = tensordot(t, cW1, 2, a1, b1, u, ws, st))) return e;                    // a h k d f
  const int a2[] = {2}, b2[] = {2};
  if ((e = tensordot(u, cR, 1, a2, b2, v, ws, st))) return e;                     // a h d f l j
  const int a3[] = {0, 1, 3}, b3[] = {0, 2, 4};
  if ((e = tensordot(o.gy, v, 3, a3, b3, g, ws, st))) return e;                   // g h f j
  return emit(g, {2, 0, 1, 3}, out, odt, ws, st);
}

static int promote(int a, int b) { return (a == RENO_C128 || b == RENO_C128) ? RENO_C128 : RENO_F64; }

// the whole backward; ws.dry() sizes the workspace without launching
static int run(reno_ctx* ctx, const reno_heff_desc* d, const void* L, const void* W1, const void* W2, const void* R,
               const void* psi, const void* gy, void* gpsi, void* gL, void* gW1, void* gW2, void* gR, Bump& ws) {
  const int64_t ml = d->ml, mr = d->mr, wl = d->wl, wm = d->wm, wr = d->wr, d1 = d->d1, d2 = d->d2;
  const int n = d->nsite;
  const int ydt = promote(promote(d->env_dtype, d->psi_dtype), n ? d->mpo_dtype : RENO_F64);
  const int gdt = ydt;  // gradients of every operand in the output's type
  cudaStream_t st = ctx ? ctx->stream : nullptr;
  Ops o;
  o.nsite = n;
  o.L = contiguous(L, d->env_dtype, {ml, wl, ml});
  o.R = contiguous(R, d->env_dtype, {mr, wr, mr});
  if (n == 1) o.W1 = contiguous(W1, d->mpo_dtype, {wl, d1, d1, wr});
  if (n == 2) {
    o.W1 = contiguous(W1, d->mpo_dtype, {wl, d1, d1, wm});
    o.W2 = contiguous(W2, d->mpo_dtype, {wm, d2, d2, wr});
  }
  if (n == 0) {
    o.P = contiguous(psi, d->psi_dtype, {ml, mr});
    o.gy = contiguous(gy, ydt, {ml, mr});
  } else if (n == 1) {
    o.P = contiguous(psi, d->psi_dtype, {ml, d1, mr});
    o.gy = contiguous(gy, ydt, {ml, d1, mr});
  } else {
    o.P = contiguous(psi, d->psi_dtype, {ml, d1, d2, mr});
    o.gy = contiguous(gy, ydt, {ml, d1, d2, mr});
  }
  cudaError_t e = cudaSuccess;
  if (gpsi) {
    // the adjoint matvec: conjugate-transposed operands, the forward path
    const size_t lbytes = (size_t)(ml * wl * ml) * esz(d->env_dtype);
    const size_t rbytes = (size_t)(mr * wr * mr) * esz(d->env_dtype);
    void* Ld = ws.take(lbytes);
    void* Rd = ws.take(rbytes);
    void* W1d = n >= 1 ? ws.take((size_t)o.W1.size() * esz(d->mpo_dtype)) : nullptr;
    void* W2d = n == 2 ? ws.take((size_t)o.W2.size() * esz(d->mpo_dtype)) : nullptr;
    reno_heff_desc dd = *d;
    dd.psi_dtype = ydt;
    size_t need = 0;
    if (reno_heff_workspace_bytes(&dd, &need) != RENO_OK) return RENO_ERR_INVALID;
    void* hws = ws.take(need);
    if (!ws.dry()) {
      const int p3[] = {2, 1, 0}, p4[] = {0, 2, 1, 3};
      e = permute_to(conj_of(o.L), p3, Ld, d->env_dtype, st);
      if (e == cudaSuccess) e = permute_to(conj_of(o.R), p3, Rd, d->env_dtype, st);
      if (e == cudaSuccess && n >= 1) e = permute_to(conj_of(o.W1), p4, W1d, d->mpo_dtype, st);
      if (e == cudaSuccess && n == 2) e = permute_to(conj_of(o.W2), p4, W2d, d->mpo_dtype, st);
      if (e != cudaSuccess) return check_cuda(ctx, e, "reno_heff_backward");
      const int s = reno_heff_apply(ctx, &dd, Ld, W1d, W2d, Rd, gy, gpsi, hws, need);
      if (s != RENO_OK) return s;
    }
  }
  const size_t mark = ws.off;
  size_t peak_off = mark;
  auto chain = [&](cudaError_t (*f)(const Ops&, void*, int, Bump&, cudaStream_t), void* out) {
    if (!out || e != cudaSuccess) return;
    Bump b(ws.base);
    b.off = mark;
    e = f(o, out, gdt, b, st);
    peak_off = std::max(peak_off, b.off);
  };
  chain(grad_L, gL);
  chain(grad_R, gR);
  if (n >= 1) chain(grad_W1, gW1);
  if (n == 2) chain(grad_W2, gW2);
  ws.off = peak_off;
  if (e != cudaSuccess) return ctx ? check_cuda(ctx, e, "reno_heff_backward") : RENO_ERR_CUDA;
  return RENO_OK;
}

}  // namespace bwd
}  // namespace reno

using namespace reno;

extern "C" int reno_heff_backward_workspace_bytes(const reno_heff_desc* d, size_t* bytes) {
  if (!d || !bytes) return RENO_ERR_INVALID;
  bwd::Bump ws(nullptr);
  const char* dummy = reinterpret_cast<const char*>(256);
  void* out = (void*)dummy;
  const int s = bwd::run(nullptr, d, dummy, dummy, dummy, dummy, dummy, dummy, out, out, d->nsite >= 1 ? out : nullptr,
                         d->nsite == 2 ? out : nullptr, out, ws);
  if (s != RENO_OK) return s;
  *bytes = ws.off + 256;
  return RENO_OK;
}

extern "C" int reno_heff_backward(reno_ctx* ctx, const reno_heff_desc* d, const void* L, const void* W1,
                                  const void* W2, const void* R, const void* psi, const void* gy, void* gpsi, void* gL,
                                  void* gW1, void* gW2, void* gR, void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!d || d->nsite < 0 || d->nsite > 2 || !L || !R || !psi || !gy || (d->nsite >= 1 && !W1) ||
      (d->nsite == 2 && !W2))
    return set_error(ctx, RENO_ERR_INVALID, "reno_heff_backward: invalid arguments");
  size_t need = 0;
  if (reno_heff_backward_workspace_bytes(d, &need) != RENO_OK)
    return set_error(ctx, RENO_ERR_INVALID, "reno_heff_backward: invalid descriptor");
  if (!ws || ws_bytes < need) return set_error(ctx, RENO_ERR_WORKSPACE, "reno_heff_backward: workspace too small");
  bwd::Bump b(ws);
  return bwd::run(ctx, d, L, W1, W2, R, psi, gy, gpsi, gL, d->nsite >= 1 ? gW1 : nullptr, d->nsite == 2 ? gW2 : nullptr,
                  gR, b);
}
