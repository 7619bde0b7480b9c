// Vector kernels of the Lanczos exponential (krylov.py:27-84) and of the
// Davidson solver (davidson.py:154-441): dot products, norms, the three-term
// Lanczos recurrence, linear combinations of Krylov vectors, allclose tests
// and the diagonal preconditioner.  Reductions are two-pass with a fixed
// block count and fixed summation order, so results are bitwise
// reproducible run to run (no atomics).
#include "reno_common.cuh"

namespace reno {

constexpr int VT = 256;          // threads per block
constexpr int VMAX_BLOCKS = 1184;  // 148 SMs x 8: partial-sum slots

static int vec_blocks(int64_t n) {
  int64_t b = ceil_div(n, (int64_t)VT * 4);
  if (b > VMAX_BLOCKS) b = VMAX_BLOCKS;
  if (b < 1) b = 1;
  return (int)b;
}

__device__ __forceinline__ double2 ld2(const void* p, int64_t i, bool cplx) {
  if (cplx) return reinterpret_cast<const double2*>(p)[i];
  return make_double2(reinterpret_cast<const double*>(p)[i], 0.0);
}
__device__ __forceinline__ void st2(void* p, int64_t i, bool cplx, double2 v) {
  if (cplx)
    reinterpret_cast<double2*>(p)[i] = v;
  else
    reinterpret_cast<double*>(p)[i] = v.x;
}

// block reduce of a double2 (fixed order)
__device__ __forceinline__ double2 block_sum(double2 v) {
  __shared__ double2 sh[VT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double2 r = make_double2(0.0, 0.0);
  if (warp == 0) {
    r = lane < VT / 32 ? sh[lane] : make_double2(0.0, 0.0);
    for (int o = 16; o > 0; o >>= 1) {
      r.x += __shfl_down_sync(0xffffffffu, r.x, o);
      r.y += __shfl_down_sync(0xffffffffu, r.y, o);
    }
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// Per-block bodies shared by the single and the grouped kernels: block b of
// the nb blocks that cover one vector walks i = b VT + t, stepping nb VT.
// Their arithmetic is written with explicitly rounded operations, so no
// kernel that inlines them can contract it into FMAs differently: a grouped
// call rounds exactly like the single one.
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }

// mode 0: sum conj(x) y ; mode 1: sum |x|^2 (in .x)
__device__ __forceinline__ double2 dot_body(int64_t n, bool cplx, const void* x, const void* y, int mode, int64_t b,
                                            int64_t nb) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = b * VT + threadIdx.x; i < n; i += nb * VT) {
    const double2 a = ld2(x, i, cplx);
    if (mode == 0) {
      const double2 c = ld2(y, i, cplx);
      acc.x = add_(acc.x, fma_(a.x, c.x, mul_(a.y, c.y)));
      acc.y = add_(acc.y, fma_(a.x, c.y, -mul_(a.y, c.x)));
    } else {
      acc.x = add_(acc.x, fma_(a.x, a.x, mul_(a.y, a.y)));
    }
  }
  return acc;
}

// w -= ab[2j] * v + ab[2j-1] * vprev ; partial |w|^2
__device__ __forceinline__ double2 orth_body(int64_t n, bool cplx, void* w, const void* v, const void* vprev,
                                             const double* ab, int j, int64_t b, int64_t nb) {
  const double alpha = ab[2 * j];
  const double beta = j > 0 ? ab[2 * j - 1] : 0.0;
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = b * VT + threadIdx.x; i < n; i += nb * VT) {
    const double2 vi = ld2(v, i, cplx);
    double2 t = make_double2(mul_(alpha, vi.x), mul_(alpha, vi.y));
    if (j > 0) {
      const double2 pi = ld2(vprev, i, cplx);
      t.x = fma_(beta, pi.x, t.x);
      t.y = fma_(beta, pi.y, t.y);
    }
    double2 wi = ld2(w, i, cplx);
    wi.x = add_(wi.x, -t.x);
    wi.y = add_(wi.y, -t.y);
    st2(w, i, cplx, wi);
    acc.x = add_(acc.x, fma_(wi.x, wi.x, mul_(wi.y, wi.y)));
  }
  return acc;
}

__device__ __forceinline__ void scale_inv_body(int64_t n, bool cplx, const void* x, const double* s, void* out,
                                               int64_t b, int64_t nb) {
  const double inv = s[0];
  for (int64_t i = b * VT + threadIdx.x; i < n; i += nb * VT) {
    double2 v = ld2(x, i, cplx);
    v.x /= inv;
    v.y /= inv;
    st2(out, i, cplx, v);
  }
}

__device__ __forceinline__ void lincomb_body(int64_t n, int k, bool cplx, const void* V, int64_t ldv,
                                             const double* coef, void* out, int64_t b, int64_t nb) {
  for (int64_t i = b * VT + threadIdx.x; i < n; i += nb * VT) {
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < k; ++j) {
      const double2 v = ld2(V, (int64_t)j * ldv + i, cplx);
      const double cr = coef[2 * j], ci = coef[2 * j + 1];
      acc.x = add_(acc.x, fma_(cr, v.x, -mul_(ci, v.y)));
      acc.y = add_(acc.y, fma_(cr, v.y, mul_(ci, v.x)));
    }
    st2(out, i, cplx, acc);
  }
}

// count of elements violating |a-b| <= atol + rtol |b|
__device__ __forceinline__ double2 allclose_body(int64_t n, bool cplx, const void* a, const void* b_, double rtol,
                                                 double atol, int64_t b, int64_t nb) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = b * VT + threadIdx.x; i < n; i += nb * VT) {
    const double2 x = ld2(a, i, cplx), y = ld2(b_, i, cplx);
    const double dx = x.x - y.x, dy = x.y - y.y;
    const double diff = cplx ? hypot(dx, dy) : fabs(dx);
    const double mag = cplx ? hypot(y.x, y.y) : fabs(y.x);
    if (!(diff <= fma_(rtol, mag, atol))) acc.x += 1.0;
  }
  return acc;
}

// second pass: the nb partials in a fixed order (valid in thread 0)
__device__ __forceinline__ double2 final_sum(int nb, const double2* part) {
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < nb; i += VT) {
    acc.x = add_(acc.x, part[i].x);
    acc.y = add_(acc.y, part[i].y);
  }
  return block_sum(acc);
}

__global__ void dot_partial(int64_t n, bool cplx, const void* x, const void* y, int mode, double2* part) {
  const double2 r = block_sum(dot_body(n, cplx, x, y, mode, blockIdx.x, gridDim.x));
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// finalize: mode 0 -> out[0..1] = sum ; mode 1 -> out[0] = sqrt(sum) ;
// mode 2 -> out[0] = sum.x (real part of a dot)
__global__ void dot_final(int nb, const double2* part, int mode, double* out) {
  const double2 r = final_sum(nb, part);
  if (threadIdx.x == 0) {
    if (mode == 0) {
      out[0] = r.x;
      out[1] = r.y;
    } else if (mode == 1) {
      out[0] = sqrt(r.x);
    } else {
      out[0] = r.x;
    }
  }
}

__global__ void orth_partial(int64_t n, bool cplx, void* w, const void* v, const void* vprev, const double* ab,
                             int j, double2* part) {
  const double2 r = block_sum(orth_body(n, cplx, w, v, vprev, ab, j, blockIdx.x, gridDim.x));
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void scale_inv_kernel(int64_t n, bool cplx, const void* x, const double* s, void* out) {
  scale_inv_body(n, cplx, x, s, out, blockIdx.x, gridDim.x);
}

__global__ void lincomb_kernel(int64_t n, int k, bool cplx, const void* V, int64_t ldv, const double* coef,
                               void* out) {
  lincomb_body(n, k, cplx, V, ldv, coef, out, blockIdx.x, gridDim.x);
}

__global__ void allclose_partial(int64_t n, bool cplx, const void* a, const void* b, double rtol, double atol,
                                 double2* part) {
  const double2 r = block_sum(allclose_body(n, cplx, a, b, rtol, atol, blockIdx.x, gridDim.x));
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void allclose_final(int nb, const double2* part, double* flag) {
  const double2 r = final_sum(nb, part);
  if (threadIdx.x == 0) flag[0] = r.x == 0.0 ? 1.0 : 0.0;
}

// ---------------------------------------------------------------- grouped
// One operation on many vectors: item p owns blocks first[p] .. first[p+1]-1
// of the launch (its single call's vec_blocks(n) of them, in the same order)
// and slots first[p].. of the partial-sum workspace.
struct VecGroup {
  reno_vec_item it[RENO_VEC_GROUP_MAX];
  int first[RENO_VEC_GROUP_MAX + 1];
  int count, op;
  double rtol, atol;
};

__device__ __forceinline__ int group_item(const VecGroup& g, int blk) {
  int lo = 0, hi = g.count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g.first[mid] <= blk) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void vec_group_partial(const __grid_constant__ VecGroup g, double2* part) {
  const int p = group_item(g, blockIdx.x);
  const reno_vec_item& it = g.it[p];
  const int64_t b = blockIdx.x - g.first[p], nb = g.first[p + 1] - g.first[p];
  const bool cplx = it.dtype == RENO_C128;
  double2 acc;
  if (g.op == RENO_VOP_NORM)
    acc = dot_body(it.n, cplx, it.x, it.x, 1, b, nb);
  else if (g.op == RENO_VOP_ALPHA)
    acc = dot_body(it.n, cplx, it.x, it.y, 0, b, nb);
  else if (g.op == RENO_VOP_ORTH)
    acc = orth_body(it.n, cplx, it.out, it.x, it.y, it.scalars, it.j, b, nb);
  else
    acc = allclose_body(it.n, cplx, it.x, it.y, g.rtol, g.atol, b, nb);
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void vec_group_final(const __grid_constant__ VecGroup g, const double2* part) {
  const int p = blockIdx.x;
  const reno_vec_item& it = g.it[p];
  const double2 r = final_sum(g.first[p + 1] - g.first[p], part + g.first[p]);
  if (threadIdx.x == 0) {
    if (g.op == RENO_VOP_NORM)
      it.scalars[0] = sqrt(r.x);
    else if (g.op == RENO_VOP_ALPHA)
      it.scalars[2 * it.j] = r.x;
    else if (g.op == RENO_VOP_ORTH)
      it.scalars[2 * it.j + 1] = sqrt(r.x);
    else
      it.scalars[0] = r.x == 0.0 ? 1.0 : 0.0;
  }
}

__global__ void vec_group_elementwise(const __grid_constant__ VecGroup g) {
  const int p = group_item(g, blockIdx.x);
  const reno_vec_item& it = g.it[p];
  const int64_t b = blockIdx.x - g.first[p], nb = g.first[p + 1] - g.first[p];
  const bool cplx = it.dtype == RENO_C128;
  if (g.op == RENO_VOP_SCALE_INV)
    scale_inv_body(it.n, cplx, it.x, it.s, it.out, b, nb);
  else
    lincomb_body(it.n, it.j, cplx, it.x, it.ldv, it.s, it.out, b, nb);
}

__global__ void axpy_kernel(int64_t n, bool cplx, void* y, const void* x, const double* c, double sgn) {
  const double cr = sgn * c[0], ci = cplx ? sgn * c[1] : 0.0;
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    const double2 xv = ld2(x, i, cplx);
    double2 yv = ld2(y, i, cplx);
    yv.x += cr * xv.x - ci * xv.y;
    yv.y += cr * xv.y + ci * xv.x;
    st2(y, i, cplx, yv);
  }
}

__global__ void precond_kernel(int64_t n, bool cplx, const void* r, const double* hdiag, const double* e,
                               double shift, void* out) {
  const double e0 = e[0];
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    double2 v = ld2(r, i, cplx);
    const double den = hdiag[i] - e0 + shift;
    v.x /= den;
    v.y /= den;
    st2(out, i, cplx, v);
  }
}

static bool dt_ok(int dt) { return dt == RENO_F64 || dt == RENO_C128; }

}  // namespace reno

using namespace reno;

extern "C" int reno_vec_workspace_bytes(int64_t n, size_t* bytes) {
  if (!bytes || n < 0) return RENO_ERR_INVALID;
  *bytes = (size_t)VMAX_BLOCKS * sizeof(double2);
  return RENO_OK;
}

#define VEC_PRE(ctx, n, dtype, ws, ws_bytes)                                                 \
  if (!ctx) return RENO_ERR_INVALID;                                                         \
  if (!dt_ok(dtype) || n < 0) return set_error(ctx, RENO_ERR_INVALID, "vector op: bad args"); \
  if (ws_bytes < (size_t)VMAX_BLOCKS * sizeof(double2) || !ws)                               \
    return set_error(ctx, RENO_ERR_WORKSPACE, "vector op: workspace too small");

extern "C" int reno_vec_dotc(reno_ctx* ctx, int64_t n, int32_t dtype, const void* x, const void* y, double* out,
                             void* ws, size_t ws_bytes) {
  VEC_PRE(ctx, n, dtype, ws, ws_bytes);
  const int nb = vec_blocks(n);
  count_launch(2);
  dot_partial<<<nb, VT, 0, ctx->stream>>>(n, dtype == RENO_C128, x, y, 0, (double2*)ws);
  dot_final<<<1, VT, 0, ctx->stream>>>(nb, (double2*)ws, 0, out);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_dotc");
}

extern "C" int reno_vec_norm(reno_ctx* ctx, int64_t n, int32_t dtype, const void* x, double* out, void* ws,
                             size_t ws_bytes) {
  VEC_PRE(ctx, n, dtype, ws, ws_bytes);
  const int nb = vec_blocks(n);
  count_launch(2);
  dot_partial<<<nb, VT, 0, ctx->stream>>>(n, dtype == RENO_C128, x, x, 1, (double2*)ws);
  dot_final<<<1, VT, 0, ctx->stream>>>(nb, (double2*)ws, 1, out);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_norm");
}

extern "C" int reno_krylov_alpha(reno_ctx* ctx, int64_t n, int32_t dtype, const void* w, const void* v, double* ab,
                                 int32_t j, void* ws, size_t ws_bytes) {
  VEC_PRE(ctx, n, dtype, ws, ws_bytes);
  if (j < 0 || !ab) return set_error(ctx, RENO_ERR_INVALID, "reno_krylov_alpha: bad index");
  const int nb = vec_blocks(n);
  count_launch(2);
  dot_partial<<<nb, VT, 0, ctx->stream>>>(n, dtype == RENO_C128, w, v, 0, (double2*)ws);
  dot_final<<<1, VT, 0, ctx->stream>>>(nb, (double2*)ws, 2, ab + 2 * j);
  return check_cuda(ctx, cudaGetLastError(), "reno_krylov_alpha");
}

extern "C" int reno_krylov_orth(reno_ctx* ctx, int64_t n, int32_t dtype, void* w, const void* v, const void* vprev,
                                double* ab, int32_t j, void* ws, size_t ws_bytes) {
  VEC_PRE(ctx, n, dtype, ws, ws_bytes);
  if (j < 0 || !ab || (j > 0 && !vprev)) return set_error(ctx, RENO_ERR_INVALID, "reno_krylov_orth: bad args");
  const int nb = vec_blocks(n);
  count_launch(2);
  orth_partial<<<nb, VT, 0, ctx->stream>>>(n, dtype == RENO_C128, w, v, vprev, ab, j, (double2*)ws);
  dot_final<<<1, VT, 0, ctx->stream>>>(nb, (double2*)ws, 1, ab + 2 * j + 1);
  return check_cuda(ctx, cudaGetLastError(), "reno_krylov_orth");
}

extern "C" int reno_vec_scale_inv(reno_ctx* ctx, int64_t n, int32_t dtype, const void* x, const double* s,
                                  void* out) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!dt_ok(dtype) || n < 0 || !s) return set_error(ctx, RENO_ERR_INVALID, "reno_vec_scale_inv: bad args");
  count_launch(1);
  scale_inv_kernel<<<vec_blocks(n), VT, 0, ctx->stream>>>(n, dtype == RENO_C128, x, s, out);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_scale_inv");
}

extern "C" int reno_vec_lincomb(reno_ctx* ctx, int64_t n, int32_t k, int32_t dtype, const void* V, int64_t ldv,
                                const double* coef, void* out) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!dt_ok(dtype) || n < 0 || k < 0 || ldv < n || !coef)
    return set_error(ctx, RENO_ERR_INVALID, "reno_vec_lincomb: bad args");
  count_launch(1);
  lincomb_kernel<<<vec_blocks(n), VT, 0, ctx->stream>>>(n, k, dtype == RENO_C128, V, ldv, coef, out);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_lincomb");
}

extern "C" int reno_vec_allclose(reno_ctx* ctx, int64_t n, int32_t dtype, const void* a, const void* b, double rtol,
                                 double atol, double* flag, void* ws, size_t ws_bytes) {
  VEC_PRE(ctx, n, dtype, ws, ws_bytes);
  const int nb = vec_blocks(n);
  count_launch(2);
  allclose_partial<<<nb, VT, 0, ctx->stream>>>(n, dtype == RENO_C128, a, b, rtol, atol, (double2*)ws);
  allclose_final<<<1, VT, 0, ctx->stream>>>(nb, (double2*)ws, flag);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_allclose");
}

extern "C" int reno_vec_axpy(reno_ctx* ctx, int64_t n, int32_t dtype, void* y, const void* x, const double* c,
                             double c_sign) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!dt_ok(dtype) || n < 0 || !c) return set_error(ctx, RENO_ERR_INVALID, "reno_vec_axpy: bad args");
  count_launch(1);
  axpy_kernel<<<vec_blocks(n), VT, 0, ctx->stream>>>(n, dtype == RENO_C128, y, x, c, c_sign);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_axpy");
}

extern "C" int reno_vec_precond(reno_ctx* ctx, int64_t n, int32_t dtype, const void* r, const double* hdiag,
                                const double* e, double shift, void* out) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!dt_ok(dtype) || n < 0 || !hdiag || !e) return set_error(ctx, RENO_ERR_INVALID, "reno_vec_precond: bad args");
  count_launch(1);
  precond_kernel<<<vec_blocks(n), VT, 0, ctx->stream>>>(n, dtype == RENO_C128, r, hdiag, e, shift, out);
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_precond");
}

extern "C" int reno_vec_grouped_workspace_bytes(int32_t count, size_t* bytes) {
  if (!bytes || count < 0 || count > RENO_VEC_GROUP_MAX) return RENO_ERR_INVALID;
  *bytes = (size_t)(count > 0 ? count : 1) * VMAX_BLOCKS * sizeof(double2);
  return RENO_OK;
}

extern "C" int reno_vec_grouped(reno_ctx* ctx, int32_t op, int32_t count, const reno_vec_item* items, double rtol,
                                double atol, void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (op < RENO_VOP_NORM || op > RENO_VOP_ALLCLOSE || count < 0 || count > RENO_VEC_GROUP_MAX ||
      (count > 0 && !items))
    return set_error(ctx, RENO_ERR_INVALID, "reno_vec_grouped: bad op or count");
  if (count == 0) return RENO_OK;
  const bool reduces = op != RENO_VOP_SCALE_INV && op != RENO_VOP_LINCOMB;
  if (reduces && (!ws || ws_bytes < (size_t)count * VMAX_BLOCKS * sizeof(double2)))
    return set_error(ctx, RENO_ERR_WORKSPACE, "reno_vec_grouped: workspace too small");
  VecGroup g;
  g.count = count;
  g.op = op;
  g.rtol = rtol;
  g.atol = atol;
  int total = 0;
  for (int p = 0; p < count; ++p) {
    const reno_vec_item& it = items[p];
    bool ok = dt_ok(it.dtype) && it.n >= 0;
    switch (op) {
      case RENO_VOP_NORM: ok = ok && it.x && it.scalars; break;
      case RENO_VOP_ALPHA: ok = ok && it.x && it.y && it.scalars && it.j >= 0; break;
      case RENO_VOP_ORTH: ok = ok && it.out && it.x && it.scalars && it.j >= 0 && (it.j == 0 || it.y); break;
      case RENO_VOP_SCALE_INV: ok = ok && it.x && it.s && it.out; break;
      case RENO_VOP_LINCOMB: ok = ok && it.x && it.s && it.out && it.j >= 0 && it.ldv >= it.n; break;
      default: ok = ok && it.x && it.y && it.scalars; break;
    }
    if (!ok) return set_error(ctx, RENO_ERR_INVALID, "reno_vec_grouped: bad item " + std::to_string(p));
    g.it[p] = it;
    g.first[p] = total;
    total += vec_blocks(it.n);
  }
  g.first[count] = total;
  if (reduces) {
    count_launch(2);
    vec_group_partial<<<total, VT, 0, ctx->stream>>>(g, (double2*)ws);
    vec_group_final<<<count, VT, 0, ctx->stream>>>(g, (const double2*)ws);
  } else {
    count_launch(1);
    vec_group_elementwise<<<total, VT, 0, ctx->stream>>>(g);
  }
  return check_cuda(ctx, cudaGetLastError(), "reno_vec_grouped");
}
