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

// mode 0: sum conj(x) y ; mode 1: sum |x|^2 (in .x)
__global__ void dot_partial(int64_t n, bool cplx, const void* x, const void* y, int mode, double2* part) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    const double2 a = ld2(x, i, cplx);
    if (mode == 0) {
      const double2 b = ld2(y, i, cplx);
      acc.x += a.x * b.x + a.y * b.y;
      acc.y += a.x * b.y - a.y * b.x;
    } else {
      acc.x += a.x * a.x + a.y * a.y;
    }
  }
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// finalize: mode 0 -> out[0..1] = sum ; mode 1 -> out[0] = sqrt(sum) ;
// mode 2 -> out[0] = sum.x (real part of a dot)
__global__ void dot_final(int nb, const double2* part, int mode, double* out) {
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < nb; i += VT) {
    acc.x += part[i].x;
    acc.y += part[i].y;
  }
  const double2 r = block_sum(acc);
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

// w -= ab[2j] * v + ab[2j-1] * vprev ; partial |w|^2
__global__ void orth_partial(int64_t n, bool cplx, void* w, const void* v, const void* vprev, const double* ab,
                             int j, double2* part) {
  const double alpha = ab[2 * j];
  const double beta = j > 0 ? ab[2 * j - 1] : 0.0;
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    const double2 vi = ld2(v, i, cplx);
    double2 t = make_double2(alpha * vi.x, alpha * vi.y);
    if (j > 0) {
      const double2 pi = ld2(vprev, i, cplx);
      t.x += beta * pi.x;
      t.y += beta * pi.y;
    }
    double2 wi = ld2(w, i, cplx);
    wi.x -= t.x;
    wi.y -= t.y;
    st2(w, i, cplx, wi);
    acc.x += wi.x * wi.x + wi.y * wi.y;
  }
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void scale_inv_kernel(int64_t n, bool cplx, const void* x, const double* s, void* out) {
  const double inv = s[0];
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    double2 v = ld2(x, i, cplx);
    v.x /= inv;
    v.y /= inv;
    st2(out, i, cplx, v);
  }
}

__global__ void lincomb_kernel(int64_t n, int k, bool cplx, const void* V, int64_t ldv, const double* coef,
                               void* out) {
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < k; ++j) {
      const double2 v = ld2(V, (int64_t)j * ldv + i, cplx);
      const double cr = coef[2 * j], ci = coef[2 * j + 1];
      acc.x += cr * v.x - ci * v.y;
      acc.y += cr * v.y + ci * v.x;
    }
    st2(out, i, cplx, acc);
  }
}

// count of elements violating |a-b| <= atol + rtol |b|
__global__ void allclose_partial(int64_t n, bool cplx, const void* a, const void* b, double rtol, double atol,
                                 double2* part) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = blockIdx.x * (int64_t)VT + threadIdx.x; i < n; i += (int64_t)gridDim.x * VT) {
    const double2 x = ld2(a, i, cplx), y = ld2(b, i, cplx);
    const double dx = x.x - y.x, dy = x.y - y.y;
    const double diff = cplx ? hypot(dx, dy) : fabs(dx);
    const double mag = cplx ? hypot(y.x, y.y) : fabs(y.x);
    if (!(diff <= atol + rtol * mag)) acc.x += 1.0;
  }
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void allclose_final(int nb, const double2* part, double* flag) {
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < nb; i += VT) acc.x += part[i].x;
  const double2 r = block_sum(acc);
  if (threadIdx.x == 0) flag[0] = r.x == 0.0 ? 1.0 : 0.0;
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
