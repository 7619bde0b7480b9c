// Quantum-number block movers for the QN-masked truncation.
//  gather:       block = coef_matrix[lset][:, rset]         (svd_qn.py:183-185)
//  scatter:      site[rows[i], dcols[j]] = sigma_j * U[i, scols[j]] (svd_qn.py:89-96
//                blockrecover and lib.py:311-316 select_basis column copies)
#include "reno_common.cuh"

namespace reno {
template <typename T>
__global__ void gather_kernel(const T* __restrict__ src, int64_t ld, const int64_t* __restrict__ rows, int64_t nr,
                              const int64_t* __restrict__ cols, int64_t nc, T* __restrict__ out) {
  const int64_t total = nr * nc;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / nc, j = idx % nc;
    out[idx] = src[rows[i] * ld + cols[j]];
  }
}

__device__ __forceinline__ double scale_by(double v, double s) { return v * s; }
__device__ __forceinline__ double2 scale_by(double2 v, double s) { return make_double2(v.x * s, v.y * s); }

template <typename T>
__global__ void scatter_kernel(const T* __restrict__ src, int64_t src_rs, int64_t src_cs,
                               const int64_t* __restrict__ rows, int64_t nr, const int64_t* __restrict__ scols,
                               const int64_t* __restrict__ dcols, int64_t nc, const double* __restrict__ sigma,
                               T* __restrict__ dst, int64_t dst_rs, int64_t dst_cs) {
  const int64_t total = nr * nc;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx % nr, j = idx / nr;
    T v = src[i * src_rs + scols[j] * src_cs];
    if (sigma) v = scale_by(v, sigma[j]);
    dst[rows[i] * dst_rs + dcols[j] * dst_cs] = v;
  }
}

static int qgrid(int64_t total) {
  int64_t g = ceil_div(total, 256);
  if (g > 148 * 8) g = 148 * 8;
  return g < 1 ? 1 : (int)g;
}
}  // namespace reno

using namespace reno;

extern "C" int reno_qn_gather(reno_ctx* ctx, int32_t dtype, const void* src, int64_t ld, const int64_t* rows,
                              int64_t nr, const int64_t* cols, int64_t nc, void* out) {
  if (!ctx) return RENO_ERR_INVALID;
  if ((dtype != RENO_F64 && dtype != RENO_C128) || nr < 0 || nc < 0 || ld < 0)
    return set_error(ctx, RENO_ERR_INVALID, "reno_qn_gather: bad args");
  if (nr == 0 || nc == 0) return RENO_OK;
  count_launch();
  if (dtype == RENO_C128)
    gather_kernel<double2><<<qgrid(nr * nc), 256, 0, ctx->stream>>>((const double2*)src, ld, rows, nr, cols, nc,
                                                                     (double2*)out);
  else
    gather_kernel<double><<<qgrid(nr * nc), 256, 0, ctx->stream>>>((const double*)src, ld, rows, nr, cols, nc,
                                                                    (double*)out);
  return check_cuda(ctx, cudaGetLastError(), "reno_qn_gather");
}

extern "C" int reno_qn_scatter(reno_ctx* ctx, int32_t dtype, const void* src, int64_t src_rs, int64_t src_cs,
                               const int64_t* rows, int64_t nr, const int64_t* scols, const int64_t* dcols,
                               int64_t nc, const double* sigma, void* dst, int64_t dst_rs, int64_t dst_cs) {
  if (!ctx) return RENO_ERR_INVALID;
  if ((dtype != RENO_F64 && dtype != RENO_C128) || nr < 0 || nc < 0)
    return set_error(ctx, RENO_ERR_INVALID, "reno_qn_scatter: bad args");
  if (nr == 0 || nc == 0) return RENO_OK;
  if (!src || !dst || !rows || !scols || !dcols) return set_error(ctx, RENO_ERR_INVALID, "reno_qn_scatter: null");
  count_launch();
  if (dtype == RENO_C128)
    scatter_kernel<double2><<<qgrid(nr * nc), 256, 0, ctx->stream>>>((const double2*)src, src_rs, src_cs, rows, nr,
                                                                      scols, dcols, nc, sigma, (double2*)dst, dst_rs,
                                                                      dst_cs);
  else
    scatter_kernel<double><<<qgrid(nr * nc), 256, 0, ctx->stream>>>((const double*)src, src_rs, src_cs, rows, nr,
                                                                     scols, dcols, nc, sigma, (double*)dst, dst_rs,
                                                                     dst_cs);
  return check_cuda(ctx, cudaGetLastError(), "reno_qn_scatter");
}
