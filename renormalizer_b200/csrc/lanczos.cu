// reno_lanczos_expm: the Lanczos exponential psi <- exp(dt H_eff) psi of
// renormalizer/lib/krylov/krylov.py:27-84 (expm_krylov with hop_expr as the
// operator) behind one C call, so that a host without Python can drive the
// local updates of a sweep.
//
// Every matvec (reno_heff_apply) and vector operation (norm, alpha, the
// three-term recurrence, the combination V c, allclose) runs on the device in
// FP64.  The host reads the Lanczos scalars only where the reference makes a
// decision with them: at its convergence checks (every even j > 3), where the
// breakdown test beta_i < 100 n eps is also applied to every beta since the
// previous check -- the Krylov vectors up to a breakdown do not depend on
// what came after it, so the result and the count are the reference's.  The
// small tridiagonal eigenproblem of krylov.py:15-24 is solved on the host by
// implicit QL iterations with shifts (the EISPACK tql2 method of Bowdler,
// Martin, Reinsch and Wilkinson, Numer. Math. 11, 1968).
#include <cfloat>
#include <cmath>
#include <vector>
#include "reno_common.cuh"

using namespace reno;

namespace {

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int64_t psi_elems(const reno_heff_desc* d) {
  if (d->nsite == 0) return (int64_t)d->ml * d->mr;
  if (d->nsite == 1) return (int64_t)d->ml * d->d1 * d->mr;
  return (int64_t)d->ml * d->d1 * d->d2 * d->mr;
}

struct LzLayout {
  size_t V, w, ra, rb, ab, scal, heff, vec, total;
};

int lz_layout(const reno_heff_desc* d, int kmax, LzLayout& L) {
  size_t hb = 0, vb = 0;
  if (reno_heff_workspace_bytes(d, &hb) != RENO_OK) return RENO_ERR_INVALID;
  const int64_t n = psi_elems(d);
  if (reno_vec_workspace_bytes(n, &vb) != RENO_OK) return RENO_ERR_INVALID;
  const size_t vbytes = (size_t)n * 16;
  size_t o = 0;
  L.V = o;
  o = al256(o + (size_t)(kmax + 1) * vbytes);
  L.w = o;
  o = al256(o + vbytes);
  L.ra = o;
  o = al256(o + vbytes);
  L.rb = o;
  o = al256(o + vbytes);
  L.ab = o;
  o = al256(o + (2 * (size_t)kmax + 4) * sizeof(double));
  L.scal = o;
  o = al256(o + 4 * sizeof(double));
  L.heff = o;
  o = al256(o + hb);
  L.vec = o;
  o = al256(o + vb);
  L.total = o;
  return RENO_OK;
}

// Eigenvalues (d, overwritten) and eigenvectors (Z, k x k row-major, column j
// = eigenvector j) of the symmetric tridiagonal matrix with diagonal d and
// off-diagonal e[0..k-2].  Implicit QL with a shift from the leading 2 x 2
// block, one plane rotation at a time, accumulated into Z.
bool tridiag_eig(int k, std::vector<double>& d, std::vector<double> e, std::vector<double>& Z) {
  Z.assign((size_t)k * k, 0.0);
  for (int i = 0; i < k; ++i) Z[(size_t)i * k + i] = 1.0;
  e.resize(k, 0.0);
  e[k - 1] = 0.0;
  for (int l = 0; l < k; ++l) {
    for (int iter = 0;; ++iter) {
      int m = l;
      for (; m < k - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= DBL_EPSILON * dd) break;
      }
      if (m == l) break;
      if (iter >= 64) return false;
      // shift: the eigenvalue of the leading 2 x 2 block nearer to d[l]
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool deflated = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // split: the rotation chain stops here
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int q = 0; q < k; ++q) {
          double* zq = &Z[(size_t)q * k];
          const double t = zq[i + 1];
          zq[i + 1] = s * zq[i] + c * t;
          zq[i] = c * zq[i] - s * t;
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return true;
}

// krylov.py:15-24: coefficients u (nrmv exp(dt w) u[0]) of the Krylov vectors
// for the leading tridiagonal block of order k, as (re, im) pairs
bool tridiag_coeffs(int k, const std::vector<double>& alpha, const std::vector<double>& beta, double nrmv,
                    double dt_re, double dt_im, std::vector<double>& coef) {
  std::vector<double> d(alpha.begin(), alpha.begin() + k), e(beta.begin(), beta.begin() + (k > 0 ? k - 1 : 0)), Z;
  for (double x : d)
    if (!std::isfinite(x)) return false;
  for (double x : e)
    if (!std::isfinite(x)) return false;
  if (!tridiag_eig(k, d, e, Z)) return false;
  coef.assign(2 * (size_t)k, 0.0);
  for (int j = 0; j < k; ++j) {
    const double mag = nrmv * std::exp(dt_re * d[j]) * Z[j];  // Z[0][j]
    const double cr = mag * std::cos(dt_im * d[j]), ci = mag * std::sin(dt_im * d[j]);
    for (int i = 0; i < k; ++i) {
      coef[2 * i] += Z[(size_t)i * k + j] * cr;
      coef[2 * i + 1] += Z[(size_t)i * k + j] * ci;
    }
  }
  return true;
}

}  // namespace

extern "C" int reno_lanczos_workspace_bytes(const reno_heff_desc* desc, int32_t kmax, size_t* bytes) {
  if (!desc || !bytes || kmax < 1) return RENO_ERR_INVALID;
  LzLayout L;
  const int rc = lz_layout(desc, kmax, L);
  if (rc != RENO_OK) return rc;
  *bytes = L.total;
  return RENO_OK;
}

extern "C" int reno_lanczos_expm(reno_ctx* ctx, const reno_heff_desc* desc, const void* L, const void* W1,
                                 const void* W2, const void* R, double dt_re, double dt_im, void* psi, int32_t kmax,
                                 int32_t* out_k, void* ws, size_t ws_bytes) {
  if (!ctx) return RENO_ERR_INVALID;
  if (!desc || !psi || !out_k || !ws || kmax < 1)
    return set_error(ctx, RENO_ERR_INVALID, "reno_lanczos_expm: null argument or kmax < 1");
  if (desc->psi_dtype != RENO_C128)
    return set_error(ctx, RENO_ERR_INVALID, "reno_lanczos_expm: psi must be complex128");
  LzLayout Lz;
  if (lz_layout(desc, kmax, Lz) != RENO_OK) return set_error(ctx, RENO_ERR_INVALID, "reno_lanczos_expm: bad descriptor");
  if (ws_bytes < Lz.total) return set_error(ctx, RENO_ERR_WORKSPACE, "reno_lanczos_expm: workspace too small");
  const int64_t n = psi_elems(desc);
  char* base = static_cast<char*>(ws);
  double2* V = reinterpret_cast<double2*>(base + Lz.V);
  double2* w = reinterpret_cast<double2*>(base + Lz.w);
  double2* res[2] = {reinterpret_cast<double2*>(base + Lz.ra), reinterpret_cast<double2*>(base + Lz.rb)};
  double* ab = reinterpret_cast<double*>(base + Lz.ab);
  double* scal = reinterpret_cast<double*>(base + Lz.scal);
  void* hws = base + Lz.heff;
  void* vws = base + Lz.vec;
  size_t hbytes = 0, vbytes = 0;
  reno_heff_workspace_bytes(desc, &hbytes);
  reno_vec_workspace_bytes(n, &vbytes);
  cudaStream_t st = ctx->stream;
  const double thresh = 100.0 * (double)n * DBL_EPSILON;
  int rc;
#define LZ_TRY(call)              \
  do {                            \
    rc = (call);                  \
    if (rc != RENO_OK) return rc; \
  } while (0)
  LZ_TRY(check_cuda(ctx, cudaMemsetAsync(ab, 0, (2 * (size_t)kmax + 4) * sizeof(double), st),
                    "reno_lanczos_expm: memset"));
  LZ_TRY(reno_vec_norm(ctx, n, RENO_C128, psi, scal, vws, vbytes));
  LZ_TRY(reno_vec_scale_inv(ctx, n, RENO_C128, psi, scal, V));
  std::vector<double> hab(2 * (size_t)kmax + 4), alpha, beta, coef;
  double nrmv = -1.0;
  int checked = 0, last = -1;  // last: index of res[] holding the previous check's result
  auto read_scalars = [&](int j) -> int {
    int r = check_cuda(ctx, cudaMemcpyAsync(hab.data(), ab, (2 * (size_t)j + 2) * sizeof(double),
                                            cudaMemcpyDeviceToHost, st), "reno_lanczos_expm: scalars");
    if (r == RENO_OK && nrmv < 0) {
      r = check_cuda(ctx, cudaMemcpyAsync(&nrmv, scal, sizeof(double), cudaMemcpyDeviceToHost, st),
                     "reno_lanczos_expm: norm");
    }
    if (r == RENO_OK) r = check_cuda(ctx, cudaStreamSynchronize(st), "reno_lanczos_expm: sync");
    if (r != RENO_OK) return r;
    if (!(nrmv > 0.0) || !std::isfinite(nrmv))
      return set_error(ctx, RENO_ERR_NONFINITE, "reno_lanczos_expm: start vector is zero or not finite");
    alpha.assign(j + 1, 0.0);
    beta.assign(j + 1, 0.0);
    for (int i = 0; i <= j; ++i) {
      alpha[i] = hab[2 * i];
      beta[i] = hab[2 * i + 1];
    }
    return RENO_OK;
  };
  // the result (V[0:k] coef, already formed in `from`) becomes psi
  auto finish = [&](int k, const double2* from) -> int {
    *out_k = k;
    return check_cuda(ctx, cudaMemcpyAsync(psi, from, (size_t)n * 16, cudaMemcpyDeviceToDevice, st),
                      "reno_lanczos_expm: copy out");
  };
  for (int j = 0; j < n; ++j) {
    if (j >= kmax)
      return set_error(ctx, RENO_ERR_WORKSPACE, "reno_lanczos_expm: no convergence within kmax = " +
                                                    std::to_string(kmax) + " Krylov vectors; raise kmax");
    LZ_TRY(reno_heff_apply(ctx, desc, L, W1, W2, R, V + (size_t)j * n, w, hws, hbytes));
    LZ_TRY(reno_krylov_alpha(ctx, n, RENO_C128, w, V + (size_t)j * n, ab, j, vws, vbytes));
    const bool exhausted = (j == n - 1);
    if (!exhausted) {
      LZ_TRY(reno_krylov_orth(ctx, n, RENO_C128, w, V + (size_t)j * n, j > 0 ? V + (size_t)(j - 1) * n : nullptr,
                              ab, j, vws, vbytes));
      LZ_TRY(reno_vec_scale_inv(ctx, n, RENO_C128, w, ab + 2 * (size_t)j + 1, V + (size_t)(j + 1) * n));
    }
    if (!(exhausted || (j > 3 && j % 2 == 0))) continue;
    LZ_TRY(read_scalars(j));
    int kk = -1;  // breakdown before this point
    for (int i = checked; i < (exhausted ? j : j + 1); ++i)
      if (beta[i] < thresh) {
        kk = i;
        break;
      }
    checked = exhausted ? j : j + 1;
    const int k = kk >= 0 ? kk + 1 : j + 1;
    if (!tridiag_coeffs(k, alpha, beta, nrmv, dt_re, dt_im, coef))
      return set_error(ctx, RENO_ERR_NONFINITE, "reno_lanczos_expm: Lanczos scalars are not finite");
    // coefficients to the device (the scalars area past the Lanczos entries)
    double* dcoef = reinterpret_cast<double*>(w);  // w is free until the next matvec
    LZ_TRY(check_cuda(ctx, cudaMemcpyAsync(dcoef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice,
                                           st), "reno_lanczos_expm: coefficients"));
    const int slot = last == 0 ? 1 : 0;
    LZ_TRY(reno_vec_lincomb(ctx, n, k, RENO_C128, V, n, dcoef, res[slot]));
    if (kk >= 0 || exhausted) return finish(k, res[slot]);
    if (last >= 0) {
      LZ_TRY(reno_vec_allclose(ctx, n, RENO_C128, res[last], res[slot], 1e-5, 1e-8, scal + 2, vws, vbytes));
      double flag = 0.0;
      LZ_TRY(check_cuda(ctx, cudaMemcpyAsync(&flag, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st),
                        "reno_lanczos_expm: allclose"));
      LZ_TRY(check_cuda(ctx, cudaStreamSynchronize(st), "reno_lanczos_expm: sync"));
      if (flag == 1.0) return finish(k, res[slot]);
    }
    last = slot;
  }
#undef LZ_TRY
  return set_error(ctx, RENO_ERR_INVALID, "reno_lanczos_expm: empty vector");
}
