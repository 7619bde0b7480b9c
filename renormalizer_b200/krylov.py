"""Lanczos exponential on the GPU, drop-in for
renormalizer/lib/krylov/krylov.py:27-84 (``expm_krylov``).

The Krylov basis V, the matvecs and every vector operation (vdot, norm,
three-term recurrence, V @ coeffs, allclose) stay in HBM and run in
libreno_b200; alpha/beta are produced on the device in FP64.  The small
tridiagonal eigenproblem is solved in FP64 on the host with the same SciPy
routine the reference uses (krylov.py:15-24), so the stopping decisions
(breakdown at beta < 100 n eps, ``allclose`` every even j > 3) follow the
reference exactly.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.linalg import eigh_tridiagonal

from ._native import Engine
from .hop_expr import as_device

EPS = np.finfo(float).eps


def _tridiag_coeffs(alpha, beta, v_norm, dt):
    """krylov.py:15-24 : u_hess @ (v_norm * exp(dt * w_hess) * u_hess[0])."""
    try:
        w_hess, u_hess = eigh_tridiagonal(alpha, beta)
    except np.linalg.LinAlgError:
        h = np.diag(alpha) + np.diag(beta, k=-1) + np.diag(beta, k=1)
        w_hess, u_hess = np.linalg.eigh(h)
    return u_hess @ (v_norm * np.exp(dt * w_hess) * u_hess[0])


class _Krylov:
    def __init__(self, eng: Engine, n: int, dtype, device, block_size):
        self.eng = eng
        self.n = n
        self.dtype = dtype
        self.code = 1 if dtype == torch.complex128 else 0
        self.V = torch.empty((block_size, n), dtype=dtype, device=device)
        self.ab = torch.zeros(2 * block_size + 2, dtype=torch.float64, device=device)
        self.tmp = torch.zeros(4, dtype=torch.float64, device=device)
        self.coef = torch.zeros(2 * block_size, dtype=torch.float64, device=device)

    def grow(self, block_size):
        V = torch.empty((self.V.shape[0] + block_size, self.n), dtype=self.dtype, device=self.V.device)
        V[: self.V.shape[0]] = self.V
        self.V = V
        ab = torch.zeros(2 * self.V.shape[0] + 2, dtype=torch.float64, device=self.V.device)
        ab[: self.ab.numel()] = self.ab
        self.ab = ab
        self.coef = torch.zeros(2 * self.V.shape[0], dtype=torch.float64, device=self.V.device)

    def combine(self, k, coeffs, out):
        c = np.zeros(2 * k)
        c[0::2] = np.real(coeffs)
        c[1::2] = np.imag(coeffs) if np.iscomplexobj(coeffs) else 0.0
        self.coef[: 2 * k].copy_(torch.from_numpy(c), non_blocking=False)
        self.eng.lincomb(self.V, k, self.coef, out)
        return out


def expm_krylov(Afunc, dt, vstart, block_size=50):
    """Krylov approximation of expm(dt*A) @ vstart for Hermitian A.

    Returns (vector, number of matvecs) like the reference.  ``Afunc`` maps a
    1-D device vector to a 1-D device vector (e.g. a HeffOperator)."""
    if not np.iscomplex(dt):
        dt = dt.real
    v = as_device(vstart).reshape(-1)
    n = v.numel()
    eng = Engine.get(v.device)
    dt_cplx = np.iscomplexobj(dt) and np.iscomplex(dt)
    # the result is complex when exp(dt*w) is complex (krylov.py:24)
    work_dtype = torch.complex128 if (v.is_complex() or dt_cplx) else torch.float64
    if v.dtype != work_dtype:
        v = v.to(work_dtype)
    K = _Krylov(eng, n, work_dtype, v.device, block_size)
    code = K.code
    # nrmv = ||vstart||; V[0] = vstart / nrmv
    eng.vec_norm(v, K.tmp)
    nrmv = float(K.tmp[0].item())
    assert nrmv > 0
    if not np.isfinite(nrmv):
        raise FloatingPointError("expm_krylov: start vector is not finite")
    eng.scale_inv(v, K.tmp, K.V[0])
    res_prev = None
    out_a = torch.empty(n, dtype=work_dtype, device=v.device)
    out_b = torch.empty(n, dtype=work_dtype, device=v.device)
    for j in range(n):
        w = Afunc(K.V[j])
        w = w.reshape(-1)
        if w.dtype != work_dtype:
            w = w.to(work_dtype)
        if not w.is_contiguous():
            w = w.contiguous()
        eng.krylov_alpha(w, K.V[j], K.ab, j)
        if j == n - 1:
            ab = K.ab[: 2 * j + 2].cpu().numpy()
            coeffs = _tridiag_coeffs(ab[0::2][: j + 1], ab[1::2][:j], nrmv, dt)
            return K.combine(j + 1, coeffs, out_a), j + 1
        if K.V.shape[0] == j + 1:
            K.grow(block_size)
        vprev = K.V[j - 1] if j > 0 else None
        eng.krylov_orth(w, K.V[j], vprev, K.ab, j)
        ab = K.ab[: 2 * j + 2].cpu().numpy()
        alpha, beta = ab[0::2][: j + 1], ab[1::2][: j + 1]
        if not np.isfinite(beta[j]):
            raise FloatingPointError("expm_krylov: Lanczos vector is not finite")
        if beta[j] < 100 * n * EPS:
            coeffs = _tridiag_coeffs(alpha, beta[:j], nrmv, dt)
            return K.combine(j + 1, coeffs, out_a), j + 1
        if 3 < j and j % 2 == 0:
            coeffs = _tridiag_coeffs(alpha, beta[:j], nrmv, dt)
            new_res = K.combine(j + 1, coeffs, out_b if res_prev is out_a else out_a)
            if res_prev is not None:
                flag = K.tmp[2:3]
                eng.allclose(res_prev, new_res, 1e-5, 1e-8, flag)
                if float(flag.item()) == 1.0:
                    return new_res, j + 1
            res_prev = new_res
        # V[j+1] = w / beta[j]
        eng.scale_inv(w, K.ab[2 * j + 1:], K.V[j + 1])
