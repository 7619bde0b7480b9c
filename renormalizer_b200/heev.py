"""Leading eigenpairs of the truncation's Hermitian Gram blocks on the device.

The QN-blocked truncation (svd_qn.py:12-49 with mp.py:693-778 in the
reference, which takes LAPACK gesdd of every block) diagonalises each block's
Gram matrix.  Under a fixed cap k only the leading k + 64 eigenvectors of a
block are used, and cuSOLVER's dense eigensolver spends most of its time in a
tridiagonal reduction kernel (about 25 ms of a 37 ms call on a 2048^2 complex
block).  ``heev_top`` runs the whole eigensolver in libreno_b200 instead:

* reno_heev_top: Householder reduction to a real tridiagonal T in one
  cooperative launch (one grid barrier per column), the kt largest
  eigenvalues of T by Sturm-count multisection and their eigenvectors by
  inverse iteration;
* CholeskyQR2 of the kt tridiagonal eigenvectors (inverse iteration leaves
  vectors of eigenvalues closer than the rounding level non-orthogonal);
* the residual max ||T z - lambda z|| / max |lambda| and the reduction's
  status word, returned as a device tensor so that the caller reads them with
  the singular values it already brings to the host;
* reno_heev_backtransform: K = Q Z in blocks of 64 reflectors (compact WY
  form, three FP64 GEMMs per block).

The caller falls back to cuSOLVER for a block whose check fails.
"""
from __future__ import annotations

import os

import torch

from ._native import Engine


class HeevOptions:
    """``enabled``: use the device eigensolver for Gram blocks of order at
    least ``min_n`` when only the leading kt < n eigenpairs are needed;
    ``tol``: the largest accepted residual relative to max |lambda|.
    RENO_HEEV="0" / "1" overrides ``enabled``."""

    def __init__(self, enabled=False, min_n=512, tol=1e-12):
        env = os.environ.get("RENO_HEEV")
        self.enabled = enabled if env is None else env not in ("0", "")
        self.min_n = min_n
        self.tol = tol
        self.calls = 0
        self.fallbacks = 0


heev_opts = HeevOptions()
_WS = {}


def _workspace(eng: Engine, n: int, kt: int) -> torch.Tensor:
    key = (eng.device, n, kt)
    ws = _WS.get(key)
    if ws is None:
        if len(_WS) > 16:
            _WS.clear()
        ws = eng.heev_workspace(n, kt)
        _WS[key] = ws
    return ws


def heev_top(eng: Engine, G: torch.Tensor, kt: int):
    """The kt largest eigenpairs of the Hermitian matrix G (n x n, float64 or
    complex128, on the device), descending: (w (kt,), K (n, kt) complex128,
    check) with check = [status, Cholesky failures, relative residual] on the
    device (accept when status == 0, failures == 0, residual <= tol)."""
    n = G.shape[0]
    dev = G.device
    heev_opts.calls += 1
    A = G.to(torch.complex128).contiguous().clone()
    d = torch.empty(n, dtype=torch.float64, device=dev)
    e = torch.empty(max(n - 1, 1), dtype=torch.float64, device=dev)
    tau = torch.empty(max(n - 1, 1), dtype=torch.complex128, device=dev)
    w = torch.empty(kt, dtype=torch.float64, device=dev)
    Z = torch.empty((n, kt), dtype=torch.float64, device=dev)
    ws = _workspace(eng, n, kt)
    eng.heev_top(A, d, e, tau, w, Z, ws)
    off = eng.heev_status_offset()
    status = ws[off:off + 4].view(torch.int32).to(torch.float64)
    fails = torch.zeros(1, dtype=torch.float64, device=dev)
    for _ in range(2):
        L, info = torch.linalg.cholesky_ex(Z.transpose(0, 1) @ Z)
        fails += (info != 0).to(torch.float64)
        Z = torch.linalg.solve_triangular(L.transpose(0, 1), Z, upper=True, left=False)
    TZ = d[:, None] * Z
    if n > 1:
        TZ[:-1] += e[:n - 1, None] * Z[1:]
        TZ[1:] += e[:n - 1, None] * Z[:-1]
    scale = torch.clamp(w.abs().max(), min=torch.finfo(torch.float64).tiny)
    res = torch.nan_to_num((TZ - Z * w).abs().max() / scale, nan=float("inf"))
    K = Z.to(torch.complex128).contiguous()
    eng.heev_backtransform(A, tau, K, ws)
    check = torch.stack([status[0], fails[0], res])
    return torch.flip(w, dims=[0]), torch.flip(K, dims=[1]), check


def accepted(check_host) -> bool:
    status, fails, res = check_host
    return status == 0 and fails == 0 and res <= heev_opts.tol
