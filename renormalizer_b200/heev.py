"""Leading eigenpairs of the truncation's Hermitian Gram blocks on the device.

The QN-blocked truncation (svd_qn.py:12-49 with mp.py:693-778 in the
reference, which takes LAPACK gesdd of every block) diagonalises each block's
Gram matrix.  Under a fixed cap k only the leading k + 64 eigenvectors of a
block are used, and cuSOLVER's dense eigensolver spends most of its time in a
tridiagonal reduction kernel (about 25 ms of a 37 ms call on a 2048^2 complex
block).  ``heev_top_batched`` runs the whole eigensolver in libreno_b200
instead, for all QN blocks of a bond at once:

* reno_heev_top_batched: Householder reduction to a real tridiagonal T in one
  cooperative launch shared by the blocks (one grid barrier per column), the kt largest
  eigenvalues of T by Sturm-count multisection and their eigenvectors by
  inverse iteration;
* Householder QR of the kt tridiagonal eigenvectors, largest eigenvalue
  first (inverse iteration leaves vectors of eigenvalues closer than the
  rounding level non-orthogonal, or nearly parallel);
* the residual max ||T z - rho z|| / max |lambda| and the reduction's
  status word, returned as a device tensor so that the caller reads them with
  the singular values it already brings to the host;
* reno_heev_backtransform_batched: K = Q Z in blocks of 64 reflectors (compact WY
  form, three FP64 GEMMs per block).

The caller falls back to cuSOLVER for a block whose check fails.
"""
from __future__ import annotations

import os

import torch

from ._native import HEEV_MAX_BATCH, Engine, HeevProblem


class HeevOptions:
    """``enabled``: use the device eigensolver for Gram blocks of order at
    least ``min_n`` (default: every block; cuSOLVER only redoes a block whose
    checks fail); ``tol``: the largest accepted residual relative to
    max |lambda|.  RENO_HEEV="0" / "1" overrides ``enabled``."""

    def __init__(self, enabled=True, min_n=1, tol=1e-12):
        env = os.environ.get("RENO_HEEV")
        self.enabled = enabled if env is None else env not in ("0", "")
        self.min_n = min_n
        self.tol = tol
        self.calls = 0
        self.fallbacks = 0


heev_opts = HeevOptions()
def heev_top(eng: Engine, G: torch.Tensor, kt: int):
    """The kt largest eigenpairs of the Hermitian matrix G (n x n, float64 or
    complex128, on the device), descending: (w (kt,), K (n, kt) complex128,
    check) with check = [status, 0, relative residual] on the device (accept
    when status == 0 and residual <= tol).  One matrix of heev_top_batched."""
    return heev_top_batched(eng, [G], [kt])[0]


def accepted(check_host) -> bool:
    status, fails, res = check_host
    return status == 0 and fails == 0 and res <= heev_opts.tol


_WSB = {}


def _batched_ws(eng: Engine, nbytes: int) -> torch.Tensor:
    ws = _WSB.get(eng.device)
    if ws is None or ws.numel() < nbytes:
        ws = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=f"cuda:{eng.device}")
        _WSB[eng.device] = ws
    return ws


def _vp(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


def heev_top_batched(eng: Engine, Gs, kts):
    """heev_top for several Hermitian matrices at once (the QN blocks of one
    bond): one batched reduction launch, then per matrix the kt largest
    eigenvalues (Sturm bisection) and inverse-iteration vectors, ordered
    descending and orthonormalised together by Householder QR
    (reno_qr_blocks) -- which, unlike a Cholesky-based orthonormalisation,
    cannot fail when vectors of a tight cluster come out nearly parallel --
    then the back-transformation.  Returns per matrix (w (kt,) descending,
    K (n, kt) complex128, check) with check = [status, 0, residual] on the
    device; the residual is max_j ||T z_j - rho_j z_j|| / max |w| with rho_j
    the Rayleigh quotient of the orthonormalised z_j."""
    out = []
    for i0 in range(0, len(Gs), HEEV_MAX_BATCH):
        out += _heev_chunk(eng, Gs[i0:i0 + HEEV_MAX_BATCH], kts[i0:i0 + HEEV_MAX_BATCH])
    return out


def _heev_chunk(eng, Gs, kts):
    dev = Gs[0].device
    heev_opts.calls += len(Gs)
    mats, probs = [], []
    for G, kt in zip(Gs, kts):
        n = G.shape[0]
        A = G.to(torch.complex128).contiguous().clone()
        d = torch.empty(n, dtype=torch.float64, device=dev)
        e = torch.empty(max(n - 1, 1), dtype=torch.float64, device=dev)
        tau = torch.empty(max(n - 1, 1), dtype=torch.complex128, device=dev)
        w = torch.empty(kt, dtype=torch.float64, device=dev)
        Z = torch.empty((n, kt), dtype=torch.float64, device=dev)
        mats.append((n, kt, A, d, e, tau, w, Z))
        probs.append(HeevProblem(n, kt, _vp(A), _vp(d), _vp(e), _vp(tau), _vp(w), _vp(Z), None))
    ws = _batched_ws(eng, eng.heev_batched_bytes(probs))
    status = torch.zeros(len(Gs), dtype=torch.int32, device=dev)
    eng.heev_batched(probs, status, ws, "top")
    Qs, _ = eng.qr_blocks([Z.flip(1).contiguous() for (_, _, _, _, _, _, _, Z) in mats])
    Ks, checks = [], []
    for i, ((n, kt, A, d, e, tau, w, Z), Q) in enumerate(zip(mats, Qs)):
        TQ = d[:, None] * Q
        if n > 1:
            TQ[:-1] += e[:n - 1, None] * Q[1:]
            TQ[1:] += e[:n - 1, None] * Q[:-1]
        rho = (Q * TQ).sum(dim=0)
        scale = torch.clamp(w.abs().max(), min=torch.finfo(torch.float64).tiny)
        res = torch.nan_to_num((TQ - Q * rho).abs().max() / scale, nan=float("inf"))
        K = Q.to(torch.complex128).contiguous()
        probs[i].k = _vp(K)
        Ks.append(K)
        checks.append(torch.stack([status[i].to(torch.float64), torch.zeros((), dtype=torch.float64, device=dev),
                                   res]))
    eng.heev_batched(probs, status, ws, "back")
    return [(torch.flip(m[6], dims=[0]), K, chk) for m, K, chk in zip(mats, Ks, checks)]
