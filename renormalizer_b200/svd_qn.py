"""Quantum-number blocked SVD / QR and basis selection on the GPU.

Drop-in for renormalizer/mps/svd_qn.py:99-240 (``svd_qn``) and
renormalizer/mps/lib.py:253-322 (``select_basis``).  The coefficient
matrix never leaves HBM: QN blocks are gathered by reno_qn_gather, factorised
on the device in FP64, and the selected singular vectors are scattered
(sigma-weighted where the reference weights them) straight into the new site
tensors by reno_qn_scatter.  Only singular values and QN labels -- a few
thousand numbers -- come to the host, where the truncation rule and the
selection order are decided exactly as in the reference (stable descending
sort of sigma, zero-sigma padding columns last, ``percent`` per QN block).

The dense per-block factorisations run in libreno_b200: the truncation
diagonalises each block's Gram matrix with the device eigensolver (heev.py;
cuSOLVER only redoes a block whose checks fail) and the QR of svd_qn(QR=True)
is the batched Householder QR (reno_qr_blocks).  Padding columns (the
reference's full_matrices=True completion, svd_qn.py:43-63) are an
orthonormal completion drawn from numpy's global RNG like the reference, and
are built only when the selection reaches them.  The stand-alone SVD of
svd_qn(QR=False) (not used by the sweeps) is torch.linalg.svd.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from ._native import Engine, h2d
from . import heev


def add_outer(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """svd_qn.py:305-313"""
    assert a.shape[-1] == b.shape[-1]
    out = np.array([np.add.outer(a[..., i], b[..., i]) for i in range(a.shape[-1])])
    return out.transpose(list(range(1, out.ndim)) + [0])


def qn_sectors(labels: np.ndarray) -> set:
    """set(tuple(row) for row in labels) -- the reference's sector loop order
    (svd_qn.py:183-184) -- built from the distinct rows in first-occurrence
    order, which leaves the set, and so its iteration order, unchanged."""
    labels = np.asarray(labels)
    if labels.shape[0] == 0:
        return set()
    _, first = np.unique(labels, axis=0, return_index=True)
    return set(tuple(int(v) for v in labels[i]) for i in np.sort(first))


def get_qn_mask(qnmat: np.ndarray, qntot) -> np.ndarray:
    """svd_qn.py:316-317"""
    return np.all(qnmat == np.array(qntot), axis=-1)


def _i64(x, device):
    if device.type != "cuda":
        return torch.as_tensor(np.asarray(x, dtype=np.int64), device=device)
    return h2d(x, device, np.int64)


@dataclass
class QNBlock:
    nl: tuple
    nr: tuple
    lset: np.ndarray
    rset: np.ndarray
    U: torch.Tensor          # (m, k)
    S: Optional[np.ndarray]  # (k,) host, None for QR
    S_dev: Optional[torch.Tensor]
    Vh: torch.Tensor         # (k, n)  (reference's block_vt)
    upad: int = 0            # zero-sigma U columns the reference appends
    vpad: int = 0


def _i64_many(arrays, device, float_last=False):
    """several int64 index lists (the last one float64, carried as its bits,
    when ``float_last``) in one host-to-device transfer; returns one device
    view per list"""
    host = [np.asarray(a, dtype=np.int64) for a in (arrays[:-1] if float_last else arrays)]
    if float_last:
        host.append(np.ascontiguousarray(arrays[-1], dtype=np.float64).view(np.int64))
    flat = np.concatenate(host) if host else np.zeros(0, np.int64)
    dev = h2d(flat, device, np.int64) if device.type == "cuda" else torch.as_tensor(flat, device=device)
    out, off = [], 0
    for h in host:
        out.append(dev[off: off + h.size])
        off += h.size
    if float_last:
        out[-1] = out[-1].view(torch.float64)
    return out


def _gather(eng: Engine, mat: torch.Tensor, lset, rset) -> torch.Tensor:
    out = torch.empty((len(lset), len(rset)), dtype=mat.dtype, device=mat.device)
    rows, cols = _i64_many([lset, rset], mat.device)
    eng.qn_gather(mat, rows, cols, out)
    return out


def _pad_counts(m, n, full_matrices=True, opt_full_matrices=True):
    """Zero-sigma columns appended to U and V for one block (svd_qn.py:12-49, 66-86)."""
    if not full_matrices:
        return 0, 0
    dim = min(m, n)
    opt = opt_full_matrices and not (1 / 3 < m / n < 3)
    if not opt:
        return m - dim, n - dim
    if m < n:
        return 0, m
    return n, 0


def qn_block_svd(coef: torch.Tensor, qnbigl, qnbigr, qntot, full_matrices=True, opt_full_matrices=True):
    """Economic SVD of every QN block of coef reshaped to (prod l, prod r)."""
    eng = Engine.get(coef.device)
    rows = int(np.prod(qnbigl.shape[:-1]))
    cols = int(np.prod(qnbigr.shape[:-1]))
    mat = coef.reshape(rows, cols).contiguous()
    qntot = np.asarray(qntot)
    qs = len(qntot)
    lq = qnbigl.reshape(-1, qs)
    rq = qnbigr.reshape(-1, qs)
    blocks: List[QNBlock] = []
    for nl in qn_sectors(lq):
        nr = tuple(qntot - np.array(nl))
        rset = np.where(get_qn_mask(rq, nr))[0]
        if len(rset) == 0:
            continue
        lset = np.where(get_qn_mask(lq, nl))[0]
        blk = _gather(eng, mat, lset, rset)
        U, S, Vh = torch.linalg.svd(blk, full_matrices=False)
        upad, vpad = _pad_counts(len(lset), len(rset), full_matrices, opt_full_matrices)
        blocks.append(QNBlock(nl, nr, lset, rset, U, None, S, Vh, upad, vpad))
    if not blocks:
        raise ValueError("Invalid quantum number")
    Sh = torch.cat([b.S_dev for b in blocks]).cpu().numpy() if blocks else np.zeros(0)
    off = 0
    for b in blocks:
        k = b.S_dev.numel()
        b.S = Sh[off:off + k]
        off += k
    return blocks, rows, cols


def _qr_begin(coef: torch.Tensor, qnbigl, qnbigr, qntot, system: str):
    """The QN blocks of one QR / RQ (qn_block_qr) gathered and, for RQ,
    reversed and conjugate-transposed: (found, rows, cols), found holding
    (nl, nr, lset, rset, block to factorise) per block."""
    if system not in ("L", "R"):
        raise AssertionError("system must be L or R for QR")
    eng = Engine.get(coef.device)
    rows = int(np.prod(qnbigl.shape[:-1]))
    cols = int(np.prod(qnbigr.shape[:-1]))
    mat = coef.reshape(rows, cols).contiguous()
    qntot = np.asarray(qntot)
    qs = len(qntot)
    lq = qnbigl.reshape(-1, qs)
    rq = qnbigr.reshape(-1, qs)
    found = []
    for nl in qn_sectors(lq):
        nr = tuple(qntot - np.array(nl))
        rset = np.where(get_qn_mask(rq, nr))[0]
        if len(rset) == 0:
            continue
        lset = np.where(get_qn_mask(lq, nl))[0]
        blk = _gather(eng, mat, lset, rset)
        if system == "R":
            blk = blk.flip([0, 1]).mH.resolve_conj().contiguous()
        found.append((nl, nr, lset, rset, blk))
    if not found:
        raise ValueError("Invalid quantum number")
    return found, rows, cols


def _qr_end(found, Qs, Rs, system: str):
    blocks = []
    for (nl, nr, lset, rset, _), Q, R in zip(found, Qs, Rs):
        if system == "L":
            blocks.append(QNBlock(nl, nr, lset, rset, Q, None, None, R))
        else:
            blocks.append(QNBlock(nl, nr, lset, rset, R.mH.flip([0, 1]).resolve_conj().contiguous(), None, None,
                                  Q.mH.flip([0, 1]).resolve_conj().contiguous()))
    return blocks


def qn_block_qr(coef: torch.Tensor, qnbigl, qnbigr, qntot, system: str):
    """Per-block QR (system "L") or RQ (system "R"), economic (svd_qn.py:195-204),
    every QN block of the site in one batched Householder QR (reno_qr_blocks,
    LAPACK's sign conventions).  RQ comes from the QR of the reversed
    conjugate transpose: (J A J)^H = Q1 R1 gives A = (J R1^H J)(J Q1^H J), with
    J R1^H J upper triangular.  Householder QR processes the entries in the
    same order as LAPACK's RQ (last row first, pivot on its last entry), so R
    and Q agree with scipy.linalg.rq including the signs, not only up to a
    rotation."""
    found, rows, cols = _qr_begin(coef, qnbigl, qnbigr, qntot, system)
    Qs, Rs = Engine.get(coef.device).qr_blocks([f[4] for f in found])
    return _qr_end(found, Qs, Rs, system), rows, cols


def _scatter(eng: Engine, src: torch.Tensor, rows, scols, dcols, sigma, dst: torch.Tensor, dst_rs, dst_cs):
    """dst[rows[i]*dst_rs + dcols[j]*dst_cs] = sigma_j * src[i, scols[j]] (src: any 2-D view)"""
    if len(rows) == 0 or len(scols) == 0:
        return
    # the kernel does not bound-check its index lists: check them here
    r, c = np.asarray(rows, dtype=np.int64), np.asarray(scols, dtype=np.int64)
    dc = np.asarray(dcols, dtype=np.int64)
    if (len(r) > src.shape[0] or len(dc) != len(c) or c.min() < 0 or c.max() >= src.shape[1] or r.min() < 0
            or dc.min() < 0 or int(r.max()) * dst_rs + int(dc.max()) * dst_cs >= dst.numel()):
        raise IndexError(f"qn scatter out of range: src {tuple(src.shape)}, {len(r)} rows (max {r.max()}), "
                         f"source columns up to {c.max()}, dst {tuple(dst.shape)}")
    dev = dst.device
    if sigma is None:
        ri, ci, di = _i64_many([r, c, dc], dev)
        sig = None
    else:
        ri, ci, di, sig = _i64_many([r, c, dc, sigma], dev, float_last=True)
    eng.qn_scatter(src, ri, ci, di, sig, dst, dst_rs, dst_cs)


def _select_by_code(sset: np.ndarray, codes: np.ndarray, visit: List[int], Mmax: int, percent=0) -> List[int]:
    """select_basis_indices on integer QN codes; ``visit`` lists the codes in
    the order the reference's set(qnlist) iterates the QNs they stand for."""
    n = len(sset)
    nbasis = min(n, Mmax)
    alive = np.ones(n, dtype=bool)
    sidx: List[int] = []
    if percent != 0:
        nbas_block = int(nbasis * percent / len(visit))
        for c in visit:
            cand = np.flatnonzero(alive & (codes == c))
            take = cand[np.argsort(-sset[cand], kind="stable")][:nbas_block]
            alive[take] = False
            sidx += take.tolist()
    nbasis = nbasis - len(sidx)
    cand = np.flatnonzero(alive)
    sidx += cand[np.argsort(-sset[cand], kind="stable")][:nbasis].tolist()
    assert len(sidx) == len(set(sidx))
    return sidx


def select_basis_indices(sset: np.ndarray, qnlist: List[tuple], Mmax: int, percent=0) -> List[int]:
    """The index choice of lib.py:253-298 (select_basis) on host scalars.

    Same order and tie-breaking as the reference's sorted(..., reverse=True)
    over index-ordered dicts (equal sigma keep index order), with the QN
    blocks of the reserved fraction visited in the reference's set order;
    each selection is one stable numpy argsort instead of dict rebuilding."""
    qnlist = [tuple(q) for q in qnlist]
    code = {}
    for q in qnlist:
        code.setdefault(q, len(code))
    codes = np.fromiter((code[q] for q in qnlist), dtype=np.int64, count=len(qnlist))
    return _select_by_code(np.asarray(sset, dtype=np.float64), codes, [code[q] for q in set(qnlist)], Mmax,
                           percent)


def _completion(vecs: torch.Tensor, npad: int) -> torch.Tensor:
    """npad orthonormal columns orthogonal to the columns of vecs (m x k),
    drawn like svd_qn.py:52-63 from numpy's global RNG."""
    m, k = vecs.shape
    eng = Engine.get(vecs.device)
    vecs = vecs.contiguous()
    a = torch.as_tensor(np.random.rand(m, npad), device=vecs.device).to(vecs.dtype)

    def project_out(x):
        return x - eng.matmul(vecs, eng.matmul(vecs.transpose(0, 1), x, conj_a=True))

    q = eng.qr_blocks([project_out(a)])[0][0]
    # second pass for orthogonality to vecs at FP64 rounding level
    return eng.qr_blocks([project_out(q)])[0][0]


class TruncatedSplit:
    """Result of a QN-blocked SVD truncation of a (rows, cols) coefficient:
    ``left`` (rows, m) and ``right`` (m, cols) with left @ right the truncated
    coefficient.  The kept side has orthonormal columns (left) or rows
    (right); the other side carries the singular values."""

    def __init__(self, left, right, qn, mdim, sigma):
        self.left = left
        self.right = right
        self.qn = qn
        self.mdim = mdim
        self.sigma = sigma


class SubspaceOptions:
    """Top-k truncation of large QN blocks by block subspace iteration.

    A block X whose smaller side has at least ``min_dim`` rows, when the
    bond's cap k on the kept dimension is known (``fixed`` criteria), needs
    only its leading k singular triplets: the selection takes at most k from
    any one block and the fixed rule reads only min(k, len(sigma)).  They
    come from ``iters`` + 1 products with X X^H (two FP64 GEMMs each, an
    orthonormalisation in between) on kk = k + oversample columns, a
    Rayleigh-Ritz step on the kk x kk projection and the norms of the
    projected rows.  Acceptance uses the excess discarded weight the Ritz
    basis can carry, estimated from the residuals
    r_i = ||X X^H u_i - lambda_i u_i|| of the leading k as
    sum_i r_i^2 / max(lambda_i - lambda_kk, r_i): it must stay below
    ``rtol`` * ||X||_F^2.  A block that misses it runs ``iters`` + 1 more
    products from its current basis and is checked again; if it still
    misses, it falls back to the full Gram eigendecomposition.
    Off by default (``min_dim = 0``): on the two-site TDVP workload (96 sites,
    M = 256) the Ritz vectors near the cut differ between runs that differ
    only in rounding, and split-precision and FP64 trajectories drifted apart
    by 1.2e-5 in the populations over 8 steps (2e-7 with the full
    decomposition), with 40 % of the blocks needing a retry or the fallback.
    ``orth`` picks the orthonormalisation
    ("householder", or "cholqr": shifted CholeskyQR3, which needs full column
    rank and so fails -- and falls back -- on rank-deficient blocks).
    RENO_SUBSPACE=
    "min_dim,iters,oversample,rtol[,orth]" overrides the defaults."""

    def __init__(self, min_dim=0, iters=3, oversample=64, rtol=1e-13, orth="householder"):
        env = os.environ.get("RENO_SUBSPACE")
        if env:
            parts = env.split(",")
            min_dim, iters, oversample, rtol = int(parts[0]), int(parts[1]), int(parts[2]), float(parts[3])
            if len(parts) > 4:
                orth = parts[4]
        self.orth = orth
        self.min_dim = min_dim
        self.iters = iters
        self.oversample = oversample
        self.rtol = rtol
        self.calls = 0
        self.retries = 0
        self.fallbacks = 0


subspace = SubspaceOptions()


class RefineOptions:
    """Second pass for the small singular values of a block.

    The Gram matrix carries absolute rounding errors of about eps ||X||^2, so
    its eigenvectors for sigma below ~sqrt(eps) ||X|| are mixed within that
    cluster, and the projected norms ||u^H X|| of such mixtures lie anywhere
    in the cluster's range.  When the truncation's cut (the smallest selected
    sigma) lies below 2 ``tau`` times the largest sigma, every block whose
    projected sigma include values below ``tau`` times its own largest is
    refined: its cluster rows of P (sigma-scaled singular vectors, mutually
    orthogonal to within eps sigma_i sigma_j) are projected twice onto the
    complement of its other rows, the small Gram matrix of what remains
    (entries of order sigma_cluster^2, accurate to eps relative) goes through
    the device eigensolver, and its eigenvectors rotate the cluster's kept
    basis and rows (K P is unchanged).  The refined sigma are accurate to
    about sqrt(eps) tau ||X|| instead of sqrt(eps) ||X||, and the kept
    vectors at such a cut are the true singular vectors (the reference's
    gesdd choice): without the pass, an imaginary-time TDVP-PS2 step of a
    density operator whose cut sits at 1e-7 moved its energy by 4e-8 against
    the reference, with it by 3e-14.

    Compressions (bond expansion, canonical compress) refine however small
    the cut's weight: which directions they keep at a cut of weight 1e-20
    (the 1e-10 bond expansion of a start state) sets the bond space that
    one-site TDVP then evolves in, and with the Gram eigenvectors' choice
    there a TDVP-PS density-operator trajectory left the reference's by 2e-4.
    The two-site sweeps pass ``sweep_floor`` (default 0: refine at any
    weight): a cut below that fraction of the largest sigma is left as the
    Gram eigenvectors give it.  With 1e-9 the 96-site TDVP-PS2 bench ran fewer
    passes (241 against 376 in two steps) yet took 17.4 s per step instead of
    13.6 (truncation 14.1 s against 10.4; single runs on different machines
    of the same kind).  The directions kept at such cuts carry the QN labels
    of the next bond, so they shape the QN blocks of later truncations, which
    is the likely route.  ``tau`` = 0 turns the pass off."""

    def __init__(self, tau=1e-6, sweep_floor=0.0):
        env = os.environ.get("RENO_REFINE_TAU")
        self.tau = float(env) if env else tau
        self.sweep_floor = sweep_floor
        self.calls = 0
        self.blocks = 0


refine = RefineOptions()
# eigenpairs computed beyond a block's fixed cap k (a block contributes at most
# k entries to the selection; the others only fill the list the rule reads).
# RENO_TOP_MARGIN overrides it.
TOP_MARGIN = int(os.environ.get("RENO_TOP_MARGIN", "64"))
# when a list, svd_truncate appends the algorithmic FP64 flops of each call's
# block factorisations (see _block_flops)
flop_log = None


def _block_flops(m, n, k, cplx):
    """Gram 8 s^2 l, tridiagonal reduction 16/3 s^3, back-transformation
    8 s^2 k, projection 8 s l k for a block with smaller / larger side s / l
    and k eigenvectors used (complex counts; a real block a quarter)"""
    s, l = min(m, n), max(m, n)
    f = 8.0 * s * s * l + 16.0 / 3.0 * s ** 3 + 8.0 * s * s * k + 8.0 * s * l * k
    return f if cplx else f / 4.0
_OMEGA = {}


def _omega(rows, kk, dtype, device):
    """a fixed seeded Gaussian start block per shape (deterministic runs)"""
    key = (rows, kk, dtype, str(device))
    om = _OMEGA.get(key)
    if om is None:
        if len(_OMEGA) > 64:
            _OMEGA.clear()
        g = torch.Generator(device=device).manual_seed(0x5EED + 7919 * rows + kk)
        om = torch.randn((rows, kk), dtype=torch.float64, device=device, generator=g)
        if dtype.is_complex:
            om = torch.complex(om, torch.randn((rows, kk), dtype=torch.float64, device=device, generator=g))
        _OMEGA[key] = om
    return om


def _orthonormalise(eng: Engine, Y: torch.Tensor, method: str) -> torch.Tensor:
    """An orthonormal basis of the columns of Y (r x kk, r >= kk).

    "householder": the engine's Householder QR.  "cholqr": shifted CholeskyQR3 (Fukaya,
    Kannan, Nakatsukasa, Yamamoto, Yanagisawa, SIAM J. Sci. Comput. 2020): one
    Cholesky QR of the Gram matrix shifted by 11 (r kk + kk (kk + 1)) u tr(G),
    which keeps it positive definite for any column rank, then two plain
    Cholesky QR passes that restore orthonormality to rounding level -- three
    kk x kk Gram GEMMs, Cholesky factorisations and triangular solves, with no
    host synchronisation."""
    if method == "householder":
        return eng.qr_blocks([Y.contiguous()])[0][0]
    r, kk = Y.shape
    u = np.finfo(np.float64).eps / 2
    for shifted in (True, False, False):
        G = eng.matmul(Y.transpose(0, 1), Y, conj_a=True)
        if shifted:
            tr = torch.diagonal(G).real.sum()
            G.diagonal().add_((11.0 * (r * kk + kk * (kk + 1)) * u * tr).to(G.dtype))
        Lc, _ = torch.linalg.cholesky_ex(G)
        Y = torch.linalg.solve_triangular(Lc.transpose(0, 1).conj(), Y, upper=True, left=False)
    return Y


def _topk_kept_side(eng: Engine, A: torch.Tensor, k: int, opts: SubspaceOptions, Q=None, iters=None):
    """Leading k left singular vectors of A (r x c, any 2-D view) by block
    subspace iteration, from the seeded Gaussian block or from a previous
    call's basis Q.  Returns K (r x k, descending), P = K^H A (k x c),
    S (k, device: row norms of P), a device pair (excess-weight estimate,
    ||A||_F^2) for the acceptance test, and the iterated basis Q."""
    r = A.shape[0]
    kk = min(k + opts.oversample, r)
    if Q is None:
        Q = _omega(r, kk, A.dtype, A.device)
        iters = opts.iters + 1
    for _ in range(iters):
        Y = eng.matmul(A, eng.matmul(A.transpose(0, 1), Q, conj_a=True))
        Q = _orthonormalise(eng, Y, opts.orth)
    B = eng.matmul(Q.transpose(0, 1), A, conj_a=True)          # kk x c
    T = eng.matmul(B, B.transpose(0, 1), conj_b=True)          # kk x kk
    w, W = torch.linalg.eigh(T)                                 # ascending
    Wk = torch.flip(W[:, kk - k:], dims=[1])
    lam = torch.flip(w[kk - k:], dims=[0])
    K = eng.matmul(Q, Wk)                                       # r x k
    P = eng.matmul(Wk.transpose(0, 1), B, conj_a=True)         # k x c
    AP = eng.matmul(A, P.transpose(0, 1), conj_b=True)          # A A^H K
    res = torch.linalg.vector_norm(AP - K * lam.to(K.dtype), dim=0)
    gap = torch.maximum(lam - w[0], res)
    excess = torch.sum(res * res / torch.clamp(gap, min=1e-300))
    fro2 = torch.linalg.vector_norm(A) ** 2
    S = torch.linalg.vector_norm(P, dim=1)
    return K, P, S, torch.stack([excess, fro2]), Q


def _subspace_block(eng, X, keep_left, k, opts, Q=None, iters=None):
    """_topk_kept_side on the kept side of block X: (K, P, S, check, Q) with
    P = sigma Vh (keep_left) or U sigma (keep right)."""
    if keep_left:
        return _topk_kept_side(eng, X, k, opts, Q, iters)
    K, Ph, S, chk, Q = _topk_kept_side(eng, X.transpose(0, 1).conj(), k, opts, Q, iters)
    return K, Ph.transpose(0, 1).conj().resolve_conj(), S, chk, Q


def _gram_eigh(eng: Engine, G: torch.Tensor, kt: int, use_heev: bool):
    """Eigenpairs of the Gram matrix G, descending: (w, V, check).  With the
    device eigensolver (``heev.heev_opts``) only the leading kt are computed
    (w has kt entries) and check is its device-side acceptance triple;
    otherwise cuSOLVER's full decomposition and check None."""
    n = G.shape[0]
    if use_heev and heev.heev_opts.enabled and kt < n and n >= heev.heev_opts.min_n and G.is_cuda:
        w, V, chk = heev.heev_top(eng, G, kt)
        if not G.is_complex():
            V = V.real.contiguous()
        return w, V, chk
    w, V = torch.linalg.eigh(G)
    return torch.flip(w, dims=[0]), torch.flip(V, dims=[1]), None


def _gram_of(eng: Engine, X: torch.Tensor, keep_left: bool):
    """(G, left) with G the Gram matrix of X's smaller side, X X^H (left) or
    X^H X; a square block takes the kept side."""
    m, n = X.shape
    if m < n or (m == n and keep_left):
        return eng.matmul(X, X.transpose(0, 1), conj_b=True), True
    return eng.matmul(X.transpose(0, 1), X, conj_a=True), False


def _finish_kept_side(eng: Engine, X: torch.Tensor, keep_left: bool, kt: int, w, E, chk, qr_out=None):
    """Kept-side basis K, projection P and sigma S of block X from the
    leading kt eigenvectors E of its smaller-side Gram matrix (w descending):
    see _full_kept_side.  When the kept side is the larger one, the projected
    vectors are orthonormalised by Householder QR; ``qr_out`` carries that QR
    (computed for all blocks at once) and is None on the first pass, which
    returns the matrix to factorise instead."""
    m, n = X.shape
    dim = min(m, n)

    def tail(w_desc, head):
        # only the leading kt eigenvalues may be known: the others then read
        # as 0, which the cap below reaches anyway
        t = torch.sqrt(torch.clamp(w_desc[kt:dim], min=0.0)) if w_desc.numel() >= dim else \
            torch.zeros(dim - kt, dtype=torch.float64, device=head.device)
        return torch.minimum(t, head.min()) if kt < dim and head.numel() else t

    if keep_left and m <= n:
        K = E[:, :kt]
        P = eng.matmul(K.transpose(0, 1).contiguous(), X, conj_a=True)       # (kt, n) = sigma Vh
        S = torch.linalg.vector_norm(P, dim=1)
        return dict(K=K, P=P, S=torch.cat([S, tail(w, S)]), dim=dim, chk=chk)
    if not keep_left and n <= m:
        K = E[:, :kt]
        P = eng.matmul(X, K.contiguous())                                     # (m, kt) = U sigma
        S = torch.linalg.vector_norm(P, dim=0)
        return dict(K=K, P=P, S=torch.cat([S, tail(w, S)]), dim=dim, chk=chk)
    if keep_left:
        Us = eng.matmul(X, E[:, :kt].contiguous())                            # (m, kt) = U sigma
        if qr_out is None:
            return dict(need_qr=Us)
        S = torch.linalg.vector_norm(Us, dim=0)
        K = qr_out
        P = eng.matmul(K.transpose(0, 1).contiguous(), X, conj_a=True)
        return dict(K=K, P=P, S=torch.cat([S, tail(w, S)]), dim=dim, chk=chk)
    Vs = eng.matmul(X.transpose(0, 1), E[:, :kt].contiguous(), conj_a=True)   # (n, kt): sigma v
    if qr_out is None:
        return dict(need_qr=Vs)
    S = torch.linalg.vector_norm(Vs, dim=0)
    K = qr_out
    P = eng.matmul(X, K)
    return dict(K=K, P=P, S=torch.cat([S, tail(w, S)]), dim=dim, chk=chk)


def _device_eig_ok(G: torch.Tensor) -> bool:
    """whether the device eigensolver takes Gram block G (size 1 .. 4096)"""
    n = G.shape[0]
    return heev.heev_opts.enabled and G.is_cuda and heev.heev_opts.min_n <= n <= 4096


def _kept_sides(eng: Engine, Xs, keep_left: bool, ktops, use_heev: bool = True) -> list:
    """_full_kept_side for all QN blocks of one truncation: one Gram matrix
    per block, the device eigensolver on all of them at once
    (heev_top_batched; blocks above its size limit, or with the device
    eigensolver switched off, take cuSOLVER), and one batched Householder QR
    where a projected basis needs orthonormalising."""
    items = []
    for X, ktop in zip(Xs, ktops):
        m, n = X.shape
        dim = min(m, n)
        kt = dim if ktop is None else min(int(ktop), dim)
        G, _ = _gram_of(eng, X, keep_left)
        items.append(dict(X=X, G=G, kt=kt, dim=dim))
    dev_idx = [i for i, it in enumerate(items) if use_heev and _device_eig_ok(it["G"])]
    if dev_idx:
        res = heev.heev_top_batched(eng, [items[i]["G"] for i in dev_idx], [items[i]["kt"] for i in dev_idx])
        for i, (w, K, chk) in zip(dev_idx, res):
            items[i].update(w=w, E=K if items[i]["G"].is_complex() else K.real.contiguous(), chk=chk)
    for it in items:
        if "E" not in it:
            w, V = torch.linalg.eigh(it["G"])
            it.update(w=torch.flip(w, dims=[0]), E=torch.flip(V, dims=[1]), chk=None)
    outs = [_finish_kept_side(eng, it["X"], keep_left, it["kt"], it["w"], it["E"], it["chk"]) for it in items]
    need = [i for i, o in enumerate(outs) if "need_qr" in o]
    if need:
        Qs, _ = eng.qr_blocks([outs[i]["need_qr"] for i in need])
        for i, Q in zip(need, Qs):
            it = items[i]
            outs[i] = _finish_kept_side(eng, it["X"], keep_left, it["kt"], it["w"], it["E"], it["chk"], Q)
    return outs


def _full_kept_side(eng: Engine, X: torch.Tensor, keep_left: bool, ktop: Optional[int] = None,
                    use_heev: bool = True) -> dict:
    """Kept-side basis K, projection P and sigma S of one block from the
    Hermitian eigendecomposition of the Gram matrix of its smaller side (all
    min(m, n) triplets).

    With ``ktop`` < min(m, n) (a fixed cap on the kept dimension is known and
    the block is larger) only the leading ktop singular vectors are projected:
    P has ktop rows/columns and the other sigma come from the Gram
    eigenvalues, sqrt(max(lambda, 0)), capped at the smallest projected
    sigma.  The cap matters: below sqrt(eps) ||X|| the Gram eigenvalues are
    rounding noise, so an uncapped tail value (~1e-8 ||X||) can exceed the
    true, projected sigma of the head (1e-10 and below in a nearly product
    state) and be selected although it has no projection.  Capped, every tail
    entry sorts after every head entry of its block, and since a block
    contributes at most the cap (< ktop) entries, none is selected; they only
    fill the list the truncation rule reads."""
    return _kept_sides(eng, [X], keep_left, [ktop], use_heev)[0]


def svd_truncate(coef: torch.Tensor, qnbigl, qnbigr, qntot, keep_left: bool, m_trunc_fn, percent=0,
                 full_matrices=True, kcap: Optional[int] = None, refine_floor: float = 0.0):
    """Fused svd_qn + compute_m_trunc + select_basis of mp.py:693-778.

    keep_left=True keeps U (left-to-right sweep: left = U, right = sigma Vh);
    otherwise V is kept (left = U sigma, right = Vh).  Per QN block X the
    kept side comes from the Hermitian eigendecomposition of its Gram matrix
    (X X^H for U, X^H X for V; FP64 GEMM + cuSOLVER), which also supplies the
    zero-sigma completion columns the reference appends with
    full_matrices=True (svd_qn.py:12-86).  The singular values used for
    ordering and truncation are the norms of the projected rows/columns
    (||u_j^H X|| or ||X v_j||), which stay accurate far below sqrt(eps).

    ``kcap`` (the bond's fixed cap on the kept dimension, None when the rule
    is threshold-based) lets large blocks use the top-k subspace solver
    (``subspace`` options); its residual norms come to the host with the
    singular values and a block whose Ritz pairs miss the tolerance is redone
    with the full decomposition.

    ``refine_floor``: a cut below this fraction of the largest sigma skips the
    small-sigma refinement (RefineOptions) unless every entry is kept."""
    st = _trunc_begin(coef, qnbigl, qnbigr, qntot, keep_left, m_trunc_fn, percent, full_matrices, kcap,
                      refine_floor)
    _trunc_eig([st])
    host = torch.cat(_trunc_host_tensors(st)).cpu().numpy()
    return _trunc_end(st, host)


def svd_truncate_batch(calls) -> List["TruncatedSplit"]:
    """svd_truncate for several independent coefficients at once (the
    truncations of lockstep realisations, evolve_batch): every QN block of
    every call goes through one batched device eigensolver pass (per kept
    side) and their singular values and checks reach the host in one
    transfer.  ``calls`` holds svd_truncate's keyword arguments; each result
    equals that call's own svd_truncate."""
    states = [_trunc_begin(**c) for c in calls]
    _trunc_eig(states)
    parts = [_trunc_host_tensors(st) for st in states]
    lens = [sum(t.numel() for t in p) for p in parts]
    host = torch.cat([t for p in parts for t in p]).cpu().numpy()
    sels, off = [], 0
    for st, n in zip(states, lens):
        sels.append(_trunc_select(st, host[off:off + n]))
        off += n
    # the small-sigma refinements of every call that asks for one: one pass
    need = [i for i, sel in enumerate(sels) if sel["refine"]]
    if need:
        hit = _refine_groups(states[0]["eng"], [(states[i]["blocks"], states[i]["keep_left"]) for i in need])
        for i, h in zip(need, hit):
            if h:
                sels[i]["sig"], sels[i]["sidx"] = sels[i]["select"]()
    return [_trunc_place(st, sel) for st, sel in zip(states, sels)]


def _trunc_begin(coef, qnbigl, qnbigr, qntot, keep_left, m_trunc_fn, percent=0, full_matrices=True, kcap=None,
                 refine_floor=0.0):
    """Gather the QN blocks of one truncation (the subspace blocks, when that
    opt-in route applies, are factorised here)."""
    eng = Engine.get(coef.device)
    rows = int(np.prod(qnbigl.shape[:-1]))
    cols = int(np.prod(qnbigr.shape[:-1]))
    mat = coef.reshape(rows, cols).contiguous()
    qntot = np.asarray(qntot)
    qs = len(qntot)
    lq = qnbigl.reshape(-1, qs)
    rq = qnbigr.reshape(-1, qs)
    blocks = []
    pending = []
    for nl in qn_sectors(lq):
        nr = tuple(qntot - np.array(nl))
        rset = np.where(get_qn_mask(rq, nr))[0]
        if len(rset) == 0:
            continue
        lset = np.where(get_qn_mask(lq, nl))[0]
        X = _gather(eng, mat, lset, rset)
        m, n = X.shape
        dim = min(m, n)
        upad, vpad = _pad_counts(m, n, full_matrices)
        ksub = min(kcap, dim) if kcap is not None else 0
        npad = upad if keep_left else vpad
        if (subspace.min_dim and kcap is not None and dim >= subspace.min_dim
                and dim >= 2 * (ksub + subspace.oversample)):
            subspace.calls += 1
            K, P, S, chk, Q = _subspace_block(eng, X, keep_left, ksub, subspace)
            blocks.append(dict(nl=nl, nr=nr, lset=lset, rset=rset, K=K, P=P, S=S, dim=ksub, npad=npad, res=chk,
                               X=X, Q=Q))
            continue
        ktop = kcap + TOP_MARGIN if kcap is not None and kcap + TOP_MARGIN < dim else None
        blk = dict(nl=nl, nr=nr, lset=lset, rset=rset, dim=dim, npad=npad, X=X, ktop=ktop)
        blocks.append(blk)
        pending.append(blk)
    if not blocks:
        raise ValueError("Invalid quantum number")
    return dict(eng=eng, coef=coef, rows=rows, cols=cols, keep_left=keep_left, m_trunc_fn=m_trunc_fn,
                refine_floor=refine_floor,
                percent=percent, blocks=blocks, pending=pending)


def _trunc_eig(states):
    """Kept sides of the pending blocks of every state: one _kept_sides pass
    per kept side over all of them."""
    for keep_left in (True, False):
        group = [b for st in states if st["keep_left"] == keep_left for b in st["pending"]]
        if not group:
            continue
        if flop_log is not None:
            for b in group:
                m_, n_ = b["X"].shape
                flop_log.append(_block_flops(m_, n_, b["ktop"] or min(m_, n_), b["X"].is_complex()))
        fulls = _kept_sides(states[0]["eng"], [b["X"] for b in group], keep_left, [b["ktop"] for b in group])
        for b, full in zip(group, fulls):
            b.update(K=full["K"], P=full["P"], S=full["S"])
            if full["chk"] is not None:
                b["chk"] = full["chk"]
            else:
                b.pop("X")


def _trunc_host_tensors(st):
    """The device values the host needs: every block's sigma, the subspace
    residual pairs and the device eigensolver's check triples."""
    blocks = st["blocks"]
    return [b["S"] for b in blocks] + [b["res"] for b in blocks if "res" in b] + \
        [b["chk"] for b in blocks if "chk" in b]


def _refine_clusters(eng: Engine, blocks, keep_left: bool) -> bool:
    """The RefineOptions pass over the blocks of one truncation (host sigma
    ``Sh`` already known): all cluster Gram matrices in one device
    eigensolver call, their checks and refined sigma in one host transfer.
    Returns whether any block was refined."""
    return _refine_groups(eng, [(blocks, keep_left)])[0]


def _refine_groups(eng: Engine, groups) -> List[bool]:
    """_refine_clusters for several truncations at once (groups of (blocks,
    keep_left)): the cluster Gram matrices of all of them in one device
    eigensolver call and one host transfer.  Returns per group whether any of
    its blocks was refined."""
    todo = []
    for g, (blocks, keep_left) in enumerate(groups):
        for b in blocks:
            t = _refine_prepare(eng, b, keep_left)
            if t is not None:
                t["g"] = g
                todo.append(t)
    if not todo:
        return [False] * len(groups)
    _refine_apply(eng, todo)
    hit = set(t["g"] for t in todo)
    return [g in hit for g in range(len(groups))]


def _refine_prepare(eng: Engine, b, keep_left: bool):
    """the projected cluster Gram matrix of block b, or None when b has no
    cluster below the refinement threshold"""
    kt = b["K"].shape[1]
    head = np.asarray(b["Sh"][:kt], dtype=np.float64)
    if kt < 2 or not np.all(np.isfinite(head)) or head.max() <= 0:
        return None
    cl = np.nonzero(head < refine.tau * head.max())[0]
    if len(cl) == 0:
        return None
    lg = np.nonzero(head >= refine.tau * head.max())[0]
    dev = b["S"].device
    ic, il = _i64(cl, dev), _i64(lg, dev)
    Z = b["P"] if keep_left else b["P"].transpose(0, 1).conj()
    Zc, Zl = Z.index_select(0, ic), Z.index_select(0, il)
    sl2 = b["S"].index_select(0, il) ** 2
    for _ in range(2):
        coef = eng.matmul(Zc, Zl.transpose(0, 1), conj_b=True) / sl2[None, :]
        Zc = Zc - eng.matmul(coef, Zl)
    C = eng.matmul(Zc, Zc.transpose(0, 1), conj_b=True)
    scale = torch.clamp(torch.diagonal(C).real.sum(), min=1e-300)
    return dict(b=b, cl=cl, ic=ic, C=(C / scale).contiguous(), scale=scale, keep_left=keep_left)


def _refine_apply(eng: Engine, todo):
    refine.calls += len(set(t.get("g", 0) for t in todo))  # truncations refined
    refine.blocks += len(todo)
    dev_idx = [i for i, t in enumerate(todo) if _device_eig_ok(t["C"])]
    if dev_idx:
        res = heev.heev_top_batched(eng, [todo[i]["C"] for i in dev_idx], [len(todo[i]["cl"]) for i in dev_idx])
        for i, (w, R, chk) in zip(dev_idx, res):
            todo[i].update(w=w, R=R if todo[i]["C"].is_complex() else R.real.contiguous(), chk=chk)
    for t in todo:
        if "R" not in t:
            w, V = torch.linalg.eigh(t["C"])
            t.update(w=torch.flip(w, dims=[0]), R=torch.flip(V, dims=[1]))
        t["sig"] = torch.sqrt(torch.clamp(t["w"] * t["scale"], min=0.0))
    host = torch.cat([t["sig"] for t in todo] + [t["chk"] for t in todo if "chk" in t]).cpu().numpy()
    off = sum(len(t["cl"]) for t in todo)
    for t in todo:
        if "chk" in t:
            if not heev.accepted(host[off:off + 3]):
                heev.heev_opts.fallbacks += 1
                w, V = torch.linalg.eigh(t["C"])
                t.update(R=torch.flip(V, dims=[1]))
                t["sig"] = torch.sqrt(torch.clamp(torch.flip(w, dims=[0]) * t["scale"], min=0.0))
                t["sig_h"] = t["sig"].cpu().numpy()
            off += 3
    off = 0
    for t in todo:
        b, ic, R, keep_left = t["b"], t["ic"], t["R"], t["keep_left"]
        c = len(t["cl"])
        sig_h = t.get("sig_h", host[off:off + c])
        off += c
        b["K"][:, ic] = eng.matmul(b["K"].index_select(1, ic), R)
        if keep_left:
            b["P"][ic] = eng.matmul(R.transpose(0, 1), b["P"].index_select(0, ic), conj_a=True)
        else:
            b["P"][:, ic] = eng.matmul(b["P"].index_select(1, ic), R)
        b["S"][ic] = t["sig"]
        Sh = np.array(b["Sh"], dtype=np.float64, copy=True)
        Sh[t["cl"]] = sig_h
        kt = b["K"].shape[1]
        if len(Sh) > kt:
            # unprojected tail values stay below every projected one
            Sh[kt:] = np.minimum(Sh[kt:], Sh[:kt].min())
        b["Sh"] = Sh


def _trunc_select(st, host):
    """Checks (redo of failed blocks) and the reference's selection, from the
    host copy of _trunc_host_tensors; says whether the cut asks for the
    small-sigma refinement."""
    eng = st["eng"]
    keep_left, m_trunc_fn, percent, blocks = st["keep_left"], st["m_trunc_fn"], st["percent"], st["blocks"]
    sub = [b for b in blocks if "res" in b]
    dev_eig = [b for b in blocks if "chk" in b]
    off = 0
    for b in blocks:
        b["Sh"] = host[off:off + b["dim"]]
        off += b["dim"]
    off_chk = off + 2 * len(sub)
    for i, b in enumerate(dev_eig):
        if not heev.accepted(host[off_chk + 3 * i: off_chk + 3 * i + 3]):
            # the device eigensolver missed its checks on this block: cuSOLVER
            heev.heev_opts.fallbacks += 1
            b.update(_full_kept_side(eng, b["X"], keep_left, b["ktop"], use_heev=False))
            b["Sh"] = b["S"].cpu().numpy()
        b.pop("X", None)
        b.pop("chk", None)
    ok = lambda e, f: bool(np.isfinite(e) and e <= subspace.rtol * f)
    retry = []
    for b in sub:
        if not ok(host[off], host[off + 1]):
            retry.append(b)
        off += 2
    if retry:
        # continue those blocks' iteration from their current basis, check once
        # more, then fall back to the full decomposition
        for b in retry:
            subspace.retries += 1
            b["K"], b["P"], b["S"], b["res"], b["Q"] = _subspace_block(eng, b["X"], keep_left, b["dim"], subspace,
                                                                       b["Q"], subspace.iters + 1)
        host2 = torch.cat([t for b in retry for t in (b["S"], b["res"])]).cpu().numpy()
        off = 0
        for b in retry:
            b["Sh"] = host2[off:off + b["dim"]]
            e, f = host2[off + b["dim"]], host2[off + b["dim"] + 1]
            off += b["dim"] + 2
            if not ok(e, f):
                subspace.fallbacks += 1
                b.update(_full_kept_side(eng, b["X"], keep_left))
                b["Sh"] = b["S"].cpu().numpy()
    for b in sub:
        b.pop("X", None)
        b.pop("Q", None)
    # the reference's concatenated order: nonzero parts block by block, then
    # the zero-sigma paddings block by block (svd_qn.py:222-230)
    # (entry -> block bi, position j); block bi's QN is its code: the blocks'
    # sectors are distinct and appear in block order
    blk = np.concatenate([np.full(b["dim"], bi, dtype=np.int64) for bi, b in enumerate(blocks)] +
                         [np.full(b["npad"], bi, dtype=np.int64) for bi, b in enumerate(blocks)])
    pos = np.concatenate([np.arange(b["dim"], dtype=np.int64) for b in blocks] +
                         [b["dim"] + np.arange(b["npad"], dtype=np.int64) for b in blocks])
    qkey = [tuple(b["nl"] if keep_left else b["nr"]) for b in blocks]
    code_of = {q: bi for bi, q in enumerate(qkey)}
    # the reference iterates set(qnlist) over the per-entry QN list in entry
    # order, where a block without nonzero entries first appears among the
    # paddings; inserting the distinct QNs in first-occurrence order builds
    # the same set (duplicates leave a set's table unchanged)
    _, first = np.unique(blk, return_index=True)
    visit_set = set(qkey[int(blk[i])] for i in np.sort(first))

    def select():
        sig = np.concatenate([np.asarray(b["Sh"][:b["dim"]], dtype=np.float64) for b in blocks] +
                             [np.zeros(b["npad"]) for b in blocks])
        return sig, _select_by_code(sig, blk, [code_of[q] for q in visit_set], m_trunc_fn(sig), percent)

    sig, sidx = select()
    keeps_all = len(sidx) >= sum(b["dim"] for b in blocks)
    wants = bool(refine.tau > 0 and len(sidx) and sig.max() > 0 and sig[sidx].min() < 2 * refine.tau * sig.max()
                 and (keeps_all or sig[sidx].min() >= st["refine_floor"] * sig.max()))
    return dict(select=select, sig=sig, sidx=sidx, refine=wants, blk=blk, pos=pos, qkey=qkey)


def _trunc_end(st, host):
    """_trunc_select, the small-sigma refinement where the cut asks for it
    and the scatter of the kept columns (_trunc_place)."""
    sel = _trunc_select(st, host)
    if sel["refine"] and _refine_clusters(st["eng"], st["blocks"], st["keep_left"]):
        sel["sig"], sel["sidx"] = sel["select"]()
    return _trunc_place(st, sel)


def _trunc_place(st, sel):
    """The kept columns of the selection scattered into the new left / right
    tensors (completion columns drawn where selected)."""
    eng, coef, rows, cols = st["eng"], st["coef"], st["rows"], st["cols"]
    keep_left, blocks = st["keep_left"], st["blocks"]
    sig, sidx, blk, pos, qkey = sel["sig"], sel["sidx"], sel["blk"], sel["pos"], sel["qkey"]
    mdim = len(sidx)
    left = torch.zeros((rows, mdim), dtype=coef.dtype, device=coef.device)
    right = torch.zeros((mdim, cols), dtype=coef.dtype, device=coef.device)
    per_block = {}
    for out_col, (bi, j) in enumerate(zip(blk[sidx].tolist(), pos[sidx].tolist())):
        per_block.setdefault(bi, ([], []))
        per_block[bi][0].append(j)
        per_block[bi][1].append(out_col)
    for bi, (kc, oc) in per_block.items():
        b = blocks[bi]
        if max(kc) >= b["K"].shape[1]:
            # completion columns beyond the computed basis: orthonormal, drawn like
            # svd_qn.py:52-63 from numpy's global RNG, built only when selected
            b["K"] = torch.cat([b["K"], _completion(b["K"], max(kc) + 1 - b["K"].shape[1])], dim=1)
        nz = [(j, o) for j, o in zip(kc, oc) if j < b["dim"]]
        if keep_left:
            # left[lset[i], out] = K[i, j] (kept basis incl. completion columns)
            _scatter(eng, b["K"], b["lset"], kc, oc, None, left, mdim, 1)
            if nz:
                # right[out, rset[i]] = P[j, i]  (= sigma_j Vh[j, i]); completion rows stay 0
                _scatter(eng, b["P"].transpose(0, 1), b["rset"], [j for j, _ in nz], [o for _, o in nz], None, right,
                         1, cols)
        else:
            # right[out, rset[i]] = conj(K[i, j]) : the reference's v = Vt.T rows
            _scatter(eng, b["K"].conj().resolve_conj() if b["K"].is_complex() else b["K"], b["rset"], kc, oc, None,
                     right, 1, cols)
            if nz:
                _scatter(eng, b["P"], b["lset"], [j for j, _ in nz], [o for _, o in nz], None, left, mdim, 1)
    qn_new = np.array([qkey[bi] for bi in blk[sidx].tolist()]).reshape(mdim, -1)
    return TruncatedSplit(left, right, qn_new, mdim, sig[sidx])


def qr_split(coef: torch.Tensor, qnbigl, qnbigr, qntot, system: str):
    """svd_qn(QR=True, full_matrices=False) of mp.py:890-908 / mps.py:1318-1327:
    returns (u (rows, k), qnl list, vt (k, cols), qnr list) as device tensors."""
    blocks, rows, cols = qn_block_qr(coef, qnbigl, qnbigr, qntot, system)
    return _qr_assemble(blocks, rows, cols, coef)


def qr_split_batch(calls):
    """qr_split for several independent calls (keyword dicts of qr_split), the
    QN blocks of all of them in shared batched QR launches (lockstep
    realisations); every result is that call's own qr_split."""
    begun = [_qr_begin(**c) for c in calls]
    mats = [f[4] for found, _, _ in begun for f in found]
    if not mats:
        return []
    Qs, Rs = Engine.get(mats[0].device).qr_blocks(mats)
    out, off = [], 0
    for c, (found, rows, cols) in zip(calls, begun):
        k = len(found)
        blocks = _qr_end(found, Qs[off:off + k], Rs[off:off + k], c["system"])
        off += k
        out.append(_qr_assemble(blocks, rows, cols, c["coef"]))
    return out


def _qr_assemble(blocks, rows, cols, coef):
    eng = Engine.get(coef.device)
    ks = [min(len(b.lset), len(b.rset)) for b in blocks]
    ktot = sum(ks)
    u = torch.zeros((rows, ktot), dtype=coef.dtype, device=coef.device)
    vt = torch.zeros((ktot, cols), dtype=coef.dtype, device=coef.device)
    qnl, qnr = [], []
    off = 0
    for b, k in zip(blocks, ks):
        cidx = list(range(k))
        out = list(range(off, off + k))
        _scatter(eng, b.U, b.lset, cidx, out, None, u, ktot, 1)
        # vt rows: dst (row=off+j, col=rset[i]) <- Vh[j, i]
        _scatter(eng, b.Vh.transpose(0, 1), b.rset, cidx, out, None, vt, 1, cols)
        qnl += [b.nl] * k
        qnr += [b.nr] * k
        off += k
    return u, qnl, vt, qnr


def svd_qn(coef_array, qnbigl, qnbigr, qntot, QR=False, system=None, full_matrices=True, opt_full_matrices=True):
    """Drop-in for svd_qn.py:99-240 with device tensors.  Returns
    (u, su, qnl, v, sv, qnr) or (u, qnl, v, qnr) for QR like the reference."""
    from .hop_expr import as_device
    coef = as_device(coef_array)
    if QR:
        u, qnl, vt, qnr = qr_split(coef, qnbigl, qnbigr, qntot, system)
        return u, qnl, vt.transpose(0, 1), qnr
    blocks, rows, cols = qn_block_svd(coef, qnbigl, qnbigr, qntot, full_matrices, opt_full_matrices)
    eng = Engine.get(coef.device)
    ucols = [b.S.size for b in blocks] + [b.upad for b in blocks]
    vcols = [b.S.size for b in blocks] + [b.vpad for b in blocks]
    u = torch.zeros((rows, sum(ucols)), dtype=coef.dtype, device=coef.device)
    v = torch.zeros((cols, sum(vcols)), dtype=coef.dtype, device=coef.device)
    su, sv, qnl, qnr = [], [], [], []
    off = 0
    for b in blocks:
        k = b.S.size
        _scatter(eng, b.U, b.lset, list(range(k)), list(range(off, off + k)), None, u, u.shape[1], 1)
        _scatter(eng, b.Vh.transpose(0, 1), b.rset, list(range(k)), list(range(off, off + k)), None, v,
                 v.shape[1], 1)
        su.append(b.S)
        sv.append(b.S)
        qnl += [b.nl] * k
        qnr += [b.nr] * k
        off += k
    uo, vo = off, off
    for b in blocks:
        if b.upad:
            pad = _completion(b.U, b.upad)
            _scatter(eng, pad, b.lset, list(range(b.upad)), list(range(uo, uo + b.upad)), None, u, u.shape[1], 1)
            uo += b.upad
        su.append(np.zeros(b.upad))
        qnl += [b.nl] * b.upad
        if b.vpad:
            pad = _completion(b.Vh.transpose(0, 1).contiguous(), b.vpad).contiguous()
            _scatter(eng, pad, b.rset, list(range(b.vpad)), list(range(vo, vo + b.vpad)), None, v, v.shape[1], 1)
            vo += b.vpad
        sv.append(np.zeros(b.vpad))
        qnr += [b.nr] * b.vpad
    su = np.concatenate(su)
    sv = np.concatenate(sv)
    if not full_matrices:
        order = np.argsort(su)[::-1].copy()
        o = torch.as_tensor(order, device=u.device)
        u, v = u[:, o], v[:, o]
        su = sv = su[order]
        qnl = [qnl[i] for i in order]
        qnr = [qnr[i] for i in order]
    return u, su, qnl, v, sv, qnr
