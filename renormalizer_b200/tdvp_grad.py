"""Gradients of observables with respect to Hamiltonian couplings through a
one-site TDVP-PS trajectory (renormalizer/mps/mps.py:1267-1404), by reverse
mode through the sweep.

The step is the engine's 1-site projector splitting: on each site the local
exponential exp(-i H_eff dt/2), a QR (RQ on the way back) that moves the
centre, the environment update, and the backward bond exponential
exp(+i H_0 dt/2); two half-sweeps, then the centre is normalised (evolve's
``mps_only`` normalisation).  Every contraction runs on the engine:

* matvecs through ``autodiff.heff`` (hand-written H_eff backward);
* environment updates and the small bond products through ``Contract``, a
  tensordot on the engine GEMM whose backward is two more engine GEMMs.

Local exponentials use a fixed number of Lanczos vectors (the reference's
adaptive stopping rule is a branch, not a differentiable function) with the
small projected exponential taken by torch.linalg.matrix_exp.  The QR runs
on whole site matrices rather than per QN block: it spans the same bond
subspace, so the state, and every observable, is the same.  Steps are
checkpointed: only the site tensors at step boundaries are kept and each
step is recomputed during the backward pass.

The MPO enters as W(g) = W(g0) + sum_j (g_j - g0_j) dW/dg_j with dW/dg_j from
the MPO builder at g0 +- e_j (exact: the Holstein MPO is at most quadratic
in a coupling), so W(g0) is the MPO itself and the gradient at g0 is exact.

``contract="einsum"`` runs the same trajectory on torch.tensordot in FP64
(torch's own autograd everywhere): the reference gradient the engine's
is checked against, together with central finite differences.
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from .autodiff import heff, tensordot

class Contract(torch.autograd.Function):
    """c = tensordot(a, b, (ia, ib)) on the engine GEMM; backward: grad_a =
    g . conj(b), grad_b = conj(a) . g, each one engine GEMM."""

    @staticmethod
    def forward(ctx, a, b, ia, ib):
        ctx.save_for_backward(a, b)
        ctx.ia, ctx.ib = list(ia), list(ib)
        return tensordot(a, b, (list(ia), list(ib)))

    @staticmethod
    def backward(ctx, g):
        a, b = ctx.saved_tensors
        ia, ib = ctx.ia, ctx.ib
        fa = [i for i in range(a.dim()) if i not in ia]
        fb = [i for i in range(b.dim()) if i not in ib]
        ga = gb = None
        if ctx.needs_input_grad[0]:
            t = tensordot(g, b.conj(), (list(range(len(fa), len(fa) + len(fb))), fb))
            axes = fa + [ia[ib.index(x)] for x in sorted(ib)]
            ga = t.permute([axes.index(i) for i in range(a.dim())])
            ga = ga if a.is_complex() else ga.real
        if ctx.needs_input_grad[1]:
            t = tensordot(a.conj(), g, (fa, list(range(len(fa)))))
            axes = [ib[ia.index(x)] for x in sorted(ia)] + fb
            gb = t.permute([axes.index(i) for i in range(b.dim())])
            gb = gb if b.is_complex() else gb.real
        return ga, gb, None, None


class _Ops:
    """the contraction backend: the engine (default) or plain torch (the
    autograd-through-einsum reference)"""

    def __init__(self, kind: str):
        assert kind in ("engine", "einsum")
        self.kind = kind

    def td(self, a, b, ia, ib):
        if self.kind == "engine":
            return Contract.apply(a, b, tuple(ia), tuple(ib))
        dt = torch.complex128 if (a.is_complex() or b.is_complex()) else torch.float64
        return torch.tensordot(a.to(dt), b.to(dt), dims=(list(ia), list(ib)))

    def hop(self, psi, L, Ws, R):
        if self.kind == "engine":
            return heff(psi, L, Ws, R, prec="fp64")
        # the hop_expr contraction in an explicit pairwise order (torch.einsum
        # without a path optimiser would form an (M d)^2 M^2 intermediate)
        c = lambda t: t.to(torch.complex128)
        if not Ws:                                                      # abc, lbk, ck -> al
            t = torch.tensordot(c(L), c(psi), dims=([2], [0]))          # a b k
            return torch.tensordot(t, c(R), dims=([1, 2], [1, 2]))      # a l
        t = torch.tensordot(c(L), c(psi), dims=([2], [0]))              # a b e k
        t = torch.tensordot(t, c(Ws[0]), dims=([1, 2], [0, 2]))         # a k d f
        return torch.tensordot(t, c(R), dims=([3, 1], [1, 2]))          # a d l

    def env_L(self, E, ms, W):
        """lib.py:200-205: L'[f,g,h] = sum E[a,b,c] conj(ms[a,d,f]) W[b,d,e,g] ms[c,e,h]"""
        t = self.td(E, ms.conj(), [0], [0])            # b c d f
        t = self.td(t, W, [0, 2], [0, 1])              # c f e g
        return self.td(t, ms, [0, 2], [0, 1])          # f g h

    def env_R(self, E, ms, W):
        """lib.py:232-237: R'[f,g,h] = sum conj(ms[f,d,a]) E[a,b,c] W[g,d,e,b] ms[h,e,c]"""
        t = self.td(ms.conj(), E, [2], [0])            # f d b c
        t = self.td(t, W, [1, 2], [1, 3])              # f c g e
        return self.td(t, ms, [1, 3], [2, 1])          # f g h


class _BatchedOps(_Ops):
    """Plain torch FP64 contractions over a leading batch axis (many coupling
    sets of one trajectory at once: the finite-difference checks).  Tensor
    indices in ``td`` count the per-instance axes; a batch of one
    broadcasts."""

    batched = True

    def __init__(self):
        super().__init__("einsum")

    def td(self, a, b, ia, ib):
        na, nb = a.dim() - 1, b.dim() - 1
        la = [chr(97 + i) for i in range(na)]
        lb = [chr(97 + na + i) for i in range(nb)]
        for x, y in zip(ia, ib):
            lb[y] = la[x]
        out = [c for i, c in enumerate(la) if i not in ia] + [c for i, c in enumerate(lb) if i not in ib]
        dt = torch.complex128 if (a.is_complex() or b.is_complex()) else torch.float64
        return torch.einsum(f"...{''.join(la)},...{''.join(lb)}->...{''.join(out)}", a.to(dt), b.to(dt))

    def hop(self, psi, L, Ws, R):
        if not Ws:
            t = self.td(L, psi, [2], [0])                               # a b k
            return self.td(t, R, [1, 2], [1, 2])                        # a l
        t = self.td(L, psi, [2], [0])                                   # a b e k
        t = self.td(t, Ws[0], [1, 2], [0, 2])                           # a k d f
        return self.td(t, R, [3, 1], [1, 2])                            # a d l


def _bdot(x, y, nb):
    """<x, y> over all but the first nb axes"""
    return (x.conj() * y).reshape(*x.shape[:nb], -1).sum(-1) if nb else torch.vdot(x.reshape(-1), y.reshape(-1))


def expm_krylov_fixed(apply: Callable, dt: complex, v: torch.Tensor, k: int, nb: int = 0) -> torch.Tensor:
    """exp(dt A) v from k Lanczos vectors (three-term recurrence as in
    krylov.py:27-84, fixed length; stops early on the reference's breakdown
    test beta < 100 n eps, krylov.py:72-74, which also bounds the local
    Krylov space by the local dimension).  With ``nb`` = 1, v carries a
    leading batch axis and every instance runs the same recurrence; an
    instance that breaks down while others go on gets beta_j = 0 and zero
    vectors from there on, which decouples the rest of its tridiagonal matrix
    (exp of a block-diagonal T), so its result is that of its own run."""
    vol = v[0].numel() if nb else v.numel()
    red = (lambda x: torch.linalg.vector_norm(x.reshape(x.shape[0], -1), dim=1)) if nb else torch.linalg.vector_norm
    bshape = (-1,) + (1,) * (v.dim() - 1) if nb else ()
    nrm = red(v)
    tiny = 100 * vol * np.finfo(np.float64).eps
    Q = [v / nrm.reshape(bshape)]
    alphas, betas = [], []
    for j in range(k):
        w = apply(Q[j])
        a = torch.real(_bdot(Q[j], w, nb))
        w = w - a.reshape(bshape) * Q[j]
        if j > 0:
            w = w - betas[-1].reshape(bshape) * Q[j - 1]
        alphas.append(a)
        if j == k - 1:
            break
        b = red(w)
        small = (b.detach() < tiny)
        if bool(small.all()):
            break
        if nb and bool(small.any()):
            b = torch.where(small, torch.zeros_like(b), b)
            safe = torch.where(small, torch.ones_like(b), b)
            betas.append(b)
            Q.append(torch.where(small.reshape(bshape), torch.zeros_like(w), w / safe.reshape(bshape)))
            continue
        betas.append(b)
        Q.append(w / b.reshape(bshape))
    m = len(alphas)
    T = torch.diag_embed(torch.stack(alphas, dim=-1)).to(torch.complex128)
    if m > 1:
        off = torch.stack(betas[: m - 1], dim=-1).to(torch.complex128)
        T = T + torch.diag_embed(off, 1) + torch.diag_embed(off, -1)
    e = torch.linalg.matrix_exp(dt * T)[..., :, 0]
    coef = lambda j: e[..., j].reshape(bshape)
    out = coef(0) * Q[0]
    for j in range(1, m):
        out = out + coef(j) * Q[j]
    return nrm.reshape(bshape) * out


def tdvp_ps_step(sites: List[torch.Tensor], Ws: Sequence[torch.Tensor], dt: float, k: int, ops: _Ops):
    """One TDVP-PS step from a right-canonical MPS (centre on site 0): a
    right half-sweep then a left half-sweep, centre normalised; returns the
    new right-canonical sites (mps.py:1267-1404).  With batched ops
    (_BatchedOps) every tensor carries a leading batch axis."""
    n = len(sites)
    sites = list(sites)
    nb = 1 if getattr(ops, "batched", False) else 0
    lead = tuple(sites[0].shape[:nb])
    one = torch.ones(lead + (1, 1, 1), dtype=torch.float64, device=sites[0].device)
    R = [None] * (n + 1)
    R[n] = one
    for i in range(n - 1, 0, -1):
        R[i] = ops.env_R(R[i + 1], sites[i], Ws[i])
    Ls = [one] + [None] * n
    for i in range(n):
        L = Ls[i]
        sites[i] = expm_krylov_fixed(lambda x: ops.hop(x, L, [Ws[i]], R[i + 1]), -0.5j * dt, sites[i], k, nb)
        if i == n - 1:
            break
        ml, d, mr = sites[i].shape[nb:]
        q, r = torch.linalg.qr(sites[i].reshape(lead + (ml * d, mr)))
        sites[i] = q.reshape(lead + (ml, d, q.shape[-1]))
        Ls[i + 1] = ops.env_L(L, sites[i], Ws[i])
        c = expm_krylov_fixed(lambda x: ops.hop(x, Ls[i + 1], [], R[i + 1]), 0.5j * dt, r, k, nb)
        sites[i + 1] = ops.td(c, sites[i + 1], [1], [0])
    Rc = one
    for i in range(n - 1, -1, -1):
        sites[i] = expm_krylov_fixed(lambda x: ops.hop(x, Ls[i], [Ws[i]], Rc), -0.5j * dt, sites[i], k, nb)
        if i == 0:
            break
        ml, d, mr = sites[i].shape[nb:]
        q1, r1 = torch.linalg.qr(sites[i].reshape(lead + (ml, d * mr)).mH)     # site = r1^H q1^H
        sites[i] = q1.mH.reshape(lead + (q1.shape[-1], d, mr))
        Rn = ops.env_R(Rc, sites[i], Ws[i])
        c = expm_krylov_fixed(lambda x: ops.hop(x, Ls[i], [], Rn), 0.5j * dt, r1.mH, k, nb)
        sites[i - 1] = ops.td(sites[i - 1], c, [2], [0])
        Rc = Rn
    if nb:
        s0 = sites[0]
        sites[0] = s0 / torch.linalg.vector_norm(s0.reshape(s0.shape[0], -1), dim=1).reshape(-1, 1, 1, 1)
    else:
        sites[0] = sites[0] / torch.linalg.vector_norm(sites[0])
    return sites


def site_expectation(sites: Sequence[torch.Tensor], site: int, op: torch.Tensor, ops: _Ops):
    """<psi| O_site |psi> / <psi|psi> by a left-environment sweep (one value
    per instance with batched ops)."""
    dev = sites[0].device
    nb = 1 if getattr(ops, "batched", False) else 0
    one = (1,) * nb
    E = torch.ones(one + (1, 1, 1), dtype=torch.float64, device=dev)
    N = E
    for i, ms in enumerate(sites):
        d = ms.shape[nb + 1]
        eye = torch.eye(d, dtype=torch.float64, device=dev).reshape(one + (1, d, d, 1))
        W = op.reshape(one + (1, d, d, 1)) if i == site else eye
        E = ops.env_L(E, ms, W)
        N = ops.env_L(N, ms, eye)
    if nb:
        return torch.real(E.reshape(E.shape[0], -1)[:, 0]) / torch.real(N.reshape(N.shape[0], -1)[:, 0])
    return torch.real(E.reshape(-1)[0]) / torch.real(N.reshape(-1)[0])


def mpo_derivatives(build: Callable[[np.ndarray], Sequence[np.ndarray]], g0: np.ndarray):
    """W(g0) and dW/dg_j per site from the MPO builder at g0 +- e_j (exact for
    MPOs at most quadratic in each coupling)."""
    W0 = [np.asarray(w, dtype=float) for w in build(np.asarray(g0, dtype=float))]
    dW = []
    for j in range(len(g0)):
        e = np.zeros(len(g0))
        e[j] = 1.0
        wp = build(g0 + e)
        wm = build(g0 - e)
        for a, b, c in zip(wp, wm, W0):
            if a.shape != c.shape or b.shape != c.shape:
                raise AssertionError("the MPO structure changes with the coupling")
        dW.append([(np.asarray(a) - np.asarray(b)) / 2.0 for a, b in zip(wp, wm)])
    return W0, dW


def trajectory_value(Ws: Sequence[np.ndarray], sites0: Sequence[torch.Tensor], dt: float, nsteps: int,
                     obs_site: int, op: np.ndarray, krylov: int = 8, contract: str = "engine") -> float:
    """<O_obs_site>(t = nsteps dt) for given MPO tensors (no gradient)."""
    ops = _Ops(contract)
    dev = sites0[0].device
    Wd = [torch.as_tensor(np.asarray(w, dtype=float), device=dev) for w in Ws]
    with torch.no_grad():
        sites = [s.to(torch.complex128) for s in sites0]
        for _ in range(nsteps):
            sites = tdvp_ps_step(sites, Wd, dt, krylov, ops)
        return float(site_expectation(sites, obs_site, torch.as_tensor(op, dtype=torch.float64, device=dev), ops))


def trajectory_values(Ws_list: Sequence[Sequence[np.ndarray]], sites0: Sequence[torch.Tensor], dt: float,
                      nsteps: int, obs_site: int, op: np.ndarray, krylov: int = 8) -> np.ndarray:
    """trajectory_value(contract="einsum") for many MPOs of one structure at
    once (batched FP64 torch contractions; used for finite differences)."""
    ops = _BatchedOps()
    dev = sites0[0].device
    B = len(Ws_list)
    Wd = [torch.stack([torch.as_tensor(np.asarray(Ws[i], dtype=float)) for Ws in Ws_list]).to(dev)
          for i in range(len(Ws_list[0]))]
    with torch.no_grad():
        sites = [s.to(torch.complex128).unsqueeze(0).expand((B,) + tuple(s.shape)).contiguous() for s in sites0]
        for _ in range(nsteps):
            sites = tdvp_ps_step(sites, Wd, dt, krylov, ops)
        opd = torch.as_tensor(op, dtype=torch.float64, device=dev)
        return site_expectation(sites, obs_site, opd, ops).cpu().numpy()


def coupling_gradient(build: Callable[[np.ndarray], Sequence[np.ndarray]], g0, sites0: Sequence[torch.Tensor],
                      dt: float, nsteps: int, obs_site: int, op: np.ndarray, krylov: int = 8,
                      checkpoint_every: int = 1, contract: str = "engine"):
    """d <O_obs_site>(t = nsteps dt) / d g at g0 through the TDVP-PS trajectory
    from the right-canonical ``sites0``.  Steps run in checkpointed segments
    of ``checkpoint_every`` steps (0: no checkpointing): only the segment
    boundaries are stored and each segment is recomputed in the backward
    pass.  Returns (value, gradient)."""
    ops = _Ops(contract)
    dev = sites0[0].device
    g0 = np.asarray(g0, dtype=float)
    W0, dW = mpo_derivatives(build, g0)
    g = torch.tensor(g0, dtype=torch.float64, device=dev, requires_grad=True)
    dg = g - torch.tensor(g0, dtype=torch.float64, device=dev)
    Ws = []
    for i in range(len(W0)):
        w = torch.as_tensor(W0[i], device=dev)
        for j in range(len(g0)):
            dj = dW[j][i]
            if np.any(dj):
                w = w + dg[j] * torch.as_tensor(dj, device=dev)
        Ws.append(w)
    sites = [s.to(torch.complex128) for s in sites0]
    ns = len(sites)

    def segment(nstep, *a):
        cur = list(a[:ns])
        for _ in range(nstep):
            cur = tdvp_ps_step(cur, a[ns:], dt, krylov, ops)
        return tuple(cur)

    done = 0
    while done < nsteps:
        seg = nsteps - done if checkpoint_every <= 0 else min(checkpoint_every, nsteps - done)
        if checkpoint_every > 0:
            sites = list(checkpoint(segment, seg, *sites, *Ws, use_reentrant=False))
        else:
            sites = list(segment(seg, *sites, *Ws))
        done += seg
    val = site_expectation(sites, obs_site, torch.as_tensor(op, dtype=torch.float64, device=dev), ops)
    grad, = torch.autograd.grad(val, g)
    return float(val.detach()), grad.detach().cpu().numpy()
