"""Hand-written backward of the effective-Hamiltonian matvec
(renormalizer/mps/hop_expr.py:57-103) behind a torch.autograd.Function.

For y = H_eff(L, W.., R) psi, a multilinear map, the gradient with respect to
each operand is the contraction of the upstream gradient gy with the complex
conjugates of the other operands (torch's convention for complex tensors:
grad_x = J^H grad_y):

* d psi: the same matvec with L'[c,b,a] = conj L[a,b,c], W'[b,e,d,f] =
  conj W[b,d,e,f] and R'[k,f,l] = conj R[l,f,k] applied to gy -- it runs on
  the engine's matvec kernels (fused split chain included);
* d L, d R, d W: fixed chains of pairwise contractions (``tensordot`` below),
  each one GEMM on the engine's FP64 DMMA kernel after a layout permute.

Real operands (MPO tensors, DMRG environments) receive the real part.  The
reference has no gradients; ``tests/test_autodiff.py`` checks these against
torch autograd through an FP64 einsum of the same contraction and against
central finite differences.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np
import torch

from ._native import Engine
from .backend import backend


def tensordot(a: torch.Tensor, b: torch.Tensor, axes, eng: Engine = None) -> torch.Tensor:
    """numpy.tensordot(a, b, axes) as one FP64 GEMM on the engine (conj views
    are folded into the GEMM)."""
    ia, ib = (list(axes[0]), list(axes[1]))
    fa = [i for i in range(a.dim()) if i not in ia]
    fb = [i for i in range(b.dim()) if i not in ib]
    ka = int(np.prod([a.shape[i] for i in ia])) if ia else 1
    A = a.permute(fa + ia).reshape(-1, ka)
    B = b.permute(ib + fb).reshape(ka, -1)
    eng = eng or Engine.get(a.device)
    C = eng.matmul(A, B)
    return C.reshape([a.shape[i] for i in fa] + [b.shape[i] for i in fb])


def _c(t: Optional[torch.Tensor]) -> Optional[torch.Tensor]:
    return None if t is None else (t.conj() if t.is_complex() else t)


def _dagger_operands(L, Ws, R):
    """operands of the adjoint matvec: L'[c,b,a] = conj L[a,b,c], W'[b,e,d,f] =
    conj W[b,d,e,f], R'[k,f,l] = conj R[l,f,k]"""
    fix = lambda t: t.resolve_conj().contiguous()
    return (fix(_c(L).permute(2, 1, 0)), [fix(_c(w).permute(0, 2, 1, 3)) for w in Ws],
            fix(_c(R).permute(2, 1, 0)))


def heff_backward(L, Ws: Sequence[torch.Tensor], R, psi, gy, need_psi=True, need_L=False, need_W=(False, False),
                  need_R=False, prec: str = None):
    """Gradients of Re<gy, y> style losses for y = H_eff psi (0, 1 or 2 sites).
    Returns (g_psi, g_L, [g_W1, g_W2], g_R) with None where not requested."""
    from .hop_expr import HeffOperator
    eng = Engine.get(psi.device)
    n = len(Ws)
    gpsi = gL = gR = None
    gW: List[Optional[torch.Tensor]] = [None] * n
    if need_psi:
        Ld, Wd, Rd = _dagger_operands(L, Ws, R)
        gpsi = HeffOperator(Ld, Rd, Wd, psi.shape, prec=prec).apply(gy.resolve_conj().contiguous())
    cL, cR, cP = _c(L), _c(R), _c(psi)
    cW = [_c(w) for w in Ws]
    td = lambda x, y, ax: tensordot(x, y, ax, eng)
    if need_L:
        if n == 0:
            T = td(cP, cR, ([1], [2]))                                  # c l b
            gL = td(gy, T, ([1], [1])).permute(0, 2, 1)                 # a c b -> a b c
        elif n == 1:
            T = td(cP, cR, ([2], [2]))                                  # c e l f
            T = td(T, cW[0], ([1, 3], [2, 3]))                          # c l b d
            gL = td(gy, T, ([1, 2], [3, 1])).permute(0, 2, 1)           # a c b -> a b c
        else:
            T = td(cP, cR, ([3], [2]))                                  # c e h l j
            T = td(T, cW[1], ([2, 4], [2, 3]))                          # c e l f g
            T = td(T, cW[0], ([1, 3], [2, 3]))                          # c l g b d
            gL = td(gy, T, ([1, 2, 3], [4, 2, 1])).permute(0, 2, 1)     # a c b -> a b c
    if need_R:
        if n == 0:
            T = td(cL, cP, ([2], [0]))                                  # a b k
            gR = td(gy, T, ([0], [0]))                                  # l b k
        elif n == 1:
            T = td(cL, cP, ([2], [0]))                                  # a b e k
            T = td(T, cW[0], ([1, 2], [0, 2]))                          # a k d f
            gR = td(gy, T, ([0, 1], [0, 2])).permute(0, 2, 1)           # l k f -> l f k
        else:
            T = td(cL, cP, ([2], [0]))                                  # a b e h k
            T = td(T, cW[0], ([1, 2], [0, 2]))                          # a h k d f
            T = td(T, cW[1], ([4, 1], [0, 2]))                          # a k d g j
            gR = td(gy, T, ([0, 1, 2], [0, 2, 3])).permute(0, 2, 1)     # l k j -> l j k
    if n >= 1 and need_W[0]:
        if n == 1:
            T = td(cL, cP, ([2], [0]))                                  # a b e k
            T = td(T, cR, ([3], [2]))                                   # a b e l f
            gW[0] = td(gy, T, ([0, 2], [0, 3])).permute(1, 0, 2, 3)     # d b e f -> b d e f
        else:
            T = td(cP, cR, ([3], [2]))                                  # c e h l j
            T = td(T, cW[1], ([2, 4], [2, 3]))                          # c e l f g
            T = td(T, cL, ([0], [2]))                                   # e l f g a b
            gW[0] = td(gy, T, ([0, 2, 3], [4, 3, 1])).permute(3, 0, 1, 2)   # d e f b -> b d e f
    if n == 2 and need_W[1]:
        T = td(cL, cP, ([2], [0]))                                      # a b e h k
        T = td(T, cW[0], ([1, 2], [0, 2]))                              # a h k d f
        T = td(T, cR, ([2], [2]))                                       # a h d f l j
        gW[1] = td(gy, T, ([0, 1, 3], [0, 2, 4])).permute(2, 0, 1, 3)  # g h f j -> f g h j
    fix = lambda g, like: None if g is None else (g.contiguous() if like.is_complex() else g.real.contiguous())
    return (fix(gpsi, psi), fix(gL, L), [fix(g, w) for g, w in zip(gW, Ws)], fix(gR, R))


class HeffFunction(torch.autograd.Function):
    """y = H_eff(L, W1[, W2], R) psi with the engine's matvec forward and the
    hand-written backward above (W2 is None for one active site, W1 and W2
    are None for the 0-site form)."""

    @staticmethod
    def forward(ctx, psi, L, W1, W2, R, prec):
        from .hop_expr import HeffOperator
        Ws = [w for w in (W1, W2) if w is not None]
        ctx.save_for_backward(psi, L, W1, W2, R)
        ctx.prec = prec
        return HeffOperator(L, R, Ws, psi.shape, prec=prec).apply(psi)

    @staticmethod
    def backward(ctx, gy):
        psi, L, W1, W2, R = ctx.saved_tensors
        Ws = [w for w in (W1, W2) if w is not None]
        need = ctx.needs_input_grad
        gpsi, gL, gW, gR = heff_backward(L, Ws, R, psi, gy, need_psi=need[0], need_L=need[1],
                                         need_W=(need[2], need[3]), need_R=need[4], prec=ctx.prec)
        gW = gW + [None] * (2 - len(gW))
        return gpsi, gL, gW[0], gW[1], gR, None


def heff(psi, L, Ws: Sequence[torch.Tensor], R, prec: str = None) -> torch.Tensor:
    """Differentiable H_eff psi (0, 1 or 2 active sites)."""
    Ws = list(Ws) + [None] * (2 - len(Ws))
    return HeffFunction.apply(psi, L, Ws[0], Ws[1], R, prec or backend.prec)
