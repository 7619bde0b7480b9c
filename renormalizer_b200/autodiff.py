"""Hand-written backward of the effective-Hamiltonian matvec
(renormalizer/mps/hop_expr.py:57-103) behind a torch.autograd.Function.

For y = H_eff(L, W.., R) psi, a multilinear map, the gradient with respect to
each operand is the contraction of the upstream gradient gy with the complex
conjugates of the other operands (torch's convention for complex tensors:
grad_x = J^H grad_y).  All of it runs in libreno_b200's reno_heff_backward:

* d psi: the same matvec with L'[c,b,a] = conj L[a,b,c], W'[b,e,d,f] =
  conj W[b,d,e,f] and R'[k,f,l] = conj R[l,f,k] applied to gy, on the
  engine's matvec kernels (fused split chain included);
* d L, d R, d W: fixed chains of pairwise contractions, each a permute-copy
  kernel per operand and one FP64 DMMA GEMM.

Real operands (MPO tensors, DMRG environments) receive the real part.
``tensordot`` below is the same contraction primitive for host-side use (the
TDVP gradient's environment updates).  The reference has no gradients;
``tests/test_autodiff.py`` checks these against
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


def heff_backward(L, Ws: Sequence[torch.Tensor], R, psi, gy, need_psi=True, need_L=False, need_W=(False, False),
                  need_R=False, prec: str = None):
    """Gradients for y = H_eff psi (0, 1 or 2 sites) given gy, through
    reno_heff_backward.  Returns (g_psi, g_L, [g_W1, g_W2], g_R) with None
    where not requested; real operands get the real part."""
    import ctypes
    from ._native import dtype_code
    from .hop_expr import HeffOperator
    op = HeffOperator(L, R, list(Ws), psi.shape, prec=prec)
    p = psi.reshape(op.cshape)
    if p.dtype not in (torch.float64, torch.complex128):
        p = p.to(torch.complex128 if p.is_complex() else torch.float64)
    p = p.resolve_conj().contiguous()
    desc = type(op.desc)()
    ctypes.pointer(desc)[0] = op.desc
    desc.psi_dtype = dtype_code(p)
    ydt = op.out_dtype(p)
    g = gy.reshape(op.cshape).to(ydt).resolve_conj().contiguous()
    new = lambda like, cond: torch.empty(like.shape, dtype=ydt, device=p.device) if cond else None
    n = len(op.W)
    gpsi, gL, gR = new(p, need_psi), new(op.L, need_L), new(op.R, need_R)
    gW = [new(op.W[i], need_W[i]) if i < n else None for i in range(2)]
    op.engine.sync_stream()
    op.engine.heff_backward(desc, op.L, op.W[0] if n >= 1 else None, op.W[1] if n == 2 else None, op.R, p, g,
                            gpsi, gL, gW[0], gW[1], gR)
    fix = lambda t, like: None if t is None else (t if like.is_complex() else t.real.contiguous())
    return (fix(gpsi, psi), fix(gL, L), [fix(gW[i], Ws[i]) for i in range(len(Ws))], fix(gR, R))


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
