"""Effective-Hamiltonian matvec on the GPU, the drop-in for
renormalizer/mps/hop_expr.py:7-117.

``hop_expr(ltensor, rtensor, cmo, cshape)`` returns a callable ``expr(psi)``
exactly like the reference: L, R and the MPO site tensors are captured as
constants and ``psi`` (shape ``cshape``) is contracted with them.  The
contraction runs in libreno_b200 (reno_heff_apply) at the backend's
arithmetic (FP64 DMMA or BF16x3 / TF32x3 split products).
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import numpy as np
import torch

from ._native import Engine, HeffDesc, PREC, dtype_code
from .backend import backend


def as_device(t, device=None, dtype=None) -> torch.Tensor:
    """numpy / torch -> contiguous float64 or complex128 tensor on the GPU."""
    if device is None:
        device = backend.device
    if isinstance(t, torch.Tensor):
        out = t.to(device=device)
    else:
        out = torch.from_numpy(np.ascontiguousarray(np.asarray(t))).to(device=device)
    if dtype is not None:
        out = out.to(dtype)
    elif out.dtype not in (torch.float64, torch.complex128):
        out = out.to(torch.complex128 if out.is_complex() else torch.float64)
    return out.contiguous()


class HeffOperator:
    """The captured H_eff of one local problem (0, 1 or 2 active sites)."""

    def __init__(self, ltensor, rtensor, cmo: Sequence, cshape, prec: str = None):
        self.L = as_device(ltensor)
        self.R = as_device(rtensor)
        self.W = [as_device(w) for w in cmo]
        self.nsite = len(self.W)
        self.cshape = tuple(int(s) for s in cshape)
        assert self.nsite + 2 == len(self.cshape), "ancilla (MPDM) sites are not part of the sweep engine"
        self.prec = prec or backend.prec
        self.engine = Engine.get(self.L.device)
        ml, wl, ml2 = self.L.shape
        mr, wr, mr2 = self.R.shape
        assert ml == ml2 and mr == mr2
        assert self.cshape[0] == ml and self.cshape[-1] == mr
        d = HeffDesc()
        d.nsite, d.ml, d.mr, d.wl, d.wr = self.nsite, ml, mr, wl, wr
        d.wm, d.d1, d.d2 = 1, 1, 1
        if self.nsite == 0:
            assert wl == wr
        elif self.nsite == 1:
            assert self.W[0].shape == (wl, self.cshape[1], self.cshape[1], wr)
            d.d1 = self.cshape[1]
        else:
            d.d1, d.d2 = self.cshape[1], self.cshape[2]
            d.wm = self.W[0].shape[3]
            assert self.W[0].shape == (wl, d.d1, d.d1, d.wm)
            assert self.W[1].shape == (d.wm, d.d2, d.d2, wr)
        if self.L.dtype != self.R.dtype:
            # e.g. the real ones((1,1,1)) boundary sentinel next to a complex environment
            self.L = self.L.to(torch.complex128)
            self.R = self.R.to(torch.complex128)
        d.env_dtype = dtype_code(self.L)
        d.mpo_dtype = dtype_code(self.W[0]) if self.W else 0
        for w in self.W:
            if dtype_code(w) != d.mpo_dtype:
                self.W = [x.to(torch.complex128) for x in self.W]
                d.mpo_dtype = 1
        d.prec = PREC[self.prec]
        self.desc = d
        self.complex_env = self.L.is_complex() or any(w.is_complex() for w in self.W)

    def out_dtype(self, psi: torch.Tensor):
        return torch.complex128 if (psi.is_complex() or self.complex_env) else torch.float64

    def apply(self, psi: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
        psi = psi.reshape(self.cshape)
        if not psi.is_contiguous():
            psi = psi.contiguous()
        if psi.dtype not in (torch.float64, torch.complex128):
            psi = psi.to(torch.complex128 if psi.is_complex() else torch.float64)
        self.desc.psi_dtype = dtype_code(psi)
        if out is None:
            out = torch.empty(self.cshape, dtype=self.out_dtype(psi), device=psi.device)
        self.engine.sync_stream()
        W1 = self.W[0] if self.nsite >= 1 else None
        W2 = self.W[1] if self.nsite == 2 else None
        self.engine.heff_apply(self.desc, self.L, W1, W2, self.R, psi, out)
        return out

    def diag(self) -> torch.Tensor:
        """Real diagonal of H_eff (gs.py:419-445)."""
        assert self.nsite >= 1
        out = torch.empty(self.cshape, dtype=torch.float64, device=self.L.device)
        W2 = self.W[1] if self.nsite == 2 else None
        self.engine.heff_diag(self.desc, self.L, self.W[0], W2, self.R, out)
        return out

    def __call__(self, psi, *args, **kwargs):
        if isinstance(psi, np.ndarray):
            psi = as_device(psi, self.L.device)
        return self.apply(psi)


MAX_GROUP = 128  # problems per grouped launch (reno_heff_apply_grouped)


def apply_grouped(ops: Sequence["HeffOperator"], psis: Sequence[torch.Tensor]) -> List[torch.Tensor]:
    """[op.apply(psi) for op, psi in zip(ops, psis)] for independent local
    problems.  FP64 operators with the same number of sites and dtypes go
    through reno_heff_apply_grouped, up to 128 per launch; split-precision
    operators (whose fused chains are not grouped) are applied one by one.
    Each result equals that operator's own apply."""
    ys: List[torch.Tensor] = [None] * len(ops)
    batch = {}
    for i, (op, psi) in enumerate(zip(ops, psis)):
        psi = psi.reshape(op.cshape)
        if not psi.is_contiguous():
            psi = psi.contiguous()
        if psi.dtype not in (torch.float64, torch.complex128):
            psi = psi.to(torch.complex128 if psi.is_complex() else torch.float64)
        if op.prec != "fp64":
            ys[i] = op.apply(psi)
            continue
        key = (op.nsite, dtype_code(psi), op.desc.env_dtype, op.desc.mpo_dtype, op.L.device)
        batch.setdefault(key, []).append((i, psi))
    for items in batch.values():
        for c0 in range(0, len(items), MAX_GROUP):
            chunk = items[c0:c0 + MAX_GROUP]
            descs, outs = [], []
            for i, psi in chunk:
                op = ops[i]
                d = HeffDesc()
                ctypes.pointer(d)[0] = op.desc
                d.psi_dtype = dtype_code(psi)
                descs.append(d)
                outs.append(torch.empty(op.cshape, dtype=op.out_dtype(psi), device=psi.device))
            sel = [ops[i] for i, _ in chunk]
            eng = sel[0].engine
            eng.sync_stream()
            eng.heff_apply_grouped(descs, [o.L for o in sel], [o.W[0] if o.nsite >= 1 else None for o in sel],
                                   [o.W[1] if o.nsite == 2 else None for o in sel], [o.R for o in sel],
                                   [psi for _, psi in chunk], outs)
            for (i, _), y in zip(chunk, outs):
                ys[i] = y
    return ys


def hop_expr(ltensor, rtensor, cmo: List, cshape, twolayer: bool = False):
    """Drop-in for renormalizer.mps.hop_expr.hop_expr (hop_expr.py:7)."""
    if twolayer:
        raise NotImplementedError("the (H - omega)^2 two-layer matvec is outside the sweep engine")
    return HeffOperator(ltensor, rtensor, cmo, cshape)
