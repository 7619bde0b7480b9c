"""Environments of the sweep, drop-in for renormalizer/mps/lib.py:12-250.

``Environ`` keeps every L/R environment tensor resident in HBM (the
reference's ``_virtual_disk`` host dict, lib.py:20,114-118, becomes a dict of
device tensors: no host round trip per read/write) and
``contract_one_site`` runs reno_env_update.
"""
from __future__ import annotations

import numpy as np
import torch

from ._native import Engine, EnvDesc, PREC, dtype_code
from .backend import backend
from .hop_expr import as_device


def contract_one_site(environ, ms, mo, domain, ms_conj=None, prec: str = None) -> torch.Tensor:
    """lib.py:169-250: one environment update (3-leg MPS sites)."""
    assert domain in ["L", "R"]
    E = as_device(environ)
    ket = as_device(ms)
    W = as_device(mo)
    bra = as_device(ms_conj) if ms_conj is not None else None
    assert ket.dim() == 3, "ancilla (MPDM) sites are not part of the sweep engine"
    d = EnvDesc()
    d.side = 0 if domain == "L" else 1
    d.d = ket.shape[1]
    if domain == "L":
        # E (bra_in, w_in, ket_in), ket (ket_in, d, ket_out), W (w_in, d, d, w_out)
        assert E.shape[1] == W.shape[0] and E.shape[2] == ket.shape[0]
        d.w_in, d.w_out = W.shape[0], W.shape[3]
        d.mk_in, d.mk_out = ket.shape[0], ket.shape[2]
        if bra is not None:
            assert E.shape[0] == bra.shape[0]
            d.mb_in, d.mb_out = bra.shape[0], bra.shape[2]
        else:
            assert E.shape[0] == ket.shape[0]
            d.mb_in, d.mb_out = d.mk_in, d.mk_out
    else:
        assert E.shape[1] == W.shape[3] and E.shape[2] == ket.shape[2]
        d.w_in, d.w_out = W.shape[3], W.shape[0]
        d.mk_in, d.mk_out = ket.shape[2], ket.shape[0]
        if bra is not None:
            assert E.shape[0] == bra.shape[2]
            d.mb_in, d.mb_out = bra.shape[2], bra.shape[0]
        else:
            assert E.shape[0] == ket.shape[2]
            d.mb_in, d.mb_out = d.mk_in, d.mk_out
    assert W.shape[1] == W.shape[2] == d.d
    d.env_dtype, d.ket_dtype, d.mpo_dtype = dtype_code(E), dtype_code(ket), dtype_code(W)
    d.bra_dtype = dtype_code(bra) if bra is not None else d.ket_dtype
    d.prec = PREC[prec or backend.prec]
    cplx = any(t is not None and t.is_complex() for t in (E, ket, W, bra))
    out = torch.empty((d.mb_out, d.w_out, d.mk_out), dtype=torch.complex128 if cplx else torch.float64,
                      device=ket.device)
    eng = Engine.get(ket.device)
    eng.env_update(d, E, W, ket, bra, out)
    return out


class Environ:
    """lib.py:12-118 with device-resident storage.

    idx convention: L(idx-1) - mpo(idx) - R(idx+1); out-of-range reads of
    GetLR return the ones((1,1,1)) sentinel (lib.py:80-81).

    ``prec`` (not in the reference) fixes the arithmetic of every update of
    this environment; None follows the backend's precision at each call.
    The ground-state search keeps its environments in FP64: their rounding
    accumulates along the chain into every later effective Hamiltonian."""

    def __init__(self, mps, mpo, domain=None, mps_conj=None, prec: str = None):
        self.prec = prec
        self._virtual_disk = {}
        self.sentinel = torch.ones((1, 1, 1), dtype=torch.float64, device=backend.device)
        self._construct(mps, mpo, domain, mps_conj)

    def _construct(self, mps, mpo, domain=None, mps_conj=None):
        assert domain in ["L", "R", None]
        if domain is None:
            self._construct(mps, mpo, "L", mps_conj)
            self._construct(mps, mpo, "R", mps_conj)
            return
        if domain == "L":
            start, end, inc = 0, len(mps) - 1, 1
        else:
            start, end, inc = len(mps) - 1, 0, -1
        self.write("L", -1, self.sentinel)
        self.write("R", len(mps), self.sentinel)
        tensor = self.sentinel
        for idx in range(start, end, inc):
            conj = mps_conj[idx] if mps_conj is not None else None
            tensor = contract_one_site(tensor, mps[idx], mpo[idx], domain, ms_conj=conj, prec=self.prec)
            self.write(domain, idx, tensor)

    def GetLR(self, domain, siteidx, mps, mpo, itensor=None, method="Scratch", mps_conj=None):
        assert domain in ["L", "R"]
        assert method in ["Enviro", "System", "Scratch"]
        if siteidx not in range(len(mps)):
            return self.sentinel
        if method == "Scratch":
            itensor = self.sentinel
            sitelist = range(siteidx + 1) if domain == "L" else range(len(mps) - 1, siteidx - 1, -1)
            for imps in sitelist:
                conj = mps_conj[imps] if mps_conj is not None else None
                itensor = contract_one_site(itensor, mps[imps], mpo[imps], domain, ms_conj=conj, prec=self.prec)
        elif method == "Enviro":
            itensor = self.read(domain, siteidx)
        else:
            if itensor is None:
                offset = -1 if domain == "L" else 1
                itensor = self.read(domain, siteidx + offset)
            conj = mps_conj[siteidx] if mps_conj is not None else None
            itensor = contract_one_site(itensor, mps[siteidx], mpo[siteidx], domain, ms_conj=conj, prec=self.prec)
            self.write(domain, siteidx, itensor)
        return itensor

    def write(self, domain, siteidx, tensor):
        self._virtual_disk[(domain, siteidx)] = tensor

    def read(self, domain: str, siteidx: int):
        return self._virtual_disk[(domain, siteidx)]
