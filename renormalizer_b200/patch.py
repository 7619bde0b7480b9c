"""Install the engine at the reference package's own patch points.

The reference imports its sweep kernels by name into the sweep modules
(renormalizer/mps/mps.py:13,18-24,33 and gs.py:18,23,26), so a drop-in
replaces them there.  ``install()`` puts the engine's ``hop_expr``,
``expm_krylov`` and ``Environ`` into ``renormalizer.mps.mps`` (the TDVP
sweeps, mps.py:1267-1517) and ``hop_expr`` into ``renormalizer.mps.gs``
(DMRG); the reference's own ``Mps.evolve`` / ``optimize_mps`` then run with
the matvec, the Lanczos exponential and the environment updates on the
device.  The adapters below only translate at the boundary: the reference's
``Matrix`` site tensors are read through ``.array``, numpy inputs go to the
device, and ``expm_krylov`` returns numpy when it was given numpy (the
reference's QN-blocked SVD/QR then runs on the host as before).
``uninstall()`` restores the originals.
"""
from __future__ import annotations

import importlib

import numpy as np

from .hop_expr import as_device, hop_expr as _engine_hop_expr
from .krylov import expm_krylov as _engine_expm_krylov
from .lib import Environ as _EngineEnviron

_saved = {}      # (module, name) -> the reference's original
_orig_hop = []   # the reference's hop_expr, for the forms the engine leaves to it


def _arr(x):
    return x.array if hasattr(x, "array") else x


class _Sites:
    """The reference's MPS / MPO as a sequence of plain arrays."""

    def __init__(self, mp):
        self._mp = mp

    def __len__(self):
        return len(self._mp)

    def __getitem__(self, i):
        return _arr(self._mp[i])


def _sites(mp):
    return None if mp is None else _Sites(mp)


def hop_expr(ltensor, rtensor, cmo, cshape, twolayer=False):
    """hop_expr.py:7: the engine's matvec for single-layer, non-ancilla sites;
    the two-layer and MPDM forms stay with the reference."""
    if twolayer or len(cshape) != len(cmo) + 2:
        return _orig_hop[0](ltensor, rtensor, cmo, cshape, twolayer)
    return _engine_hop_expr(ltensor, rtensor, [_arr(w) for w in cmo], cshape)


def expm_krylov(Afunc, dt, vstart, block_size=50):
    """krylov.py:27: the engine's Lanczos exponential; a host array (numpy, or
    the reference's Matrix) in, numpy out."""
    import torch
    res, n = _engine_expm_krylov(Afunc, dt, as_device(_arr(vstart)), block_size)
    if isinstance(vstart, torch.Tensor):
        return res, n
    return res.cpu().numpy(), n


class Environ(_EngineEnviron):
    """lib.py:12-118 on the device, fed with the reference's MPS objects."""

    def __init__(self, mps, mpo, domain=None, mps_conj=None):
        super().__init__(_sites(mps), _sites(mpo), domain, _sites(mps_conj))

    def GetLR(self, domain, siteidx, mps, mpo, itensor=None, method="Scratch", mps_conj=None):
        return super().GetLR(domain, siteidx, _sites(mps), _sites(mpo), itensor, method, _sites(mps_conj))


_TARGETS = {
    "renormalizer.mps.mps": {"hop_expr": hop_expr, "expm_krylov": expm_krylov, "Environ": Environ},
    "renormalizer.mps.gs": {"hop_expr": hop_expr},
}


def install():
    """Replace the reference's sweep kernels by the engine's (idempotent)."""
    for modname, repl in _TARGETS.items():
        mod = importlib.import_module(modname)
        for name, fn in repl.items():
            key = (modname, name)
            if key not in _saved:
                _saved[key] = getattr(mod, name)
            setattr(mod, name, fn)
    if not _orig_hop:
        _orig_hop.append(_saved[("renormalizer.mps.mps", "hop_expr")])


def uninstall():
    """Put the reference's own functions back."""
    for (modname, name), orig in _saved.items():
        setattr(importlib.import_module(modname), name, orig)
    _saved.clear()
    _orig_hop.clear()
