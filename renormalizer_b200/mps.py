"""Matrix product states on the GPU and the TDVP projector-splitting sweeps.

Drop-in for the parts of renormalizer.mps.Mps (mps/mps.py, mps/mp.py) that
the sweep path uses:

* constructors ``random`` (mps.py:119-185), ``hartree_product_state``
  (187-256), ``load`` / ``dump`` (npz protocol 0.4, mp.py:1085-1113 and
  mps.py:352-386);
* QN bookkeeping ``qn``, ``qnidx``, ``qntot``, ``to_right`` with
  ``move_qnidx``, ``_get_big_qn``, ``iter_idx_list``, ``_switch_direction``
  (mp.py:159-352);
* ``_update_mps`` (mp.py:651-888), ``_push_cano`` / ``canonicalise``
  (890-922), ``compress`` (437-511);
* ``evolve`` with ``tdvp_ps`` (mps.py:1267-1404) and ``tdvp_ps2``
  (1406-1517), ``normalize`` (2025-2059), ``expectation`` / ``expectations``
  / ``e_occupations`` (471-609), ``expand_bond_dimension`` (1934-2023, with
  the random or the hint-MPO expander), ``compressed_sum`` (lib.py:417-440).

Site tensors are device tensors in the reference layout (M_l, d, M_r); QN
labels are small host integer arrays.  Every contraction, vector operation
and QN block move runs in libreno_b200.
"""
from __future__ import annotations

import logging
import os
from collections import Counter
from typing import Dict, List, Optional, Union

import numpy as np
import torch

from ._native import Engine
from .backend import backend
from .configs import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, OptimizeConfig
from .hop_expr import HeffOperator, as_device
from .krylov import expm_krylov
from .lib import Environ, contract_one_site
from .model import Model, Op
from .mpo import Mpo
from .svd_qn import (qn_sectors, add_outer, get_qn_mask, qr_split, qr_split_batch, select_basis_indices, svd_truncate,
                     svd_truncate_batch)
from .svd_qn import refine as svd_refine

logger = logging.getLogger(__name__)


def _krylov_stats(steps):
    if not steps:
        return None
    a = np.asarray(steps, dtype=float)
    return {"nobs": int(a.size), "minmax": (int(a.min()), int(a.max())), "mean": float(a.mean()),
            "counts": [int(x) for x in steps]}


class TruncRequest:
    """A truncation a sweep generator yields (svd_truncate's keyword
    arguments); it receives the TruncatedSplit back."""

    def __init__(self, kwargs: dict):
        self.kwargs = kwargs


class QrRequest:
    """A canonicalising QR / RQ a sweep generator yields (qr_split's keyword
    arguments); it receives qr_split's result back."""

    def __init__(self, kwargs: dict):
        self.kwargs = kwargs


class Mps:
    is_mps = True
    is_mpo = False
    is_mpdm = False

    # ------------------------------------------------------------ construction
    def __init__(self):
        self._mp: List[torch.Tensor] = []
        self.dtype = backend.real_dtype
        self.model: Optional[Model] = None
        self.compress_config = CompressConfig()
        self.optimize_config = OptimizeConfig()
        self.evolve_config = EvolveConfig()
        self.qn: List[np.ndarray] = []
        self.qnidx: Optional[int] = None
        self.qntot: Optional[np.ndarray] = None
        self.to_right: Optional[bool] = None
        self.coeff: Union[float, complex] = 1

    @classmethod
    def from_arrays(cls, model: Model, sites, qn, qnidx, qntot, to_right) -> "Mps":
        mps = cls()
        mps.model = model
        cplx = any(np.iscomplexobj(s) if isinstance(s, np.ndarray) else s.is_complex() for s in sites)
        mps.dtype = backend.complex_dtype if cplx else backend.real_dtype
        for s in sites:
            mps.append(s)
        mps.qn = [np.asarray(q, dtype=int).reshape(len(q), -1) for q in qn]
        mps.qnidx = int(qnidx)
        mps.qntot = np.asarray(qntot, dtype=int).reshape(-1)
        mps.to_right = bool(to_right)
        return mps

    @classmethod
    def random(cls, model: Model, qntot, m_max, percent=1.0) -> "Mps":
        """mps.py:119-185: a random left-canonical MPS.  The random symmetric
        blocks are drawn from numpy's global RNG like the reference; their
        eigendecompositions and the column selection run on the device."""
        mps = cls()
        mps.model = model
        if isinstance(qntot, (int, np.integer)):
            qntot = np.array([qntot])
        qn_size = len(qntot)
        assert qn_size == model.qn_size
        qn = [np.zeros((1, qn_size), dtype=int)]
        dim_list = [1]
        sites = []
        dev = backend.device
        for imps in range(model.nsite - 1):
            qnbig = add_outer(qn[imps], model.basis[imps].sigmaqn).reshape(-1, qn_size)
            u_blocks, s_set, qnset = [], [], []
            for iblock in qn_sectors(qnbig):
                if np.all(np.array(qntot) < np.array(iblock)):
                    continue
                indices = [i for i, x in enumerate(qnbig) if tuple(x) == iblock]
                a = np.random.random([len(indices), len(indices)]) - 0.5
                a = torch.from_numpy(a + a.T).to(dev)
                s, u = torch.linalg.eigh(a)
                u_blocks.append((indices, u))
                s_set.append(s.cpu().numpy())
                qnset += [iblock] * len(indices)
            s_set = np.concatenate(s_set)
            m2 = m_max[imps + 1] if isinstance(m_max, (list, tuple, np.ndarray)) else m_max
            sidx = select_basis_indices(s_set, qnset, m2, percent)
            mt = torch.zeros((len(qnbig), len(sidx)), dtype=torch.float64, device=dev)
            offs = np.cumsum([0] + [u.shape[1] for _, u in u_blocks])
            sel = np.asarray(sidx)
            blk = np.searchsorted(offs, sel, side="right") - 1
            for bi, (idx, u) in enumerate(u_blocks):
                outs = np.nonzero(blk == bi)[0]
                if len(outs) == 0:
                    continue
                r = torch.as_tensor(idx, device=dev)[:, None]
                c = torch.as_tensor(outs, device=dev)[None, :]
                mt[r, c] = u[:, torch.as_tensor(sel[outs] - offs[bi], device=dev)]
            dim_list.append(len(sidx))
            sites.append(mt.reshape((dim_list[imps], -1, dim_list[imps + 1])))
            qn.append(np.array([qnset[i] for i in sidx]).reshape(len(sidx), -1))
        qn.append(np.zeros((1, qn_size), dtype=int))
        dim_list.append(1)
        last = np.random.random([dim_list[-2], model.pbond_list[-1], dim_list[-1]]) - 0.5
        qnmat = add_outer(qn[-2], model.basis[-1].sigmaqn)
        last[~get_qn_mask(qnmat, qntot)] = 0
        last /= np.linalg.norm(last.flatten())
        sites.append(last)
        return cls.from_arrays(model, sites, qn, len(sites) - 1, qntot, False)

    @classmethod
    def hartree_product_state(cls, model: Model, condition: Dict = None, qn_idx: int = None) -> "Mps":
        """mps.py:187-256"""
        condition = dict(condition or {})
        qn_size = model.qn_size
        qn = [np.zeros((1, qn_size), dtype=int)]
        cond = {model.dof_to_siteidx[k]: v for k, v in condition.items()}
        assert len(cond) == len(condition)
        sites = []
        for isite, b in enumerate(model.basis):
            ms = np.zeros((1, b.nbas, 1))
            st = cond.pop(isite, 0)
            if isinstance(st, (int, np.integer)):
                ms[0, st, 0] = 1.0
                q = b.sigmaqn[st]
            else:
                ms[0, :, 0] = st
                allq = np.array(b.sigmaqn)[np.nonzero(st)]
                if not np.allclose(allq.std(axis=0), 0):
                    raise ValueError("Quantum numbers are mixed in the condition.")
                q = allq[0]
            sites.append(ms)
            qn.append(qn[-1] + np.asarray(q).reshape(1, qn_size))
        if cond:
            raise ValueError(f"Condition not completely used: {cond}")
        mps = cls.from_arrays(model, sites, qn, model.nsite, qn[-1][0], False)
        mps.move_qnidx(model.nsite - 1 if qn_idx is None else qn_idx)
        mps.to_right = False
        return mps

    @classmethod
    def load(cls, model: Model, fname: str) -> "Mps":
        """npz protocol 0.1-0.4 reader (mps.py:352-386, mp.py:36-58)."""
        d = np.load(fname, allow_pickle=True)
        n = int(d["nsites"])
        sites = [d[f"mt_{i}"] for i in range(n)]
        if f"subqn_0" in d.files:
            qn = [d[f"subqn_{i}"].astype(int) for i in range(n + 1)]
        else:
            qn = [np.asarray(q, dtype=int) for q in d["qn"]]
        version = str(d["version"]) if "version" in d.files else "0.4"
        if version == "0.1":
            to_right = bool(d["left"])
        else:
            to_right = bool(d["to_right"])
        mps = cls.from_arrays(model, sites, qn, int(d["qnidx"]), d["qntot"].astype(int), to_right)
        if version in ("0.3", "0.4") and "coeff" in d.files:
            mps.coeff = d["coeff"].item(0)
        elif version == "0.2" and "tdh_wfns" in d.files:
            mps.coeff = d["tdh_wfns"][-1]
        return mps

    def dump(self, fname, other_attrs=None):
        """npz protocol 0.4 writer (mp.py:1085-1113)."""
        data = {"version": "0.4", "nsites": len(self)}
        for i in range(len(self._mp)):
            data[f"mt_{i}"] = self._site_for_file(i).cpu().numpy()
        data["qnidx"] = self.qnidx
        data["qntot"] = self.qntot
        arr = np.empty(len(self.qn), object)
        arr[:] = self.qn
        data["qn"] = arr
        data["to_right"] = self.to_right
        data["coeff"] = self.coeff
        for i, q in enumerate(self.qn):
            data[f"subqn_{i}"] = q
        for a in other_attrs or []:
            data[a] = getattr(self, a)
        np.savez(fname, **data)

    def _site_for_file(self, i) -> torch.Tensor:
        return self._mp[i]

    # ------------------------------------------------------------ container
    def _to_dev(self, array) -> torch.Tensor:
        t = as_device(array)
        if self.dtype == torch.complex128 and not t.is_complex():
            t = t.to(torch.complex128)
        elif self.dtype == torch.float64 and t.is_complex():
            raise AssertionError("forbid unchecked casting of a complex site into a real MPS")
        return t.contiguous()

    def append(self, array):
        t = self._to_dev(array)
        if self._mp:
            assert t.shape[0] == self._mp[-1].shape[-1]
        if t.shape[1] != self.pbond_list[len(self._mp)]:
            raise ValueError("Matrix physical bond dimension does not match system information")
        self._mp.append(t)

    def __len__(self):
        return len(self._mp)

    @property
    def site_num(self):
        return len(self._mp)

    def __getitem__(self, i) -> torch.Tensor:
        return self._mp[i]

    def __setitem__(self, i, array):
        t = self._to_dev(array)
        if t.shape[1] != self.pbond_list[i if i >= 0 else len(self) + i]:
            raise ValueError("Matrix physical bond dimension does not match system information")
        self._mp[i] = t

    def __iter__(self):
        return iter(self._mp)

    @property
    def bond_dims(self) -> List[int]:
        return [int(t.shape[0]) for t in self._mp] + [int(self._mp[-1].shape[-1])] if self._mp else []

    @property
    def pbond_list(self):
        return self.model.pbond_list

    @property
    def is_complex(self):
        return self.dtype == torch.complex128

    def metacopy(self) -> "Mps":
        new = self.__class__.__new__(self.__class__)
        new._mp = [None] * len(self)
        new.dtype = self.dtype
        new.model = self.model
        new.compress_config = self.compress_config.copy()
        new.optimize_config = self.optimize_config.copy()
        new.evolve_config = self.evolve_config.copy()
        new.qn = [q.copy() for q in self.qn]
        new.qnidx = self.qnidx
        new.qntot = None if self.qntot is None else self.qntot.copy()
        new.to_right = self.to_right
        new.coeff = self.coeff
        return new

    def copy(self) -> "Mps":
        new = self.metacopy()
        new._mp = [t.clone() for t in self._mp]
        return new

    def conj(self) -> "Mps":
        new = self.metacopy()
        new._mp = [t.conj().resolve_conj().contiguous() for t in self._mp]
        new.coeff = np.conjugate(self.coeff)
        return new

    def to_complex(self, inplace=False) -> "Mps":
        new = self if inplace else self.metacopy()
        new.dtype = backend.complex_dtype
        new._mp = [t.to(torch.complex128).contiguous() if not t.is_complex() else (t if inplace else t.clone())
                   for t in self._mp]
        new.coeff = complex(self.coeff)
        return new

    def todense(self) -> np.ndarray:
        res = np.ones((1, 1, 1))
        for mt in self._mp:
            m = mt.cpu().numpy()
            res = np.tensordot(res, m, axes=1).reshape(1, res.shape[1] * m.shape[1], m.shape[-1])
        return res[0, :, 0]

    # ------------------------------------------------------------ QN bookkeeping
    def _get_sigmaqn(self, idx):
        return self.model.basis[idx].sigmaqn

    def build_empty_qn(self):
        self.qntot = np.zeros(self.model.qn_size, dtype=int)
        if self.qnidx is None:
            self.qnidx = len(self) - 1
        self.qn = [np.zeros((d, self.model.qn_size), dtype=int) for d in self.bond_dims]
        if self.to_right is None:
            self.to_right = False

    def move_qnidx(self, dstidx: int):
        """mp.py:159-172"""
        for idx in range(self.qnidx + 1, self.site_num + 1):
            self.qn[idx] = self.qntot - self.qn[idx]
        for idx in range(self.site_num, dstidx, -1):
            self.qn[idx] = self.qntot - self.qn[idx]
        self.qnidx = dstidx

    def iter_idx_list(self, full: bool, stop_idx: int = None):
        if self.to_right:
            last = stop_idx if stop_idx is not None else (self.site_num if full else self.site_num - 1)
            return range(self.qnidx, last)
        last = stop_idx if stop_idx is not None else (-1 if full else 0)
        return range(self.qnidx, last, -1)

    def _switch_direction(self):
        assert self.to_right is not None
        if self.to_right:
            self.qnidx = self.site_num - 1
            self.to_right = False
        else:
            self.qnidx = 0
            self.to_right = True

    def _get_big_qn(self, cidx: List[int], with_mat: bool = True):
        """mp.py:308-352.  ``with_mat=False`` skips the (rows x cols x qn_size)
        outer sum qnmat (None is returned in its place): the truncation only
        needs the row and column labels, and at M = 256 with two 16-level
        sites qnmat has 16.7 M entries per bond."""
        if len(cidx) == 2:
            cidx = sorted(cidx)
            assert cidx[0] + 1 == cidx[1]
        assert self.qnidx in cidx
        sig = [np.array(self._get_sigmaqn(i)) for i in cidx]
        qnl = np.array(self.qn[cidx[0]])
        qnr = np.array(self.qn[cidx[-1] + 1])
        if len(cidx) == 1:
            if self.to_right:
                qnbigl, qnbigr = add_outer(qnl, sig[0]), qnr
            else:
                qnbigl, qnbigr = qnl, add_outer(sig[0], qnr)
        else:
            qnbigl, qnbigr = add_outer(qnl, sig[0]), add_outer(sig[1], qnr)
        return qnbigl, qnbigr, (add_outer(qnbigl, qnbigr) if with_mat else None)

    @property
    def is_left_canonical(self):
        return self.qnidx == self.site_num - 1

    @property
    def is_right_canonical(self):
        return self.qnidx == 0

    def check_left_canonical(self, atol=None):
        atol = backend.canonical_atol if atol is None else atol
        for t in self._mp[:-1]:
            m = t.reshape(-1, t.shape[-1])
            if not torch.allclose(m.mH @ m, torch.eye(m.shape[1], dtype=m.dtype, device=m.device), atol=atol):
                return False
        return True

    def check_right_canonical(self, atol=None):
        atol = backend.canonical_atol if atol is None else atol
        for t in self._mp[1:]:
            m = t.reshape(t.shape[0], -1)
            if not torch.allclose(m @ m.mH, torch.eye(m.shape[0], dtype=m.dtype, device=m.device), atol=atol):
                return False
        return True

    def ensure_left_canonical(self):
        if self.to_right or self.qnidx != self.site_num - 1 or not self.check_left_canonical():
            self.move_qnidx(0)
            self.to_right = True
            return self.canonicalise()
        return self

    def ensure_right_canonical(self):
        if (not self.to_right) or self.qnidx != 0 or not self.check_right_canonical():
            self.move_qnidx(self.site_num - 1)
            self.to_right = False
            return self.canonicalise()
        return self

    # ------------------------------------------------------------ canonical form
    def _absorb_right(self, idx, vt: torch.Tensor):
        """self[idx+1] = vt @ self[idx+1] (tensordot axes=1)"""
        nxt = self._mp[idx + 1]
        eng = Engine.get(nxt.device)
        out = eng.matmul(vt, nxt.reshape(nxt.shape[0], -1))
        self._mp[idx + 1] = out.reshape((vt.shape[0],) + tuple(nxt.shape[1:])).to(self.dtype)

    def _absorb_left(self, idx, u: torch.Tensor):
        """self[idx-1] = self[idx-1] @ u"""
        prv = self._mp[idx - 1]
        eng = Engine.get(prv.device)
        out = eng.matmul(prv.reshape(-1, prv.shape[-1]), u)
        self._mp[idx - 1] = out.reshape(tuple(prv.shape[:-1]) + (u.shape[1],)).to(self.dtype)

    def _push_cano(self, idx):
        """mp.py:890-908 with _update_ms (245-295, sigma=None)"""
        self._push_cano_place(idx, qr_split(**self._push_cano_call(idx)))

    def _push_cano_call(self, idx) -> dict:
        qnbigl, qnbigr, _ = self._get_big_qn([idx], with_mat=False)
        return dict(coef=self._mp[idx], qnbigl=qnbigl, qnbigr=qnbigr, qntot=self.qntot,
                    system="L" if self.to_right else "R")

    def _push_cano_place(self, idx, res):
        mt = self._mp[idx]
        u, qnlset, vt, qnrset = res
        m_trunc = u.shape[1]
        pd = list(mt.shape[1:-1])
        if self.to_right:
            self._absorb_right(idx, vt)
            self._mp[idx] = u.reshape([u.shape[0] // int(np.prod(pd))] + pd + [m_trunc]).to(self.dtype)
            self.qn[idx + 1] = np.array(qnlset).reshape(m_trunc, -1)
            self.qnidx = idx + 1
        else:
            self._absorb_left(idx, u)
            self._mp[idx] = vt.reshape([m_trunc] + pd + [vt.shape[1] // int(np.prod(pd))]).to(self.dtype)
            self.qn[idx] = np.array(qnrset).reshape(m_trunc, -1)
            self.qnidx = idx - 1

    def canonicalise(self, stop_idx: int = None):
        if self.to_right:
            assert self.qnidx == 0
        else:
            assert self.qnidx == self.site_num - 1
        idx = None
        for idx in self.iter_idx_list(full=False, stop_idx=stop_idx):
            self._push_cano(idx)
        if (not self.to_right and idx == 1) or (self.to_right and idx == self.site_num - 2):
            self._switch_direction()
        return self

    def compress(self, temp_m_trunc=None, ret_s=False):
        """mp.py:437-511 (SVD sweep, full_matrices=False, sigma to the next site).
        ``ret_s`` also returns the per-bond singular values (all of them,
        descending), zero-padded to a rectangle."""
        if self.to_right:
            assert self.qnidx == 0
        else:
            assert self.qnidx == self.site_num - 1
        if self.compress_config.bonddim_should_set:
            self.compress_config.set_bonddim(len(self) + 1)
        s_list = []
        for idx in self.iter_idx_list(full=False):
            mt = self._mp[idx]
            qnbigl, qnbigr, _ = self._get_big_qn([idx], with_mat=False)
            left = self.to_right

            def m_fn(sigma, idx=idx, left=left):
                if temp_m_trunc is None:
                    return self.compress_config.compute_m_trunc(sigma, idx, left)
                if isinstance(temp_m_trunc, (list, tuple, np.ndarray)):
                    m = temp_m_trunc[idx + 1 if left else idx]
                else:
                    m = temp_m_trunc
                return len(sigma) if not np.isfinite(m) else min(int(m), len(sigma))

            if temp_m_trunc is None:
                kcap = self.compress_config.fixed_cap(idx, left)
            elif isinstance(temp_m_trunc, (list, tuple, np.ndarray)):
                kcap = temp_m_trunc[idx + 1 if left else idx]
            else:
                kcap = temp_m_trunc
            kcap = int(kcap) if kcap is not None and np.isfinite(kcap) else None
            res = svd_truncate(mt, qnbigl, qnbigr, self.qntot, keep_left=left, m_trunc_fn=m_fn,
                               full_matrices=False, kcap=kcap)
            s_list.append(np.asarray(res.sigma))
            pd = list(mt.shape[1:-1])
            if left:
                self._absorb_right(idx, res.right)
                self._mp[idx] = res.left.reshape([res.left.shape[0] // int(np.prod(pd))] + pd + [res.mdim])
                self.qn[idx + 1] = res.qn
                self.qnidx = idx + 1
            else:
                self._absorb_left(idx, res.left)
                self._mp[idx] = res.right.reshape([res.mdim] + pd + [res.right.shape[1] // int(np.prod(pd))])
                self.qn[idx] = res.qn
                self.qnidx = idx - 1
        self._switch_direction()
        if not ret_s:
            return self
        width = max(len(x) for x in s_list)
        return self, np.array([np.pad(x, (0, width - len(x))) for x in s_list])

    def _update_mps(self, cstruct: torch.Tensor, cidx: List[int], qnbigl, qnbigr, percent=0):
        """mp.py:651-888, one root, no OFS: QN-blocked SVD truncation of the
        active coefficient and placement of the kept / complementary parts."""
        res = svd_truncate(**self._truncation_call(cstruct, cidx, qnbigl, qnbigr, percent))
        self._place_truncation(res, cidx, qnbigl, qnbigr)

    def _truncation_call(self, cstruct: torch.Tensor, cidx: List[int], qnbigl, qnbigr, percent=0) -> dict:
        """svd_truncate's arguments for the truncation of _update_mps"""
        if self.compress_config.bonddim_should_set:
            self.compress_config.set_bonddim(len(self) + 1)
        left = bool(self.to_right)
        bond_site = cidx[0] if left else cidx[-1]
        cfg = self.compress_config
        return dict(coef=cstruct, qnbigl=qnbigl, qnbigr=qnbigr, qntot=self.qntot, keep_left=left,
                    m_trunc_fn=lambda s: cfg.compute_m_trunc(s, bond_site, left), percent=percent,
                    kcap=cfg.fixed_cap(bond_site, left), refine_floor=svd_refine.sweep_floor)

    def _place_truncation(self, res, cidx: List[int], qnbigl, qnbigr):
        """the kept / complementary parts of a truncation into the sites (mp.py:779-888)"""
        left = bool(self.to_right)
        ldims = list(qnbigl.shape[:-1])
        rdims = list(qnbigr.shape[:-1])
        lmat = res.left.reshape(ldims + [res.mdim])
        rmat = res.right.reshape([res.mdim] + rdims)
        n = len(self)
        if len(cidx) == 1:
            c0 = cidx[0]
            if left:
                self._mp[c0] = lmat.to(self.dtype)
                if c0 != n - 1:
                    self._absorb_right(c0, res.right)
                    self.qn[c0 + 1] = res.qn
                    self.qnidx = c0 + 1
                else:
                    eng = Engine.get(res.right.device)
                    self._mp[c0] = eng.matmul(lmat.reshape(-1, res.mdim).contiguous(), res.right).reshape(
                        self._mp[c0].shape[:-1] + (-1,))
                    self.qnidx = n - 1
            else:
                self._mp[c0] = rmat.to(self.dtype)
                if c0 != 0:
                    self._absorb_left(c0, res.left)
                    self.qn[c0] = res.qn
                    self.qnidx = c0 - 1
                else:
                    eng = Engine.get(res.left.device)
                    self._mp[c0] = eng.matmul(res.left, rmat.reshape(res.mdim, -1).contiguous()).reshape(
                        (-1,) + tuple(rmat.shape[1:]))
                    self.qnidx = 0
        else:
            self._mp[cidx[0]] = lmat.to(self.dtype).contiguous()
            self._mp[cidx[1]] = rmat.to(self.dtype).contiguous()
            self.qnidx = cidx[1] if left else cidx[0]
            self.qn[cidx[1]] = res.qn
        return None

    # ------------------------------------------------------------ algebra
    def dot(self, other: "Mps") -> complex:
        """mp.py:933-956: sum over all indices of self[i] (as given) x other[i]"""
        e0 = torch.ones((1, 1), dtype=torch.complex128, device=self._mp[0].device)
        eng = Engine.get(e0.device)
        for mt1, mt2 in zip(self._mp, other._mp):
            # e0[x, y] -> e0 @ mt2 : (x, p, y') ; contract (x, p) with mt1
            t = eng.matmul(e0, mt2.reshape(mt2.shape[0], -1)).reshape(e0.shape[0], -1)
            t = t.reshape(e0.shape[0] * mt2.shape[1], mt2.shape[2])
            m1 = mt1.reshape(mt1.shape[0] * mt1.shape[1], mt1.shape[2])
            e0 = eng.matmul(m1.transpose(0, 1), t)
        return complex(e0[0, 0].item())

    @property
    def mp_norm(self) -> float:
        res = self.conj().dot(self).real
        if res < 0:
            assert abs(res) < 1e-8
            res = 0.0
        return float(np.sqrt(res))

    @property
    def norm(self):
        return float(np.linalg.norm(self.coeff)) * self.mp_norm

    def scale(self, val, inplace=False) -> "Mps":
        new = self if inplace else self.copy()
        if np.iscomplex(val):
            new.to_complex(inplace=True)
        else:
            val = float(np.real(val))
        new._mp[new.qnidx] = (new._mp[new.qnidx] * val).contiguous()
        return new

    def normalize(self, kind):
        """mps.py:2025-2059"""
        n = self.mp_norm
        if kind == "mps_only":
            new_coeff = self.coeff
        elif kind == "mps_and_coeff":
            new_coeff = self.coeff / np.linalg.norm(self.coeff)
        elif kind == "mps_norm_to_coeff":
            new_coeff = self.coeff * n
        else:
            raise ValueError(f"kind={kind} is not valid.")
        self.scale(1.0 / n, inplace=True)
        self.coeff = new_coeff
        return self

    def add(self, other: "Mps") -> "Mps":
        """mp.py:374-435 (MPS direct sum)"""
        assert np.all(self.qntot == other.qntot) and len(self) == len(other)
        new = self.metacopy()
        if other.is_complex or self.is_complex:
            new.dtype = backend.complex_dtype
        dt = new.dtype
        n = len(self)
        sites = []
        for i in range(n):
            a, b = self._mp[i].to(dt), other._mp[i].to(dt)
            if i == 0:
                sites.append(torch.cat([a, b], dim=2))
            elif i == n - 1:
                sites.append(torch.cat([a, b], dim=0))
            else:
                t = torch.zeros((a.shape[0] + b.shape[0], a.shape[1], a.shape[2] + b.shape[2]), dtype=dt,
                                device=a.device)
                t[: a.shape[0], :, : a.shape[2]] = a
                t[a.shape[0]:, :, a.shape[2]:] = b
                sites.append(t)
        new._mp = [s.contiguous() for s in sites]
        new.move_qnidx(other.qnidx)
        new.to_right = other.to_right
        new.qn = [np.concatenate([q1, q2]) for q1, q2 in zip(self.qn, other.qn)]
        new.qn[0] = np.zeros((1, new.qn[0].shape[1]), dtype=int)
        new.qn[-1] = np.zeros((1, new.qn[0].shape[1]), dtype=int)
        return new

    def __add__(self, other):
        return self.add(other)

    # ------------------------------------------------------------ expectations
    def expectation(self, mpo: Mpo, self_conj: "Mps" = None) -> Union[float, complex]:
        """mps.py:471-525: <psi|O|psi> through a right-environment sweep."""
        conj = self_conj if self_conj is not None else self.conj()
        t = torch.ones((1, 1, 1), dtype=torch.float64, device=self._mp[0].device)
        for idx in range(len(self) - 1, -1, -1):
            t = contract_one_site(t, self._mp[idx], mpo[idx], "R", ms_conj=conj[idx], prec="fp64")
        val = complex(t.reshape(-1)[0].item())
        if np.isclose(val.imag, 0):
            return float(val.real)
        return val

    def expectations(self, mpos: List[Mpo], self_conj: "Mps" = None, opt: bool = True) -> np.ndarray:
        """mps.py:527-575.  With ``opt`` the left and right environments of the
        site-tensor sequences that several operators share (prefixes from the
        left, suffixes from the right) are contracted once
        (_construct_freq_environ / _get_freq_environ, mps.py:2103-2169; site
        tensors are identified by content, not by a hash of it); every operator
        then contracts only its own middle sites.  One host transfer for all
        results."""
        if not opt:
            res = np.array([self.expectation(m, self_conj) for m in mpos])
            return np.real(res) if np.allclose(np.imag(res), 0) else res
        n = len(self)
        conj = self_conj._mp if self_conj is not None else [t.conj().resolve_conj() for t in self._mp]
        key_of, tensor_of = {}, {}
        seqs = []
        for mpo in mpos:
            seq = []
            for i in range(n):
                a = np.ascontiguousarray(mpo.numpy(i))
                k = (a.shape, a.dtype.str, a.tobytes())
                if k not in key_of:
                    key_of[k] = len(key_of)
                    tensor_of[key_of[k]] = mpo[i]
                seq.append(key_of[k])
            seqs.append(seq)

        def freq_environ(domain):
            counter = Counter()
            for seq in seqs:
                for i in range(1, len(seq) + 1):
                    counter.update([tuple(seq[:i]) if domain == "L" else tuple(reversed(seq[-i:]))])
            common = sorted(counter.items(), key=lambda x: (-x[1], len(x[0])))
            chosen = []
            for keys, cnt in common:
                if cnt == 1 or n < len(chosen):
                    break
                chosen.append(keys)
            out = {(): torch.ones((1, 1, 1), dtype=torch.float64, device=self._mp[0].device)}
            for keys in chosen:
                idx = len(keys) - 1 if domain == "L" else n - len(keys)
                out[keys] = contract_one_site(out[keys[:-1]], self._mp[idx], tensor_of[keys[-1]], domain,
                                              ms_conj=conj[idx], prec="fp64")
            return out

        def lookup(env, seq, domain, max_len):
            it = seq if domain == "L" else list(reversed(seq))
            keys = []
            for k in it:
                keys.append(k)
                if tuple(keys) not in env or max_len < len(keys):
                    keys.pop()
                    break
            i = len(keys) - 1 if domain == "L" else n - len(keys)
            return env[tuple(keys)], i

        l_env, r_env = freq_environ("L"), freq_environ("R")
        vals = []
        for mpo, seq in zip(mpos, seqs):
            left, li = lookup(l_env, seq, "L", np.inf)
            right, ri = lookup(r_env, seq, "R", n - li - 1)
            for i in range(li + 1, ri):
                left = contract_one_site(left, self._mp[i], mpo[i], "L", ms_conj=conj[i], prec="fp64")
            vals.append((left.reshape(-1).to(torch.complex128) * right.reshape(-1).to(torch.complex128)).sum())
        res = torch.stack(vals).cpu().numpy()
        return np.real(res) if np.allclose(np.imag(res), 0) else res

    def _overlap_environs(self):
        """conj sites and the left / right environments of <psi|psi> (identity
        MPO) at every bond: left[i] covers sites < i, right[i] sites >= i."""
        n = len(self)
        dev = self._mp[0].device
        conj = [t.conj().resolve_conj().contiguous() for t in self._mp]
        eye = [torch.eye(t.shape[1], dtype=torch.float64, device=dev).reshape(1, t.shape[1], t.shape[1], 1)
               for t in self._mp]
        left = [torch.ones((1, 1, 1), dtype=torch.float64, device=dev)]
        for i in range(n - 1):
            left.append(contract_one_site(left[-1], self._mp[i], eye[i], "L", ms_conj=conj[i], prec="fp64"))
        right = [None] * (n + 1)
        right[n] = torch.ones((1, 1, 1), dtype=torch.float64, device=dev)
        for i in range(n - 1, 0, -1):
            right[i] = contract_one_site(right[i + 1], self._mp[i], eye[i], "R", ms_conj=conj[i], prec="fp64")
        return conj, left, right

    def calc_1site_rdm(self, idx=None) -> Dict[int, np.ndarray]:
        """mps.py:1547-1598: rho_i[p, q] = sum L[a, a'] conj(ms[a, p, b])
        R[b, b'] ms[a', q, b'] from the overlap environments, three engine
        GEMMs per site; one host transfer."""
        n = len(self)
        if idx is None:
            idx = list(range(n))
        elif isinstance(idx, (int, np.integer)):
            idx = [int(idx)]
        elif isinstance(idx, (list, tuple)):
            idx = list(idx)
        else:
            raise AssertionError("idx must be None, an int, a list or a tuple")
        eng = Engine.get(self._mp[0].device)
        conj, left, right = self._overlap_environs()
        out = []
        for i in idx:
            ms = self._mp[i]
            mb, d, mk = ms.shape
            L2 = left[i].reshape(left[i].shape[0], left[i].shape[-1])
            R2 = right[i + 1].reshape(right[i + 1].shape[0], right[i + 1].shape[-1])
            U = eng.matmul(L2, ms.reshape(mb, d * mk))                               # (a, (q, b'))
            V = eng.matmul(U.reshape(L2.shape[0] * d, mk), R2.transpose(0, 1))       # ((a, q), b)
            X = conj[i].permute(1, 0, 2).reshape(d, -1).contiguous()                 # (p, (a, b))
            Y = V.reshape(L2.shape[0], d, R2.shape[0]).permute(1, 0, 2).reshape(d, -1).contiguous()
            out.append(eng.matmul(X, Y.transpose(0, 1)))                             # (p, q)
        host = [t.cpu().numpy() for t in out]
        return {i: h for i, h in zip(idx, host)}

    def calc_bond_singular_values(self) -> np.ndarray:
        """mps.py:1759-1772: sigma at every bond from an untruncated SVD sweep
        of a right-canonical copy, zero-padded to a rectangle."""
        mps = self.copy()
        mps.ensure_right_canonical()
        _, s_array = mps.compress(temp_m_trunc=np.inf, ret_s=True)
        return s_array

    def calc_bond_entropy(self, s_array: np.ndarray = None) -> np.ndarray:
        """mps.py:1774-1793: von Neumann entropy -sum p ln p, p = sigma^2 / sum sigma^2."""
        if s_array is None:
            s_array = self.calc_bond_singular_values()
        res = []
        for sig in s_array:
            p = np.asarray(sig, dtype=float) ** 2
            p = p / p.sum()
            p = p[p > 0]
            res.append(float(-(p * np.log(p)).sum()))
        return np.array(res)

    def site_expectations(self, site_ops: Dict[int, np.ndarray]) -> Dict[int, float]:
        """<psi|O_i|psi> for one-site operators, with left/right overlap
        environments shared by all sites (the quantity e_occupations returns)."""
        conj, left, right = self._overlap_environs()
        out = {}
        vals = []
        for i, op in site_ops.items():
            W = as_device(np.asarray(op).reshape(1, op.shape[0], op.shape[1], 1))
            t = contract_one_site(left[i], self._mp[i], W, "L", ms_conj=conj[i], prec="fp64")
            vals.append((i, (t.reshape(-1) * right[i + 1].reshape(-1)).sum()))
        host = torch.stack([v for _, v in vals]).cpu().numpy() if vals else []
        for (i, _), v in zip(vals, host):
            out[i] = float(np.real(v))
        return out

    @property
    def e_occupations(self) -> np.ndarray:
        """mps.py:595-609: <a^dagger_i a_i> for every electronic DoF (model order)."""
        sites = [self.model.dof_to_siteidx[d] for d in self.model.e_dofs]
        ops = {s: self.model.basis[s].op_mat(r"a^\dagger a") for s in sites}
        res = self.site_expectations(ops)
        return np.array([res[s] for s in sites])

    @property
    def ph_occupations(self) -> np.ndarray:
        sites = [self.model.dof_to_siteidx[d] for d in self.model.v_dofs]
        ops = {s: self.model.basis[s].op_mat("n") for s in sites}
        res = self.site_expectations(ops)
        return np.array([res[s] for s in sites])

    # ------------------------------------------------------------ bond expansion
    @classmethod
    def ground_state(cls, model: Model, max_entangled: bool = False, normalize: bool = True) -> "Mps":
        """mps.py:259-350: electrons empty; SHO modes (and spins) in their
        ground state, or with ``max_entangled`` in the uniform T = infinity
        state (1 / sqrt(d) per level, 1 without ``normalize``); QN 0."""
        sites = []
        for b in model.basis:
            ms = np.zeros((1, b.nbas, 1))
            if max_entangled and (b.is_phonon or b.is_spin):
                ms[0, :, 0] = 1.0 / np.sqrt(b.nbas) if normalize else 1.0
            elif b.is_phonon or b.is_spin or b.is_electron:
                ms[0, 0, 0] = 1.0
            else:
                raise NotImplementedError(f"ground state of basis {type(b).__name__}")
            sites.append(ms)
        qn = [np.zeros((1, model.qn_size), dtype=int) for _ in range(model.nsite + 1)]
        return cls.from_arrays(model, sites, qn, model.nsite - 1, np.zeros(model.qn_size, dtype=int), False)

    def _expansion_ex_state(self) -> "Mps":
        """mps.py:1943-1949: the excited product state of the hint expander"""
        assert self.model.qn_size == 1, "the excited expander state supports one QN only"
        ex = Mps.ground_state(self.model, False)
        for _ in range(int(self.qntot[0])):
            ex = Mpo.onsite(self.model, r"a^\dagger") @ ex
        return ex

    @property
    def bond_dims_exact(self) -> np.ndarray:
        """mp.py:131-142: bond dimensions of an exact factorisation"""
        pb = np.array(self.pbond_list, dtype=float)
        with np.errstate(over="ignore"):
            d1 = [1] + list(np.cumprod(pb))
            d2 = ([1] + list(np.cumprod(pb[::-1])))[::-1]
        return np.minimum(d1, d2)

    def expand_bond_dimension(self, hint_mpo=None, coef=1e-10, include_ex=True):
        """mps.py:1934-2023: add a coef-weighted expander with the missing
        bond dimension, then canonicalise, compress to max_dims and move the
        norm to coeff.  Without ``hint_mpo`` the expander is a random MPS;
        with it, the expander is the compressed sum of the normalised states
        H psi, H^2 psi, ... (psi plus the excited product state when
        ``include_ex``), grown until every bond reaches its target or stops
        growing."""
        self.compress_config.set_bonddim(len(self.bond_dims))
        m_target = np.minimum(np.array(self.compress_config.max_dims) - np.array(self.bond_dims),
                              self.bond_dims_exact).astype(int)
        if hint_mpo is None:
            expander = self.__class__.random(self.model, self.qntot, np.maximum(m_target, 1))
        else:
            if include_ex:
                ex = self._expansion_ex_state()
                ex.compress_config = self.compress_config
                ex.move_qnidx(self.qnidx)
                ex.to_right = self.to_right
                lastone = self + ex
            else:
                lastone = self
            expander_list = []
            expander_dims = np.zeros_like(m_target)
            hint_max = int(np.max(hint_mpo.bond_dims))
            while True:
                lastone = (hint_mpo @ lastone).normalize("mps_and_coeff")
                lastone = lastone.canonicalise().compress(int(np.max(m_target)))
                expander_list.append(lastone)
                expander = compressed_sum(expander_list, temp_m_trunc=m_target)
                dims = np.array(expander.bond_dims)
                if np.all(dims >= m_target):
                    break
                if np.all(dims == expander_dims):
                    logger.warning("Expander does not increase anymore. The expand target is too high")
                    m_target2 = int(np.max(m_target - expander_dims))
                    expander2 = (hint_mpo @ lastone).canonicalise().compress(max(m_target2, 1))
                    expander = expander + expander2
                    break
                expander_dims = dims
                lastone = lastone.canonicalise().compress(int(np.max(m_target) / hint_max) + 1)
        total = self + expander.scale(coef * self.norm, inplace=True)
        total.canonicalise()
        total.compress(self.compress_config.max_dims)
        return total.normalize("mps_norm_to_coeff")

    # ------------------------------------------------------------ time evolution
    def evolve(self, mpo: Mpo, evolve_dt, normalize=True) -> "Mps":
        """mps.py:644-662"""
        new = self._drive(self._evolve_steps(mpo, evolve_dt))
        if normalize:
            new.normalize("mps_and_coeff" if np.iscomplex(evolve_dt) else "mps_only")
        return new

    def _evolve_steps(self, mpo: Mpo, evolve_dt):
        method = self.evolve_config.method
        if method == EvolveMethod.tdvp_ps:
            return self._evolve_tdvp_ps_steps(mpo, evolve_dt)
        if method == EvolveMethod.tdvp_ps2:
            return self._evolve_tdvp_ps2_steps(mpo, evolve_dt)
        raise NotImplementedError(f"{method} is outside the sweep engine (TDVP-PS / TDVP-PS2 only)")

    def _drive(self, steps):
        """Run a sweep generator, serving each local exponential it yields
        (operator, dt, vector) with expm_krylov and each truncation
        (TruncRequest) with svd_truncate; returns the new MPS."""
        try:
            req = next(steps)
            while True:
                if isinstance(req, TruncRequest):
                    req = steps.send(svd_truncate(**req.kwargs))
                elif isinstance(req, QrRequest):
                    req = steps.send(qr_split(**req.kwargs))
                else:
                    req = steps.send(self._krylov(*req))
        except StopIteration as stop:
            return stop.value

    def _krylov(self, op: HeffOperator, dt, vec: torch.Tensor):
        return expm_krylov(lambda y: op.apply(y), dt, vec.reshape(-1))

    def _evolve_tdvp_ps(self, mpo: Mpo, evolve_dt) -> "Mps":
        return self._drive(self._evolve_tdvp_ps_steps(mpo, evolve_dt))

    def _evolve_tdvp_ps2(self, mpo: Mpo, evolve_dt) -> "Mps":
        return self._drive(self._evolve_tdvp_ps2_steps(mpo, evolve_dt))

    def _evolve_tdvp_ps_steps(self, mpo: Mpo, evolve_dt):
        """mps.py:1267-1404 (Krylov propagator), as a generator that yields each
        local exponential (operator, dt, vector) and receives (vector, count)"""
        if self.evolve_config.ivp_solver != "krylov":
            raise NotImplementedError("only the Krylov propagator is part of the sweep engine")
        mps = self.copy() if np.iscomplex(evolve_dt) else self.to_complex()
        environ = Environ(mps, mpo)
        local_steps = []
        for _ in range(2):
            for imps in mps.iter_idx_list(full=True):
                system = "L" if mps.to_right else "R"
                l_array = environ.read("L", imps - 1)
                r_array = environ.read("R", imps + 1)
                shape = list(mps[imps].shape)
                hop = HeffOperator(l_array, r_array, [mpo[imps]], shape)
                mps_t, j = yield (hop, -1j * evolve_dt / 2, mps[imps])
                local_steps.append(j)
                mps_t = mps_t.reshape(shape)
                qnbigl, qnbigr, _ = mps._get_big_qn([imps], with_mat=False)
                u, qnlset, vt, qnrset = yield QrRequest(dict(coef=mps_t, qnbigl=qnbigl, qnbigr=qnbigr,
                                                             qntot=mps.qntot, system=system))
                if not mps.to_right and imps != 0:
                    mps[imps] = vt.reshape([-1] + shape[1:])
                    mps.qn[imps] = np.array(qnrset).reshape(vt.shape[0], -1)
                    mps.qnidx = imps - 1
                    r_array = environ.GetLR("R", imps, mps, mpo, itensor=r_array, method="System")
                    hop_u = HeffOperator(l_array, r_array, [], u.shape)
                    mps_u, j = yield (hop_u, 1j * evolve_dt / 2, u)
                    local_steps.append(j)
                    mps._absorb_left(imps, mps_u.reshape(u.shape))
                elif mps.to_right and imps != len(mps) - 1:
                    mps[imps] = u.reshape(shape[:-1] + [-1])
                    mps.qn[imps + 1] = np.array(qnlset).reshape(u.shape[1], -1)
                    mps.qnidx = imps + 1
                    l_array = environ.GetLR("L", imps, mps, mpo, itensor=l_array, method="System")
                    hop_v = HeffOperator(l_array, r_array, [], vt.shape)
                    mps_v, j = yield (hop_v, 1j * evolve_dt / 2, vt)
                    local_steps.append(j)
                    mps._absorb_right(imps, mps_v.reshape(vt.shape))
                else:
                    mps[imps] = mps_t
            mps._switch_direction()
        mps.evolve_config.stat = _krylov_stats(local_steps)
        return mps

    def _evolve_tdvp_ps2_steps(self, mpo: Mpo, evolve_dt):
        """mps.py:1406-1517 (Krylov propagator), as a generator like
        _evolve_tdvp_ps_steps"""
        if self.evolve_config.ivp_solver != "krylov":
            raise NotImplementedError("only the Krylov propagator is part of the sweep engine")
        mps = self.copy() if np.iscomplex(evolve_dt) else self.to_complex()
        environ = Environ(mps, mpo)
        eng = Engine.get(mps[0].device)
        local_steps = []
        for _ in range(2):
            for imps in mps.iter_idx_list(full=False):
                if mps.to_right:
                    lidx, cidx0, cidx1, ridx = range(imps - 1, imps + 3)
                    cidx2 = cidx1
                    last_idx = len(mps) - 2
                else:
                    lidx, cidx0, cidx1, ridx = range(imps - 2, imps + 2)
                    cidx2 = cidx0
                    last_idx = 1
                l_array = environ.read("L", lidx)
                r_array = environ.read("R", ridx)
                a, b = mps[cidx0], mps[cidx1]
                ms2 = eng.matmul(a.reshape(-1, a.shape[-1]), b.reshape(b.shape[0], -1))
                shape2 = [a.shape[0], a.shape[1], b.shape[1], b.shape[2]]
                hop = HeffOperator(l_array, r_array, [mpo[cidx0], mpo[cidx1]], shape2)
                mps_t, j = yield (hop, -1j * evolve_dt / 2, ms2)
                local_steps.append(j)
                mps_t = mps_t.reshape(shape2)
                qnbigl, qnbigr, _ = mps._get_big_qn([cidx0, cidx1], with_mat=False)
                res = yield TruncRequest(mps._truncation_call(mps_t, [cidx0, cidx1], qnbigl, qnbigr))
                mps._place_truncation(res, [cidx0, cidx1], qnbigl, qnbigr)
                if imps == last_idx:
                    continue
                if mps.to_right:
                    l_array = environ.GetLR("L", lidx + 1, mps, mpo, itensor=l_array, method="System")
                else:
                    r_array = environ.GetLR("R", ridx - 1, mps, mpo, itensor=r_array, method="System")
                ms1 = mps[cidx2]
                hop1 = HeffOperator(l_array, r_array, [mpo[cidx2]], list(ms1.shape))
                mps_t, j = yield (hop1, 1j * evolve_dt / 2, ms1)
                local_steps.append(j)
                mps[cidx2] = mps_t.reshape(ms1.shape)
                res = yield QrRequest(mps._push_cano_call(cidx2))
                mps._push_cano_place(cidx2, res)
            mps._switch_direction()
        mps.evolve_config.stat = _krylov_stats(local_steps)
        return mps

    def __str__(self):
        return f"mps bond dim:{self.bond_dims}"


def compressed_sum(mps_list: List[Mps], batchsize=5, temp_m_trunc=None) -> Mps:
    """lib.py:417-440: sum the list in groups of ``batchsize``, each partial
    sum canonicalised and compressed (a single MPS is compressed in place)."""
    assert len(mps_list) != 0
    queue = list(mps_list)
    if len(queue) == 1:
        new = queue[0].canonicalise()
        return new.compress(temp_m_trunc=temp_m_trunc)
    while len(queue) != 1:
        group, queue = queue[:batchsize], queue[batchsize:]
        s = group[0]
        for other in group[1:]:
            s = s.add(other)
        s.canonicalise()
        s.compress(temp_m_trunc=temp_m_trunc)
        queue.append(s)
    return queue[0]


def evolve_batch(mps_list: List[Mps], mpo_list, evolve_dt, normalize=True, precs=None) -> List[Mps]:
    """Mps.evolve for many independent MPS at once (static-disorder
    realisations, each with its own MPO and bond dimensions; the reference
    evolves them one by one through mps.py:644-662).  Every instance runs its
    own sweep; the local exponentials that are pending at the same time run
    in lockstep (expm_krylov_batch) and their matvecs as grouped launches
    (hop_expr.apply_grouped: one launch per contraction stage for all FP64
    problems), and the truncations pending at the same time share one
    batched eigensolver pass and one host transfer (svd_truncate_batch).
    Each result equals that instance's own evolve.

    ``precs`` (one contraction precision per instance, default the backend's)
    runs each instance's matvecs and environment updates in its own
    precision: every resumption of an instance's sweep runs under it."""
    from .hop_expr import apply_grouped
    from .krylov import expm_krylov_batch
    if isinstance(mpo_list, Mpo):
        mpo_list = [mpo_list] * len(mps_list)
    assert len(mpo_list) == len(mps_list)
    assert precs is None or len(precs) == len(mps_list)
    saved_prec = backend.prec
    gens = [m._evolve_steps(o, evolve_dt) for m, o in zip(mps_list, mpo_list)]
    out: List[Mps] = [None] * len(gens)
    pending = {}

    def resume(i, val, into):
        if precs is not None:
            backend.prec = precs[i]
        try:
            into[i] = next(gens[i]) if val is None else gens[i].send(val)
        except StopIteration as stop:
            out[i] = stop.value

    try:
        for i in range(len(gens)):
            resume(i, None, pending)
        while pending:
            nxt = {}
            # truncations of this round: one batched pass over all their QN blocks
            tidx = sorted(i for i in pending if isinstance(pending[i], TruncRequest))
            if tidx:
                res = svd_truncate_batch([pending[i].kwargs for i in tidx])
                for i, r in zip(tidx, res):
                    resume(i, r, nxt)
            # canonicalising QRs of this round: their QN blocks in shared launches
            qidx = sorted(i for i in pending if isinstance(pending[i], QrRequest))
            if qidx:
                res = qr_split_batch([pending[i].kwargs for i in qidx])
                for i, r in zip(qidx, res):
                    resume(i, r, nxt)
            # local exponentials of this round in lockstep, grouped matvecs
            idx = sorted(i for i in pending if not isinstance(pending[i], (TruncRequest, QrRequest)))
            if idx:
                reqs = [pending[i] for i in idx]
                ops = [r[0] for r in reqs]
                res = expm_krylov_batch(lambda sub, xs: apply_grouped([ops[k] for k in sub], xs),
                                        [r[1] for r in reqs], [r[2].reshape(-1) for r in reqs])
                for i, r in zip(idx, res):
                    resume(i, r, nxt)
            pending = nxt
    finally:
        backend.prec = saved_prec
    if normalize:
        for m in out:
            m.normalize("mps_and_coeff" if np.iscomplex(evolve_dt) else "mps_only")
    return out

