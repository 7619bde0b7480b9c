"""Matrix product operators for the sweep engine.

The reference builds its MPO symbolically (renormalizer/mps/mpo.py:250-290
with mps/symbolic_mpo.py:22-161); that construction is one-off host work and
outside the sweep path.  This module builds the same operator with a
finite-state construction of its own: every Hamiltonian term is a product of
one-site matrices; at each bond the "open" terms are grouped by their
left part (the sequence of matrices already applied), so terms sharing a
prefix share one MPO channel, and every term's factor is applied on its
last site.  For nearest-neighbour Holstein chains this yields bond dimension
<= 5 and for the spin-boson chain 3, like the reference.  The dense
operators agree with the reference's Mpo(model) (tests/golden/mpo_cases.npz).

Site tensors use the reference layout W[w_left, d_bra, d_ket, w_right]
(hop_expr.py:70-78) and live on the GPU as float64 (complex128 when an
operator is complex); ``Mpo[i]`` returns the device tensor.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple, Union

import numpy as np
import torch

from .backend import backend
from .model import Model, Op, Quantity


def _key(mat: np.ndarray):
    m = np.ascontiguousarray(mat)
    return (m.shape, m.dtype.str, m.tobytes())


def build_mpo_tensors(model: Model, terms: Sequence[Op], offset: float = 0.0) -> List[np.ndarray]:
    nsite = model.nsite
    dims = model.pbond_list
    # normalised terms: (factor, [(site, matrix), ...] sorted by site)
    norm_terms = []
    for t in terms:
        mats = t.local_mats(model)
        items = sorted(mats.items())
        norm_terms.append((t.factor, items))
    if offset != 0.0:
        norm_terms.append((-offset, [(0, np.eye(dims[0]))]))

    # channel labels per bond: "I" (nothing applied yet), "F" (term finished),
    # or a prefix tuple ((site, key), ...) of the matrices applied so far
    chans: List[Dict] = [dict() for _ in range(nsite + 1)]

    def chan(b, label):
        c = chans[b]
        if label not in c:
            c[label] = len(c)
        return c[label]

    for b in range(nsite):
        chan(b, "I")
    for b in range(1, nsite + 1):
        chan(b, "F")
    trans = [dict() for _ in range(nsite)]  # site -> {(in_label, out_label): matrix}

    def add(site, lin, lout, mat):
        # transitions into F carry the term factors and accumulate; every other
        # transition is a shared channel step that all terms with that prefix reuse
        d = trans[site]
        k = (lin, lout)
        if lout == "F" and lin != "F":
            d[k] = d[k] + mat if k in d else np.array(mat, dtype=np.result_type(mat, np.float64))
        elif k not in d:
            d[k] = np.array(mat, dtype=np.result_type(mat, np.float64))

    mat_store = {}
    for factor, items in norm_terms:
        if not items:
            continue
        sites = [s for s, _ in items]
        smap = dict(items)
        first, last = sites[0], sites[-1]
        prefix: Tuple = ()
        lin = "I"
        for s in range(first, last + 1):
            m = smap.get(s, np.eye(dims[s]))
            k = _key(m)
            mat_store[k] = m
            if s == last:
                add(s, lin, "F", factor * m)
            else:
                prefix = prefix + ((s, k),)
                chan(s + 1, prefix)
                add(s, lin, prefix, m)
                lin = prefix
    # identity propagation of I and F channels
    for s in range(nsite):
        eye = np.eye(dims[s])
        if s < nsite - 1:
            add(s, "I", "I", eye)
        if s > 0:
            add(s, "F", "F", eye)
    # boundary: only I on the far left, only F on the far right
    chans[0] = {"I": 0}
    chans[nsite] = {"F": 0}
    # drop channels that are never reached / never leave
    Ws = []
    for s in range(nsite):
        cin, cout = chans[s], chans[s + 1]
        dt = np.float64
        for (li, lo), m in trans[s].items():
            if np.iscomplexobj(m) and np.any(np.imag(m) != 0):
                dt = np.complex128
        W = np.zeros((len(cin), dims[s], dims[s], len(cout)), dtype=dt)
        for (li, lo), m in trans[s].items():
            if li in cin and lo in cout:
                W[cin[li], :, :, cout[lo]] += (m if dt == np.complex128 else np.real(m))
        Ws.append(W)
    return Ws


def mpo_qn_labels(model: Model, tensors: Sequence[np.ndarray]):
    """Bond QN labels of an MPO in the reference's convention
    (symbolic_mpo.py:105-161): the label of a channel is the QN its operators
    add to the sites on its left, the last bond is labelled 0 and the total
    goes to qntot.  Derived from the tensors: every nonzero entry
    W[a, bra, ket, b] moves QN qn[a] + sigmaqn[bra] - sigmaqn[ket] into
    channel b.  Channels no entry reaches are labelled 0."""
    n = len(tensors)
    if model is None or n == 0:
        return [], None
    qs = model.qn_size
    qn = [np.zeros((1, qs), dtype=int)]
    for i, W in enumerate(tensors):
        sq = np.asarray(model.basis[i].sigmaqn, dtype=int).reshape(W.shape[1], -1)
        lab = np.zeros((W.shape[3], qs), dtype=int)
        seen = np.zeros(W.shape[3], dtype=bool)
        a, p, q, b = np.nonzero(W)
        for ai, pi, qi, bi in zip(a, p, q, b):
            v = qn[i][ai] + sq[pi] - sq[qi]
            if not seen[bi]:
                lab[bi] = v
                seen[bi] = True
        qn.append(lab)
    qntot = qn[-1][0].copy()
    qn[-1] = np.zeros((1, qs), dtype=int)
    return qn, qntot


class Mpo:
    """Drop-in for the parts of renormalizer.mps.Mpo the sweep path reads:
    construction from a Model (optionally with an energy offset), len(),
    indexing (device site tensors), identity / onsite constructors, bond QN
    labels (qn, qnidx, qntot) and the MPO x MPS product (``@``)."""

    def __init__(self, model: Model = None, terms: Union[Op, List[Op]] = None, offset: Quantity = Quantity(0)):
        self.model = model
        self.offset = 0.0
        self._np: List[np.ndarray] = []
        self._dev: List[torch.Tensor] = []
        self.qn: List[np.ndarray] = []
        self.qntot = None
        self.qnidx = None
        if model is None:
            return
        if not isinstance(offset, Quantity):
            raise ValueError(f"offset must be Quantity object. Got {offset} of {type(offset)}.")
        self.offset = offset.as_au()
        if terms is None:
            terms = model.ham_terms
        elif isinstance(terms, Op):
            terms = [terms]
        terms = [t for t in terms if t.factor != 0]
        if len(terms) == 0:
            raise ValueError("Terms contain nothing.")
        self.set_tensors(build_mpo_tensors(model, terms, self.offset))

    @classmethod
    def from_tensors(cls, model, tensors: Sequence[np.ndarray], offset=0.0) -> "Mpo":
        mpo = cls()
        mpo.model = model
        mpo.offset = offset
        mpo.set_tensors([np.asarray(t) for t in tensors])
        return mpo

    def set_tensors(self, tensors: List[np.ndarray]):
        self._np = [np.ascontiguousarray(t) for t in tensors]
        dev = backend.device if torch.cuda.is_available() else None
        self._dev = [torch.from_numpy(t).to(dev) if dev is not None else torch.from_numpy(t) for t in self._np]
        self.qn, self.qntot = mpo_qn_labels(self.model, self._np)
        self.qnidx = len(self._np) - 1

    def apply(self, mp, canonicalise: bool = False):
        """MPO x MPS (mpo.py:331-389): site i becomes
        einsum("apqb,cqd->acpbd") reshaped to (a c, p, b d), the bond QN
        labels add as add_outer(mpo qn, mps qn) with the MPS labels taken on
        the MPO's boundary (qnidx), and the total QN adds."""
        from .mps import Mps
        from .svd_qn import add_outer
        assert len(self) == len(mp)
        new = mp.copy()
        if self.dtype == torch.complex128 and not new.is_complex:
            new.to_complex(inplace=True)
        from ._native import Engine
        dt = new.dtype
        sites = []
        # on a density operator the MPO acts on the physical index (mpo.py:331-389 via MpDm)
        Ws = self._dev
        if getattr(mp, "is_mpdm", False):
            from .mpdm import ancilla_mpo
            Ws = ancilla_mpo(self)._dev
        for W, ms in zip(Ws, new._mp):
            a, p, q, b = W.shape
            c, q2, d = ms.shape
            assert q == q2
            eng = Engine.get(ms.device)
            # (a p b, q) x (q, c d) on the engine's GEMM, then (a, c, p, b, d)
            wm = W.to(dt).permute(0, 1, 3, 2).reshape(a * p * b, q).contiguous()
            mm = ms.to(dt).permute(1, 0, 2).reshape(q, c * d).contiguous()
            t = eng.matmul(wm, mm).reshape(a, p, b, c, d).permute(0, 3, 1, 2, 4)
            sites.append(t.reshape(a * c, p, b * d).contiguous())
        new._mp = sites
        orig = new.qnidx
        new.move_qnidx(self.qnidx)
        new.qn = [add_outer(np.asarray(qo), np.asarray(qm)).reshape(-1, qo.shape[1])
                  for qo, qm in zip(self.qn, new.qn)]
        new.qntot = new.qntot + self.qntot
        new.move_qnidx(orig)
        if canonicalise:
            new.canonicalise()
        return new

    def __matmul__(self, other):
        return self.apply(other)

    @classmethod
    def identity(cls, model: Model) -> "Mpo":
        return cls.from_tensors(model, [np.eye(p).reshape(1, p, p, 1) for p in model.pbond_list])

    @classmethod
    def onsite(cls, model: Model, opera: str, dipole=False, dof_set=None) -> "Mpo":
        if dof_set is None:
            if model.n_edofs == 0:
                raise ValueError("No electronic DoF present in the model.")
            dof_set = model.e_dofs
        ops = [Op(opera, idx, model.dipole[idx] if dipole else 1.0) for idx in dof_set]
        return cls(model, ops)

    @property
    def dtype(self):
        return torch.complex128 if any(t.dtype == np.complex128 for t in self._np) else torch.float64

    @property
    def bond_dims(self):
        return [t.shape[0] for t in self._np] + [self._np[-1].shape[-1]]

    def numpy(self, i) -> np.ndarray:
        return self._np[i]

    def __len__(self):
        return len(self._np)

    def __getitem__(self, i) -> torch.Tensor:
        return self._dev[i]

    def __iter__(self):
        return iter(self._dev)

    def todense(self) -> np.ndarray:
        t = self._np[0]
        for W in self._np[1:]:
            t = np.tensordot(t, W, axes=([-1], [0]))
        t = t[0, ..., 0]
        n = len(self._np)
        t = t.transpose([2 * i for i in range(n)] + [2 * i + 1 for i in range(n)])
        dim = int(np.prod(t.shape[:n]))
        return t.reshape(dim, dim)
