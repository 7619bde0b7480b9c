"""Matrix product density operators on the sweep engine.

Drop-in for renormalizer/mps/mpdm.py (``MpDm``).  A site of the density
operator carries a physical index and an ancilla index of the same size:
(ml, d, d_anc, mr) in the reference.  Here it is held as (ml, d * d_anc, mr)
with the ancilla index fastest, and every operator acts on the physical index
only: an MPO tensor W[b, d, e, f] becomes W[b, d, e, f] delta(g, g') on the
combined index ((d, g), (e, g')).  With that the reference's ancilla forms
are the ordinary ones of the engine:

* the ancilla matvecs of hop_expr.py:80-91 ("abc, bdef, lfk, cegk -> adgl")
  and hop_expr.py:104-116 (two sites) are reno_heff_apply on (ml, d d_anc, mr);
* the ancilla environments of lib.py:206-211 / 238-243 (the ancilla bond
  traced between bra and ket) are reno_env_update on the combined index;
* the QN labels of a site are add_outer(sigmaqn, 0) (mpdm.py:69-72), flattened
  in the same order, so the QN blocks of the truncation and of the QR are
  the reference's;
* expectation values (mpdm.py:97-117: Tr(rho^dagger O rho) with the ancilla
  as a spectator) are Mps.expectation with the expanded MPO.

Extra cost against a spectator contraction: the MPO stage of a matvec runs
over d_anc^2 instead of d_anc index pairs.
"""
from __future__ import annotations

from typing import Dict

import numpy as np
import torch

from .mpo import Mpo
from .mps import Mps
from .svd_qn import add_outer


def ancilla_tensor(W: np.ndarray, d_anc: int) -> np.ndarray:
    """W[b, d, e, f] delta(g, g') on the combined index: (wl, d d_anc, d d_anc, wr)"""
    wl, d, e, wr = W.shape
    return np.einsum("bdef,gh->bdgehf", W, np.eye(d_anc)).reshape(wl, d * d_anc, e * d_anc, wr)


def ancilla_mpo(mpo: Mpo) -> Mpo:
    """The MPO acting on the physical index of a density operator (cached on
    the MPO): same bond dimensions and bond QN labels, each site tensor
    W (x) 1_ancilla."""
    anc = getattr(mpo, "_ancilla_mpo", None)
    if anc is not None:
        return anc
    anc = Mpo()
    anc.model = mpo.model
    anc.offset = mpo.offset
    anc._np = [np.ascontiguousarray(ancilla_tensor(mpo.numpy(i), mpo.numpy(i).shape[1])) for i in range(len(mpo))]
    anc._dev = [torch.from_numpy(t).to(w.device) for t, w in zip(anc._np, mpo._dev)]
    anc.qn = [q.copy() for q in mpo.qn]
    anc.qntot = None if mpo.qntot is None else np.array(mpo.qntot)
    anc.qnidx = mpo.qnidx
    mpo._ancilla_mpo = anc
    return anc


class MpDm(Mps):
    """mpdm.py:15-161: a density operator whose sites are (ml, d d_anc, mr)
    device tensors; ``site4(i)`` gives the reference's (ml, d, d_anc, mr)."""

    is_mps = False
    is_mpdm = True

    # ------------------------------------------------------------ construction
    @classmethod
    def random(cls, *args, **kwargs):
        raise ValueError("MpDm don't have to produce random state")

    @classmethod
    def ground_state(cls, model, max_entangled=False):
        raise ValueError("Use max_entangled_ex or max_entangled_gs for matrix product density matrix")

    @classmethod
    def from_mps(cls, mps: Mps) -> "MpDm":
        """mpdm.py:27-47: site[:, i, i, :] = mps site[:, i, :]"""
        new = cls()
        new.model = mps.model
        new.dtype = mps.dtype
        for ms in mps:
            ml, d, mr = ms.shape
            mo = torch.zeros((ml, d, d, mr), dtype=ms.dtype, device=ms.device)
            idx = torch.arange(d, device=ms.device)
            mo[:, idx, idx, :] = ms
            new._mp.append(mo.reshape(ml, d * d, mr).contiguous())
        new.coeff = mps.coeff
        new.optimize_config = mps.optimize_config
        new.evolve_config = mps.evolve_config
        new.qn = [q.copy() for q in mps.qn]
        new.qntot = np.array(mps.qntot)
        new.qnidx = mps.qnidx
        new.to_right = mps.to_right
        new.compress_config = mps.compress_config.copy()
        return new

    @classmethod
    def max_entangled_ex(cls, model, normalize=True) -> "MpDm":
        """mpdm.py:53-66: sum_i a^dagger_i applied to the T = infinity state"""
        mps = Mps.ground_state(model, max_entangled=True)
        ex_mps = Mpo.onsite(model, r"a^\dagger") @ mps
        if normalize:
            ex_mps.normalize("mps_and_coeff")
        return cls.from_mps(ex_mps)

    @classmethod
    def max_entangled_gs(cls, model) -> "MpDm":
        """mpdm.py:68-70"""
        return cls.from_mps(Mps.ground_state(model, max_entangled=True))

    # ------------------------------------------------------------ structure
    @property
    def pbond_list(self):
        return [p * p for p in self.model.pbond_list]

    def site4(self, i) -> torch.Tensor:
        ml, _, mr = self._mp[i].shape
        p = self.model.pbond_list[i]
        return self._mp[i].reshape(ml, p, p, mr)

    def _site_for_file(self, i) -> torch.Tensor:
        # npz files (MpDm.load / dump, the reference's format) hold 4-index sites
        return self.site4(i)

    def _to_dev(self, array) -> torch.Tensor:
        t = super()._to_dev(array)
        if t.dim() == 4:
            t = t.reshape(t.shape[0], t.shape[1] * t.shape[2], t.shape[3]).contiguous()
        return t

    def _get_sigmaqn(self, idx):
        """mpdm.py:69-72: the ancilla carries no quantum number"""
        up = np.asarray(self.model.basis[idx].sigmaqn)
        return add_outer(up, np.zeros_like(up)).reshape(-1, up.shape[-1])

    def _expansion_ex_state(self) -> "MpDm":
        """mps.py:1950-1952: the excited expander state of a density operator"""
        assert self.qntot[0] == 1 and self.model.qn_size == 1
        return MpDm.max_entangled_ex(self.model)

    def todense(self) -> np.ndarray:
        raise NotImplementedError("dense density operators are outside the sweep engine")

    # ------------------------------------------------------------ operators on the physical index
    def _evolve_steps(self, mpo: Mpo, evolve_dt):
        return super()._evolve_steps(ancilla_mpo(mpo), evolve_dt)

    def expectation(self, mpo: Mpo, self_conj: "Mps" = None):
        return super().expectation(ancilla_mpo(mpo), self_conj)

    def expectations(self, mpos, self_conj: "Mps" = None, opt: bool = True) -> np.ndarray:
        return super().expectations([ancilla_mpo(m) for m in mpos], self_conj, opt)

    def site_expectations(self, site_ops: Dict[int, np.ndarray]) -> Dict[int, float]:
        ops = {i: np.kron(np.asarray(op), np.eye(self.model.pbond_list[i])) for i, op in site_ops.items()}
        return super().site_expectations(ops)

    def calc_1site_rdm(self, idx=None):
        raise NotImplementedError("reduced density matrices of a density operator are outside the sweep engine")
