"""DMRG ground-state search on the GPU, drop-in for
renormalizer/mps/gs.py:54-576 (``optimize_mps`` / ``single_sweep`` with one
root, no omega).

Each local problem is the QN-masked effective Hamiltonian of one or two
active sites.  Blocks with fewer than 1000 elements are diagonalised
directly (gs.py:245-247, 307-407): the masked dense H_eff is assembled on the
device by applying the engine's matvec to unit vectors and handed to SciPy's
eigh in FP64 like the reference.  Larger blocks use the device Davidson
(davidson.py) with the diagonal preconditioner x / (hdiag - e + 1e-4) whose
diagonal comes from reno_heff_diag (gs.py:419-445, 532-538).  The masked
vector <-> block tensor moves (lib.py:442-457 cvec2cmat) are reno_qn
gather/scatter calls.  Truncation is the engine's QN-blocked
``Mps._update_mps`` with the procedure's ``percent``.

In split precision (backend.prec bf16x3 / tf32x3) the Davidson runs in two
stages: on the split operator until the residual reaches its rounding floor
(``SPLIT_NOISE`` times the largest diagonal entry), then on the FP64 operator
from that vector to the reference's tolerance, so energies and states carry
FP64 accuracy while most matvecs are split.  A split operator alone leaves a
Rayleigh quotient up to its error norm below the true ground state and a
residual that never reaches sqrt(tol).  The environments and the dense
small-block H_eff are FP64 for the same reason.
"""
from __future__ import annotations

import logging
from typing import List, Tuple

import numpy as np
import scipy.linalg
import torch

from ._native import Engine, h2d
from .configs import CompressConfig, CompressCriteria
from .davidson import davidson, make_diag_precond
from .hop_expr import HeffOperator
from .lib import Environ
from .mpo import Mpo
from .mps import Mps
from .svd_qn import get_qn_mask

logger = logging.getLogger(__name__)

# relative error of one split-precision H_eff matvec against FP64 (a residual
# below this times the largest diagonal entry is rounding of the split operator)
SPLIT_NOISE = {"bf16x3": 1e-4, "tf32x3": 1e-5}


class _Mask:
    """Flat indices of the QN-allowed entries of a block tensor."""

    def __init__(self, qn_mask: np.ndarray, device):
        self.shape = qn_mask.shape
        flat = np.flatnonzero(qn_mask.reshape(-1))
        self.n = len(flat)
        self.size = int(np.prod(self.shape))
        self.idx = h2d(flat, device, np.int64) if device.type == "cuda" else torch.as_tensor(flat)
        self.zero = torch.zeros(1, dtype=torch.int64, device=device)
        self.cols = torch.arange(self.n, dtype=torch.int64, device=device)
        self.eng = Engine.get(device)

    def take(self, full: torch.Tensor) -> torch.Tensor:
        """full[mask] as a 1-D vector"""
        out = torch.empty(self.n, dtype=full.dtype, device=full.device)
        self.eng.qn_gather(full.reshape(1, -1), self.zero, self.idx, out.reshape(1, -1))
        return out

    def place(self, vec: torch.Tensor, dtype) -> torch.Tensor:
        """cvec2cmat: zeros(shape) with vec at the masked entries"""
        full = torch.zeros(self.size, dtype=dtype, device=vec.device)
        self.eng.qn_scatter(vec.reshape(1, -1).to(dtype), self.zero, self.cols, self.idx, None,
                            full.reshape(1, -1), 0, 1)
        return full.reshape(self.shape)


def sign_fix(c: torch.Tensor) -> torch.Tensor:
    """gs.py:370-380 (one root): c / sign(c[argmax |c|])"""
    i = int(torch.argmax(c.abs()).item())
    v = c.reshape(-1)[i].item()
    s = np.sign(v) if not isinstance(v, complex) else v / abs(v)
    return c / s


def _dense_heff(op: HeffOperator, mask: _Mask, dtype) -> np.ndarray:
    """The masked H_eff block as a dense matrix, column by column on the device."""
    cols = []
    e = torch.zeros(mask.n, dtype=dtype, device=op.L.device)
    for j in range(mask.n):
        e.zero_()
        e[j] = 1.0
        y = op.apply(mask.place(e, dtype))
        cols.append(mask.take(y))
    return torch.stack(cols, dim=1).cpu().numpy()


def optimize_mps(mps: Mps, mpo: Mpo, omega: float = None) -> Tuple[List, Mps]:
    """gs.py:54-171: DMRG sweeps over ``mps.optimize_config.procedure``.
    Overwrites ``mps`` and returns (energies per sweep, optimised MPS)."""
    if omega is not None:
        raise NotImplementedError("the (H - omega)^2 target is outside the sweep engine")
    cfg = mps.optimize_config
    assert cfg.method in ["2site", "1site"]
    if cfg.nroots != 1:
        raise NotImplementedError("the sweep engine's DMRG optimises one root")
    if mps.is_left_canonical:
        mps.ensure_right_canonical()
        env = "R"
    else:
        mps.ensure_left_canonical()
        env = "L"
    compress_config_bk = mps.compress_config
    environ = Environ(mps, mpo, env, prec="fp64")
    macro = []
    opt_e_idx = None
    res_mps = None
    for isweep, (compress_config, percent) in enumerate(cfg.procedure):
        if isinstance(compress_config, CompressConfig):
            mps.compress_config = compress_config
        elif isinstance(compress_config, (int, np.integer)):
            mps.compress_config = CompressConfig(criteria=CompressCriteria.fixed, max_bonddim=int(compress_config))
        else:
            raise AssertionError("procedure entries are (CompressConfig | int, percent)")
        micro, res_mps = single_sweep(mps, mpo, environ, percent, opt_e_idx, res_mps)
        opt_e = min(micro)
        macro.append(opt_e[0])
        opt_e_idx = opt_e[1]
        if isweep > 0 and percent == 0:
            v1, v2 = sorted(macro)[:2]
            if np.allclose(v1, v2, rtol=cfg.e_rtol, atol=cfg.e_atol):
                logger.info("DMRG has converged!")
                break
    else:
        logger.warning("DMRG did not converge! Please increase the procedure!")
    assert res_mps is not None
    res_mps = res_mps.normalize("mps_only").ensure_left_canonical().canonicalise()
    res_mps.compress_config = compress_config_bk
    return macro, res_mps


def single_sweep(mps: Mps, mpo: Mpo, environ: Environ, percent, last_opt_e_idx, res_mps):
    """gs.py:174-304 (one root)."""
    method = mps.optimize_config.method
    micro = []
    eng = Engine.get(mps[0].device)
    for imps in mps.iter_idx_list(full=True):
        if method == "2site" and ((mps.to_right and imps == mps.site_num - 1) or
                                  ((not mps.to_right) and imps == 0)):
            break
        lmethod, rmethod = ("System", "Enviro") if mps.to_right else ("Enviro", "System")
        if method == "1site":
            lidx, cidx, ridx = imps - 1, [imps], imps + 1
        elif mps.to_right:
            lidx, cidx, ridx = imps - 1, [imps, imps + 1], imps + 2
        else:
            lidx, cidx, ridx = imps - 2, [imps - 1, imps], imps + 1
        ltensor = environ.GetLR("L", lidx, mps, mpo, itensor=None, method=lmethod)
        rtensor = environ.GetLR("R", ridx, mps, mpo, itensor=None, method=rmethod)
        qnbigl, qnbigr, qnmat = mps._get_big_qn(cidx)
        qn_mask = get_qn_mask(qnmat, mps.qntot)
        cshape = qn_mask.shape
        cmo = [mpo[i] for i in cidx]
        op = HeffOperator(ltensor, rtensor, cmo, cshape)
        op64 = op if op.prec == "fp64" else HeffOperator(ltensor, rtensor, cmo, cshape, prec="fp64")
        dtype = torch.complex128 if (mps.is_complex or op.complex_env) else torch.float64
        mask = _Mask(qn_mask, mps[0].device)
        inverse = mps.optimize_config.inverse
        if np.prod(cshape) < 1000 or mps.optimize_config.algo == "direct":
            ham = _dense_heff(op64, mask, dtype) * inverse
            w, v = scipy.linalg.eigh(ham)
            e = float(w[0])
            c = torch.as_tensor(v[:, 0]).to(mps[0].device)
            c = sign_fix(c)
        else:
            if method == "1site":
                raw = mps[cidx[0]]
            else:
                a, b = mps[cidx[0]], mps[cidx[1]]
                raw = eng.matmul(a.reshape(-1, a.shape[-1]), b.reshape(b.shape[0], -1)).reshape(cshape)
            cguess = mask.take(raw.to(dtype))
            hdiag = mask.take(op.diag()) * inverse
            precond = make_diag_precond(hdiag.contiguous())

            def aop_of(o):
                return lambda x: mask.take(o.apply(mask.place(x, dtype))) * inverse

            if op is not op64:
                # split-precision stage down to the split operator's noise
                # floor, then FP64 refinement from its vector
                floor = SPLIT_NOISE[op.prec] * float(hdiag.abs().max())
                _, cguess = davidson(aop_of(op), cguess, precond, tol=floor, tol_residual=floor, max_cycle=100)
            e, c = davidson(aop_of(op64), cguess, precond, max_cycle=100)
            c = sign_fix(c)
        micro.append((e, cidx))
        cstruct = mask.place(c, mps.dtype if not c.is_complex() else torch.complex128)
        if cidx == last_opt_e_idx:
            res_mps = mps.copy()
            res_mps._update_mps(cstruct, cidx, qnbigl, qnbigr, percent)
        mps._update_mps(cstruct, cidx, qnbigl, qnbigr, percent)
    mps._switch_direction()
    return micro, res_mps
