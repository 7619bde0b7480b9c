"""Davidson eigensolver on the GPU, drop-in for
renormalizer/lib/davidson/davidson.py:73-476 (``davidson`` / ``davidson1``,
pyscf-derived), one root.

The trial vectors, their images under the operator, the residual, the
preconditioner and the Gram-Schmidt orthogonalisation live in HBM and run in
libreno_b200 (FP64 dot products, axpy, linear combinations, diagonal
preconditioner).  The projected eigenproblem heff (at most max_space x
max_space) is solved in FP64 on the host with SciPy like the reference, and
the convergence / restart / linear-dependence decisions follow it step by
step (tol on the energy change, sqrt(tol) on the residual norm, lindep on
squared norms, restart when the space would exceed max_space).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg
import torch

from ._native import Engine, h2d


class LinearDependenceError(RuntimeError):
    pass


class _Space:
    def __init__(self, eng, n, dtype, device, rows):
        self.eng = eng
        self.n = n
        self.dtype = dtype
        self.dev = device
        self.XS = torch.empty((rows, n), dtype=dtype, device=device)
        self.AX = torch.empty((rows, n), dtype=dtype, device=device)
        self.scal = torch.zeros(2 * rows + 8, dtype=torch.float64, device=device)

    def dotc(self, x, y, slot):
        """device slot pair <- vdot(x, y)"""
        self.eng.vec_dotc(x, y, self.scal[2 * slot:2 * slot + 2])

    def read(self, k):
        s = self.scal[: 2 * k].cpu().numpy()
        return s[0::2] + 1j * s[1::2]

    def norm(self, x):
        self.eng.vec_norm(x, self.scal[-2:-1])
        return float(self.scal[-2].item())

    def scale(self, x, s):
        """x <- x * s (host scalar) in place"""
        self.scal[-3] = 1.0 / s
        self.eng.scale_inv(x, self.scal[-3:-2], x)

    def project_out(self, x, i):
        """x -= XS[i] * vdot(XS[i], x)  (no host sync)"""
        self.eng.vec_dotc(self.XS[i], x, self.scal[-6:-4])
        self.eng.axpy(x, self.XS[i], self.scal[-6:-4], -1.0)

    def combine(self, M, coeffs, k, out):
        c = np.zeros(2 * k)
        c[0::2] = np.real(coeffs[:k])
        c[1::2] = np.imag(coeffs[:k]) if np.iscomplexobj(coeffs) else 0.0
        coef = h2d(c, self.dev) if self.XS.is_cuda else torch.from_numpy(c)
        self.eng.lincomb(M, k, coef, out)
        return out


def _qr_into(space: _Space, xs, lindep, start):
    """davidson.py:453-476 _qr: Gram-Schmidt of xs into XS[start:], returns count kept."""
    nv = 0
    for x in xs:
        xi = space.XS[start + nv]
        xi.copy_(x)
        for j in range(nv):
            space.project_out(xi, start + j)
        nrm = space.norm(xi)
        if nrm * nrm > lindep:
            space.scale(xi, 1.0 / nrm)
            nv += 1
    return nv


def davidson(aop, x0, precond, tol=1e-12, max_cycle=50, max_space=12, lindep=1e-14, nroots=1, tol_residual=None,
             **kwargs):
    """Lowest eigenpair of a Hermitian operator.

    aop(x) maps a 1-D device vector to a 1-D device vector; x0 is a 1-D
    vector or a list of them; precond(dx, e, x0) returns the preconditioned
    residual (a device vector).  Converged when the energy change is below
    ``tol`` and the residual norm below ``tol_residual`` (default sqrt(tol),
    davidson.py:230-233).  Returns (e, c) like the reference with nroots=1."""
    if nroots != 1:
        raise NotImplementedError("the sweep engine's Davidson solves one root")
    if isinstance(x0, (np.ndarray, torch.Tensor)) and x0.ndim == 1:
        x0 = [x0]
    x0 = [x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x)) for x in x0]
    dev = x0[0].device
    x0 = [x.to(dev).reshape(-1) for x in x0]
    eng = Engine.get(dev)
    n = x0[0].numel()
    dtype = torch.complex128 if any(x.is_complex() for x in x0) else torch.float64
    toloose = np.sqrt(tol) if tol_residual is None else tol_residual
    rows = max_space + 2
    sp = _Space(eng, n, dtype, dev, rows)
    heff = None
    fresh_start = True
    e = 0.0
    xt_list = None
    space = 0
    x_cur = torch.empty(n, dtype=dtype, device=dev)
    ax_cur = torch.empty(n, dtype=dtype, device=dev)
    r = torch.empty(n, dtype=dtype, device=dev)
    for icyc in range(max_cycle):
        if fresh_start:
            space = 0
            src = [x.to(dtype) for x in x0]
            nt = _qr_into(sp, src, lindep, 0)
            if nt == 0:
                raise LinearDependenceError("Initial guess is empty or zero")
        else:
            nt = len(xt_list)  # one new trial vector already in XS[space]
        row0, row1 = space, space + nt
        for i in range(row0, row1):
            y = aop(sp.XS[i]).reshape(-1)
            sp.AX[i].copy_(y)
        if heff is None:
            heff = np.zeros((rows, rows), dtype=np.complex128 if dtype == torch.complex128 else np.float64)
        # _fill_heff_hermitian (davidson.py:52-70): new rows against everything
        for ip, i in enumerate(range(row0, row1)):
            for j in range(row1):
                sp.dotc(sp.XS[i], sp.AX[j], j)
            vals = sp.read(row1)
            for j in range(row0, i):
                heff[i, j] = vals[j] if heff.dtype == np.complex128 else vals[j].real
                heff[j, i] = np.conj(heff[i, j])
            heff[i, i] = vals[i].real
            for j in range(row0):
                heff[i, j] = vals[j] if heff.dtype == np.complex128 else vals[j].real
                heff[j, i] = np.conj(heff[i, j])
        space = row1
        elast = e
        w, v = scipy.linalg.eigh(heff[:space, :space])
        e = w[0]
        vv = v[:, 0]
        sp.combine(sp.XS, vv, space, x_cur)
        sp.combine(sp.AX, vv, space, ax_cur)
        de = e - elast
        # residual r = ax0 - e x0
        r.copy_(ax_cur)
        sp.scal[-8] = -e
        sp.scal[-7] = 0.0
        eng.axpy(r, x_cur, sp.scal[-8:-6], 1.0)
        dx_norm = sp.norm(r)
        if abs(de) < tol and dx_norm < toloose:
            break
        new = []
        if dx_norm ** 2 > lindep:
            t = precond(r, e, x_cur).reshape(-1).to(dtype)
            nt_ = sp.norm(t)
            sp.scale(t, 1.0 / nt_)
            new = [t]
        # orthogonalise against the space (davidson.py:390-404), in place
        kept = []
        for t in new:
            for i in range(space):
                sp.project_out(t, i)
            nrm = sp.norm(t)
            if nrm * nrm > lindep:
                sp.scale(t, 1.0 / nrm)
                kept.append(t)
        if not kept:
            break
        fresh_start = space + 1 > max_space
        if fresh_start:
            x0 = [x_cur.clone()]
            heff = None
        else:
            sp.XS[space].copy_(kept[0])
            xt_list = kept
    return float(e), x_cur.clone()


def make_diag_precond(hdiag: torch.Tensor, level_shift=1e-4):
    """gs.py:532 precond = x / (hdiag - e + 1e-4), on the device."""
    eng = Engine.get(hdiag.device)
    ebuf = torch.zeros(1, dtype=torch.float64, device=hdiag.device)

    def precond(x, e, *args):
        ebuf.fill_(float(e))
        out = torch.empty_like(x)
        eng.precond(x.reshape(-1), hdiag, ebuf, level_shift, out.reshape(-1))
        return out

    return precond
