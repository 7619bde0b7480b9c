"""Lanczos exponential on the GPU, drop-in for
renormalizer/lib/krylov/krylov.py:27-84 (``expm_krylov``).

The Krylov basis V, the matvecs and every vector operation (vdot, norm,
three-term recurrence, V @ coeffs, allclose) stay in HBM and run in
libreno_b200; alpha/beta are produced on the device in FP64.  The small
tridiagonal eigenproblem is solved in FP64 on the host with the same SciPy
routine the reference uses (krylov.py:15-24).

Host synchronisation happens only where the reference makes a decision that
needs the scalars: at its convergence checks (every even j > 3) and when the
Krylov space is exhausted.  The breakdown test beta_j < 100 n eps, which the
reference applies every iteration, is evaluated at those points for every
iteration since the last one; because the Krylov vectors up to the breakdown
index do not depend on what came after it, the returned vector and count are
the ones the reference returns.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.linalg import eigh_tridiagonal

from ._native import Engine, h2d
from .hop_expr import as_device

EPS = np.finfo(float).eps


class KrylovTolerance:
    """The convergence test of the Lanczos exponential: successive
    approximations agree within ``rtol`` / ``atol`` (numpy allclose), checked
    at every even j > 3.  The defaults are numpy allclose's, which the reference
    calls without arguments (krylov.py:78);
    tighter values make the exponential converge past the reference's stopping
    point (every parity claim is made with the defaults).  RENO_KRYLOV_TOL =
    "rtol,atol" overrides them."""

    def __init__(self, rtol=1e-5, atol=1e-8):
        import os
        env = os.environ.get("RENO_KRYLOV_TOL")
        if env:
            rtol, atol = (float(x) for x in env.split(","))
        self.rtol, self.atol = rtol, atol


tolerance = KrylovTolerance()


def _tridiag_coeffs(alpha, beta, v_norm, dt):
    """krylov.py:15-24 : u_hess @ (v_norm * exp(dt * w_hess) * u_hess[0])."""
    try:
        w_hess, u_hess = eigh_tridiagonal(alpha, beta)
    except np.linalg.LinAlgError:
        h = np.diag(alpha) + np.diag(beta, k=-1) + np.diag(beta, k=1)
        w_hess, u_hess = np.linalg.eigh(h)
    return u_hess @ (v_norm * np.exp(dt * w_hess) * u_hess[0])


class _Krylov:
    def __init__(self, eng: Engine, n: int, dtype, device, block_size):
        self.eng = eng
        self.n = n
        self.dtype = dtype
        self.V = torch.empty((block_size, n), dtype=dtype, device=device)
        # scal[0] = ||vstart||, scal[2] = allclose flag ; ab = (alpha_0, beta_0, alpha_1, ...)
        self.scal = torch.zeros(4, dtype=torch.float64, device=device)
        self.ab = torch.zeros(2 * block_size + 2, dtype=torch.float64, device=device)

    def grow(self, block_size):
        V = torch.empty((self.V.shape[0] + block_size, self.n), dtype=self.dtype, device=self.V.device)
        V[: self.V.shape[0]] = self.V
        self.V = V
        ab = torch.zeros(2 * self.V.shape[0] + 2, dtype=torch.float64, device=self.V.device)
        ab[: self.ab.numel()] = self.ab
        self.ab = ab

    def combine(self, k, coeffs, out):
        c = np.zeros(2 * k)
        c[0::2] = np.real(coeffs)
        c[1::2] = np.imag(coeffs) if np.iscomplexobj(coeffs) else 0.0
        coef = h2d(c, self.V.device) if self.V.is_cuda else torch.from_numpy(c)
        self.eng.lincomb(self.V, k, coef, out)
        return out


def _expm_krylov_steps(dt, vstart, block_size=50):
    """The Lanczos exponential as a generator: it yields each Krylov vector
    whose image under the operator it needs and receives that image, and
    returns (vector, number of matvecs).  ``expm_krylov`` serves it one
    operator; ``expm_krylov_batch`` serves many in lockstep, one grouped
    matvec per round, with every instance's arithmetic and decisions exactly
    those of its own expm_krylov."""
    if not np.iscomplex(dt):
        dt = dt.real
    v = as_device(vstart).reshape(-1)
    n = v.numel()
    eng = Engine.get(v.device)
    dt_cplx = np.iscomplexobj(dt) and np.iscomplex(dt)
    # the result is complex when exp(dt*w) is complex (krylov.py:24)
    work_dtype = torch.complex128 if (v.is_complex() or dt_cplx) else torch.float64
    if v.dtype != work_dtype:
        v = v.to(work_dtype)
    K = _Krylov(eng, n, work_dtype, v.device, block_size)
    eng.vec_norm(v, K.scal)                  # nrmv = ||vstart||
    eng.scale_inv(v, K.scal, K.V[0])         # V[0] = vstart / nrmv
    out_a = torch.empty(n, dtype=work_dtype, device=v.device)
    out_b = torch.empty(n, dtype=work_dtype, device=v.device)
    state = {"nrmv": None, "checked": 0, "res": None}

    def host_scalars(j):
        ab = K.ab[: 2 * j + 2].cpu().numpy()
        if state["nrmv"] is None:
            nrmv = float(K.scal[0].item())
            assert nrmv > 0
            if not np.isfinite(nrmv):
                raise FloatingPointError("expm_krylov: start vector is not finite")
            state["nrmv"] = nrmv
        return ab[0::2], ab[1::2]

    def coeffs_for(alpha, beta, k):
        # entries past a breakdown may be garbage; only the used ones must be finite
        a, b = alpha[: k + 1], beta[:k]
        if not (np.all(np.isfinite(a)) and np.all(np.isfinite(b))):
            raise FloatingPointError("expm_krylov: Lanczos scalars are not finite")
        return _tridiag_coeffs(a, b, state["nrmv"], dt)

    def breakdown_before(j, beta):
        # first unchecked i < j with beta_i below the reference's threshold
        for i in range(state["checked"], j):
            if beta[i] < 100 * n * EPS:
                return i
        state["checked"] = j
        return None

    for j in range(n):
        w = (yield K.V[j]).reshape(-1)
        if w.dtype != work_dtype:
            w = w.to(work_dtype)
        if not w.is_contiguous():
            w = w.contiguous()
        eng.krylov_alpha(w, K.V[j], K.ab, j)
        if j == n - 1:
            alpha, beta = host_scalars(j)
            i = breakdown_before(j, beta)
            k = j if i is None else i
            return K.combine(k + 1, coeffs_for(alpha, beta, k), out_a), k + 1
        if K.V.shape[0] == j + 1:
            K.grow(block_size)
        vprev = K.V[j - 1] if j > 0 else None
        eng.krylov_orth(w, K.V[j], vprev, K.ab, j)       # w -= ...; beta_j = ||w||
        eng.scale_inv(w, K.ab[2 * j + 1:], K.V[j + 1])   # V[j+1] = w / beta_j
        if 3 < j and j % 2 == 0:
            alpha, beta = host_scalars(j)
            i = breakdown_before(j + 1, beta)
            if i is not None:
                return K.combine(i + 1, coeffs_for(alpha, beta, i), out_a), i + 1
            coeffs = coeffs_for(alpha, beta, j)
            res_prev = state["res"]
            new_res = K.combine(j + 1, coeffs, out_b if res_prev is out_a else out_a)
            if res_prev is not None:
                eng.allclose(res_prev, new_res, tolerance.rtol, tolerance.atol, K.scal[2:3])
                if float(K.scal[2].item()) == 1.0:
                    return new_res, j + 1
            state["res"] = new_res


def expm_krylov(Afunc, dt, vstart, block_size=50):
    """Krylov approximation of expm(dt*A) @ vstart for Hermitian A.

    Returns (vector, number of matvecs) like the reference.  ``Afunc`` maps a
    1-D device vector to a device vector (e.g. a HeffOperator)."""
    gen = _expm_krylov_steps(dt, vstart, block_size)
    try:
        x = next(gen)
        while True:
            x = gen.send(Afunc(x))
    except StopIteration as stop:
        return stop.value


def expm_krylov_batch(group_apply, dts, vstarts, block_size=50):
    """expm_krylov for many independent problems in lockstep (static-disorder
    realisations, not in the reference).  ``group_apply(idx, xs)`` maps the
    Krylov vectors xs of the problems idx (a list) to their images, normally
    in one grouped launch (hop_expr.apply_grouped); ``dts`` is one step for
    all or one per problem.  Returns [(vector, number of matvecs)] in input
    order, each identical to that problem's own expm_krylov.

    All problems start together, so at every round they sit at the same
    Krylov index j: each vector operation of a round is one grouped launch
    (reno_vec_grouped, every problem's result bitwise its single call's), and
    the host reads the scalars of all problems that reach a check point
    (every even j > 3, or the end of their Krylov space) in one transfer."""
    m = len(vstarts)
    if np.ndim(dts) == 0:
        dts = [dts] * m
    if m == 0:
        return []
    return _LockstepKrylov(dts, vstarts, block_size).run(group_apply)


class _LockstepKrylov:
    """The state of expm_krylov (_expm_krylov_steps) for m problems, with the
    alpha/beta arrays of all problems in one device array AB (row p) and the
    start norms / allclose flags in SC (columns 0 / 2)."""

    def __init__(self, dts, vstarts, block_size):
        from ._native import VOP_NORM, VOP_SCALE_INV
        self.block_size = block_size
        self.dts, self.vs, self.n, self.dtype = [], [], [], []
        for dt, v0 in zip(dts, vstarts):
            if not np.iscomplex(dt):
                dt = dt.real
            v = as_device(v0).reshape(-1)
            dt_cplx = np.iscomplexobj(dt) and np.iscomplex(dt)
            work_dtype = torch.complex128 if (v.is_complex() or dt_cplx) else torch.float64
            if v.dtype != work_dtype:
                v = v.to(work_dtype)
            self.dts.append(dt)
            self.vs.append(v)
            self.n.append(v.numel())
            self.dtype.append(work_dtype)
        dev = self.vs[0].device
        assert all(v.device == dev for v in self.vs), "lockstep problems share one device"
        self.device = dev
        self.eng = Engine.get(dev)
        m = len(self.vs)
        self.V = [torch.empty((block_size, n), dtype=dt, device=dev) for n, dt in zip(self.n, self.dtype)]
        self.AB = torch.zeros((m, 2 * block_size + 2), dtype=torch.float64, device=dev)
        self.SC = torch.zeros((m, 4), dtype=torch.float64, device=dev)
        self.out = [(torch.empty(n, dtype=dt, device=dev), torch.empty(n, dtype=dt, device=dev))
                    for n, dt in zip(self.n, self.dtype)]
        self.nrmv = [None] * m
        self.checked = [0] * m
        self.res = [None] * m
        # nrmv = ||vstart|| ; V[0] = vstart / nrmv
        self._op(VOP_NORM, [(p, 0, self.vs[p], None, None, self.SC[p], None) for p in range(m)])
        self._op(VOP_SCALE_INV, [(p, 0, self.vs[p], None, self.V[p][0], None, self.SC[p]) for p in range(m)])

    def _code(self, p):
        from ._native import RENO_C128, RENO_F64
        return RENO_C128 if self.dtype[p] == torch.complex128 else RENO_F64

    def _op(self, op, rows, rtol=0.0, atol=0.0):
        """rows: (p, j, x, y, out, scalars, s) per problem"""
        if rows:
            self.eng.vec_grouped(op, [(self.n[p], self._code(p), j, x, y, out, sc, s, self.n[p])
                                      for p, j, x, y, out, sc, s in rows], rtol, atol)

    def _grow(self, p):
        bs = self.block_size
        V = torch.empty((self.V[p].shape[0] + bs, self.n[p]), dtype=self.dtype[p], device=self.device)
        V[: self.V[p].shape[0]] = self.V[p]
        self.V[p] = V
        need = 2 * V.shape[0] + 2
        if self.AB.shape[1] < need:
            AB = torch.zeros((self.AB.shape[0], need), dtype=torch.float64, device=self.device)
            AB[:, : self.AB.shape[1]] = self.AB
            self.AB = AB

    def _coeffs(self, p, alpha, beta, k):
        a, b = alpha[: k + 1], beta[:k]
        if not (np.all(np.isfinite(a)) and np.all(np.isfinite(b))):
            raise FloatingPointError("expm_krylov: Lanczos scalars are not finite")
        return _tridiag_coeffs(a, b, self.nrmv[p], self.dts[p])

    def _breakdown_before(self, p, j, beta):
        for i in range(self.checked[p], j):
            if beta[i] < 100 * self.n[p] * EPS:
                return i
        self.checked[p] = j
        return None

    def _combine(self, jobs):
        """jobs: (p, k, coeffs, out) -> out = V[p][:k] @ coeffs, one grouped launch"""
        from ._native import VOP_LINCOMB
        if not jobs:
            return
        cs = []
        for _, k, coeffs, _ in jobs:
            c = np.zeros(2 * k)
            c[0::2] = np.real(coeffs)
            c[1::2] = np.imag(coeffs) if np.iscomplexobj(coeffs) else 0.0
            cs.append(c)
        flat = np.concatenate(cs)
        coef = h2d(flat, self.device) if self.device.type == "cuda" else torch.from_numpy(flat)
        rows, off = [], 0
        for (p, k, _, out), c in zip(jobs, cs):
            rows.append((p, k, self.V[p], None, out, None, coef[off: off + c.size]))
            off += c.size
        self._op(VOP_LINCOMB, rows)

    def run(self, group_apply):
        from ._native import VOP_ALLCLOSE, VOP_ALPHA, VOP_ORTH, VOP_SCALE_INV
        m = len(self.vs)
        result = [None] * m
        active = list(range(m))
        j = 0
        while active:
            ws = group_apply(active, [self.V[p][j] for p in active])
            W = {}
            for p, w in zip(active, ws):
                w = w.reshape(-1)
                if w.dtype != self.dtype[p]:
                    w = w.to(self.dtype[p])
                if not w.is_contiguous():
                    w = w.contiguous()
                W[p] = w
            self._op(VOP_ALPHA, [(p, j, W[p], self.V[p][j], None, self.AB[p], None) for p in active])
            term = [p for p in active if j == self.n[p] - 1]
            cont = [p for p in active if j < self.n[p] - 1]
            for p in cont:
                if self.V[p].shape[0] == j + 1:
                    self._grow(p)
            self._op(VOP_ORTH, [(p, j, self.V[p][j], self.V[p][j - 1] if j > 0 else None, W[p], self.AB[p], None)
                                for p in cont])
            self._op(VOP_SCALE_INV, [(p, 0, W[p], None, self.V[p][j + 1], None, self.AB[p][2 * j + 1:])
                                     for p in cont])
            check = cont if (3 < j and j % 2 == 0) else []
            finished = set()
            if term or check:
                ab = self.AB[:, : 2 * j + 2].cpu().numpy()
                if any(self.nrmv[p] is None for p in term + check):
                    sc = self.SC[:, 0].cpu().numpy()
                    for p in term + check:
                        if self.nrmv[p] is None:
                            nrmv = float(sc[p])
                            assert nrmv > 0
                            if not np.isfinite(nrmv):
                                raise FloatingPointError("expm_krylov: start vector is not finite")
                            self.nrmv[p] = nrmv
                jobs, tests = [], []
                for p in term:
                    alpha, beta = ab[p, 0::2], ab[p, 1::2]
                    i = self._breakdown_before(p, j, beta)
                    k = j if i is None else i
                    out = self.out[p][0]
                    jobs.append((p, k + 1, self._coeffs(p, alpha, beta, k), out))
                    result[p] = (out, k + 1)
                    finished.add(p)
                for p in check:
                    alpha, beta = ab[p, 0::2], ab[p, 1::2]
                    i = self._breakdown_before(p, j + 1, beta)
                    if i is not None:
                        out = self.out[p][0]
                        jobs.append((p, i + 1, self._coeffs(p, alpha, beta, i), out))
                        result[p] = (out, i + 1)
                        finished.add(p)
                        continue
                    coeffs = self._coeffs(p, alpha, beta, j)
                    prev = self.res[p]
                    a, b = self.out[p]
                    new = b if prev is a else a
                    jobs.append((p, j + 1, coeffs, new))
                    if prev is not None:
                        tests.append((p, prev, new))
                    self.res[p] = new
                self._combine(jobs)
                if tests:
                    self._op(VOP_ALLCLOSE, [(p, 0, prev, new, None, self.SC[p][2:], None) for p, prev, new in tests],
                             tolerance.rtol, tolerance.atol)
                    flags = self.SC[:, 2].cpu().numpy()
                    for p, _, new in tests:
                        if flags[p] == 1.0:
                            result[p] = (new, j + 1)
                            finished.add(p)
            active = [p for p in cont if p not in finished]
            j += 1
        return result
