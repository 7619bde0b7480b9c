"""Numpy restatement of Renormalizer's MPS sweep hot path (the oracle).

TEST INFRASTRUCTURE ONLY -- imported by tests/, by __graft_entry__.smoke()
and by bench.py's CPU-baseline arm; never by the product package.

Each function cites the reference file:line it restates (paths inside the
Renormalizer project).  Contractions use plain numpy (tensordot/einsum); the
linear algebra uses SciPy LAPACK exactly where the reference does.  The
oracle is pinned against fixtures generated by the reference itself
(tests/golden/make_golden.py -> tests/golden/*.npz).
"""
from __future__ import annotations

import copy as _copy
from typing import List, Optional

import numpy as np
import scipy.linalg
from scipy.linalg import eigh_tridiagonal

EPS = np.finfo(float).eps


# --------------------------------------------------------------------------
# hop_expr.py:57-103 -- effective Hamiltonian matvec, single layer
# --------------------------------------------------------------------------
def hop(L, Ws, R, psi):
    """y = H_eff psi for len(Ws) in {0,1,2} (hop_expr.py:57-67, 68-79, 92-103)."""
    if len(Ws) == 0:
        # "abc, lbk, ck -> al"
        t = np.tensordot(L, psi, axes=([2], [0]))            # a b k
        return np.tensordot(t, R, axes=([1, 2], [1, 2]))     # a l
    if len(Ws) == 1:
        # "abc, bdef, lfk, cek -> adl"
        W = Ws[0]
        t = np.tensordot(L, psi, axes=([2], [0]))            # a b e k
        t = np.tensordot(t, W, axes=([1, 2], [0, 2]))        # a k d f
        return np.tensordot(t, R, axes=([3, 1], [1, 2]))     # a d l
    # "abc, bdef, fghj, ljk, cehk -> adgl"
    W1, W2 = Ws
    t = np.tensordot(L, psi, axes=([2], [0]))                # a b e h k
    t = np.tensordot(t, W1, axes=([1, 2], [0, 2]))           # a h k d f
    t = np.tensordot(t, W2, axes=([4, 1], [0, 2]))           # a k d g j
    return np.tensordot(t, R, axes=([4, 1], [1, 2]))         # a d g l


# --------------------------------------------------------------------------
# lib.py:169-250 -- contract_one_site (3-leg MPS sites)
# --------------------------------------------------------------------------
def contract_one_site(environ, ms, mo, domain, ms_conj=None):
    assert domain in ["L", "R"]
    if ms_conj is None:
        ms_conj = ms.conj()
    if domain == "L":
        assert environ.shape[0] == ms_conj.shape[0]
        assert environ.shape[1] == mo.shape[0]
        assert environ.shape[2] == ms.shape[0]
        # "abc, adf -> bcdf" ; "bcdf, bdeg -> cfeg" ; "cfeg, ceh -> fgh"
        t = np.tensordot(environ, ms_conj, axes=([0], [0]))  # b c d f
        t = np.tensordot(t, mo, axes=([0, 2], [0, 1]))       # c f e g
        return np.tensordot(t, ms, axes=([0, 2], [0, 1]))    # f g h
    assert environ.shape[0] == ms_conj.shape[-1]
    assert environ.shape[1] == mo.shape[-1]
    assert environ.shape[2] == ms.shape[-1]
    # "fda, abc -> fdbc" ; "fdbc, gdeb -> fcge" ; "fcge, hec -> fgh"
    t = np.tensordot(ms_conj, environ, axes=([2], [0]))      # f d b c
    t = np.tensordot(t, mo, axes=([1, 2], [1, 3]))           # f c g e
    return np.tensordot(t, ms, axes=([1, 3], [2, 1]))        # f g h


# --------------------------------------------------------------------------
# lib/krylov/krylov.py:15-84 -- Lanczos approximation of expm(dt*A) v
# --------------------------------------------------------------------------
def _expm_krylov(alpha, beta, V, v_norm, dt):
    try:
        w_hess, u_hess = eigh_tridiagonal(alpha, beta)
    except np.linalg.LinAlgError:
        h = np.diag(alpha) + np.diag(beta, k=-1) + np.diag(beta, k=1)
        w_hess, u_hess = np.linalg.eigh(h)
    return V @ (u_hess @ (v_norm * np.exp(dt * w_hess) * u_hess[0]))


def expm_krylov(Afunc, dt, vstart, block_size=50):
    """Returns (vector, number of matvecs), krylov.py:27-84."""
    if not np.iscomplex(dt):
        dt = dt.real
    vstart = np.asarray(vstart)
    nrmv = float(np.linalg.norm(vstart))
    assert nrmv > 0
    vstart = vstart / nrmv
    alpha = np.zeros(block_size)
    beta = np.zeros(block_size - 1)
    V = np.empty((block_size, len(vstart)), dtype=vstart.dtype)
    V[0] = vstart
    res = None
    for j in range(len(vstart)):
        w = Afunc(V[j])
        alpha[j] = np.vdot(w, V[j]).real
        if j == len(vstart) - 1:
            return _expm_krylov(alpha[:j + 1], beta[:j], V[:j + 1, :].T, nrmv, dt), j + 1
        if len(V) == j + 1:
            V, old_V = np.empty((len(V) + block_size, len(vstart)), dtype=vstart.dtype), V
            V[:len(old_V)] = old_V
            alpha = np.concatenate([alpha, np.zeros(block_size)])
            beta = np.concatenate([beta, np.zeros(block_size)])
        w -= alpha[j] * V[j] + (beta[j - 1] * V[j - 1] if j > 0 else 0)
        beta[j] = np.linalg.norm(w)
        if beta[j] < 100 * len(vstart) * EPS:
            return _expm_krylov(alpha[:j + 1], beta[:j], V[:j + 1, :].T, nrmv, dt), j + 1
        if 3 < j and j % 2 == 0:
            new_res = _expm_krylov(alpha[:j + 1], beta[:j], V[:j + 1].T, nrmv, dt)
            if res is not None and np.allclose(res, new_res):
                return new_res, j + 1
            res = new_res
        V[j + 1] = w / beta[j]


# --------------------------------------------------------------------------
# svd_qn.py -- quantum-number blocked SVD / QR
# --------------------------------------------------------------------------
def add_outer(a, b):
    """svd_qn.py:305-313 (np.add.outer keeping the last, QN-component axis)."""
    assert a.shape[-1] == b.shape[-1]
    out = np.array([np.add.outer(a[..., i], b[..., i]) for i in range(a.shape[-1])])
    return out.transpose(list(range(1, out.ndim)) + [0])


def get_qn_mask(qnmat, qntot):
    """svd_qn.py:316-317"""
    return np.all(qnmat == np.array(qntot), axis=-1)


def add_orthonormal_basis(u, rng=np.random):
    """svd_qn.py:52-63 (random completion drawn from the global numpy RNG)."""
    m, n = u.shape
    assert 2 * n < m
    a = rng.rand(m, n)
    a = a - u @ (u.T.conj() @ a)
    q, _ = scipy.linalg.qr(a, mode="economic")
    return np.concatenate([u, q], axis=1)


def optimized_svd(a, full_matrices, opt_full_matrices):
    """svd_qn.py:12-49"""
    m, n = a.shape
    if not full_matrices:
        opt_full_matrices = False
    opt = opt_full_matrices and not (1 / 3 < m / n < 3)
    try:
        U, S, Vt = scipy.linalg.svd(a, full_matrices=full_matrices and not opt, lapack_driver="gesdd")
    except scipy.linalg.LinAlgError:
        U, S, Vt = scipy.linalg.svd(a, full_matrices=full_matrices and not opt, lapack_driver="gesvd")
    if not opt:
        return U, S, Vt
    if m < n:
        Vt = add_orthonormal_basis(Vt.T).T
    elif n < m:
        U = add_orthonormal_basis(U)
    return U, S, Vt


def blockrecover(indices, U, dim):
    """svd_qn.py:89-96"""
    out = np.zeros([dim, U.shape[1]], dtype=U.dtype)
    out[indices, :] = U
    return out


def svd_qn(coef_array, qnbigl, qnbigr, qntot, QR=False, system=None, full_matrices=True,
           opt_full_matrices=True):
    """svd_qn.py:99-240.  Returns (u, su, qnl, v, sv, qnr) or (u, qnl, v, qnr) for QR."""
    SVD = not QR
    coef_matrix = coef_array.reshape((int(np.prod(qnbigl.shape[:-1])), int(np.prod(qnbigr.shape[:-1]))))
    qntot = np.asarray(qntot)
    qn_size = len(qntot)
    localqnl = qnbigl.reshape(-1, qn_size)
    localqnr = qnbigr.reshape(-1, qn_size)
    u_list, u_list0, v_list, v_list0 = [], [], [], []
    s_list, su0, sv0 = [], [], []
    qnl_list, qnl_list0, qnr_list, qnr_list0 = [], [], [], []
    for nl in set([tuple(t) for t in localqnl]):
        nr = qntot - nl
        rset = np.where(get_qn_mask(localqnr, nr))[0]
        if len(rset) == 0:
            continue
        lset = np.where(get_qn_mask(localqnl, nl))[0]
        block = coef_matrix.ravel().take((lset * coef_matrix.shape[1]).reshape(-1, 1) + rset)
        dim = min(block.shape)
        if SVD:
            bu, bs, bvt = optimized_svd(block, full_matrices=full_matrices, opt_full_matrices=opt_full_matrices)
            s_list.append(bs)
        else:
            mode = "full" if full_matrices else "economic"
            if system == "R":
                bu, bvt = scipy.linalg.rq(block, mode=mode)
            elif system == "L":
                bu, bvt = scipy.linalg.qr(block, mode=mode)
            else:
                raise AssertionError("system must be L or R for QR")
        # blockappend (svd_qn.py:66-86)
        u_list.append(blockrecover(lset, bu[:, :dim], coef_matrix.shape[0]))
        qnl_list += [nl] * dim
        v = bvt.T
        v_list.append(blockrecover(rset, v[:, :dim], coef_matrix.shape[1]))
        qnr_list += [nr] * dim
        if full_matrices:
            u_list0.append(blockrecover(lset, bu[:, dim:], coef_matrix.shape[0]))
            qnl_list0 += [nl] * (bu.shape[1] - dim)
            su0.append(np.zeros(bu.shape[1] - dim))
            v_list0.append(blockrecover(rset, v[:, dim:], coef_matrix.shape[1]))
            qnr_list0 += [nr] * (v.shape[1] - dim)
            sv0.append(np.zeros(v.shape[1] - dim))
    if len(u_list) + len(u_list0) == 0 or len(v_list) + len(v_list0) == 0:
        raise ValueError("Invalid quantum number")
    u = np.concatenate(u_list + u_list0, axis=1)
    v = np.concatenate(v_list + v_list0, axis=1)
    new_qnl = qnl_list + qnl_list0
    new_qnr = qnr_list + qnr_list0
    if QR:
        return u, new_qnl, v, new_qnr
    su = np.concatenate(s_list + su0)
    sv = np.concatenate(s_list + sv0)
    if not full_matrices:
        order = np.argsort(su)[::-1]
        u, v = u[:, order], v[:, order]
        su = sv = su[order]
        new_qnl = np.array(new_qnl)[order].tolist()
        new_qnr = np.array(new_qnr)[order].tolist()
    return u, su, new_qnl, v, sv, new_qnr


# --------------------------------------------------------------------------
# lib.py:253-322 select_basis ; utils/configs.py:196-219 compute_m_trunc
# --------------------------------------------------------------------------
def select_basis(vset, sset, qnlist, compset, Mmax, percent=0):
    qnlist = [tuple(qn) for qn in qnlist]
    qnset = set(qnlist)
    basdic = {i: [qnlist[i], sset[i]] for i in range(len(qnlist)) if qnlist[i] in qnset}

    def block_select(basdic, qn, n):
        block = {i: basdic[i] for i in basdic if basdic[i][0] == qn}
        srt = sorted(block.items(), key=lambda x: x[1][1], reverse=True)
        sidx = [i[0] for i in srt[0:min(n, len(srt))]]
        for idx in sidx:
            del basdic[idx]
        return sidx

    nbasis = min(len(basdic), Mmax)
    sidx = []
    if percent != 0:
        nbas_block = int(nbasis * percent / len(qnset))
        for iqn in qnset:
            sidx += block_select(basdic, iqn, nbas_block)
    nbasis = nbasis - len(sidx)
    srt = sorted(basdic.items(), key=lambda x: x[1][1], reverse=True)
    sidx += [i[0] for i in srt[0:nbasis]]
    assert len(sidx) == len(set(sidx))
    mpsdim = len(sidx)
    ms = np.zeros((vset.shape[0], mpsdim), dtype=vset.dtype)
    compmps = None if compset is None else np.zeros((compset.shape[0], mpsdim), dtype=compset.dtype)
    mpsqn = []
    for idim in range(mpsdim):
        ms[:, idim] = vset[:, sidx[idim]]
        if compset is not None and sidx[idim] < compset.shape[1]:
            compmps[:, idim] = compset[:, sidx[idim]] * sset[sidx[idim]]
        mpsqn.append(qnlist[sidx[idim]])
    return ms, mpsdim, np.array(mpsqn), compmps


class Compress:
    """The subset of CompressConfig (utils/configs.py:41-264) the sweep path reads."""

    def __init__(self, criteria="fixed", threshold=1e-3, max_bonddim=32):
        self.criteria = criteria
        self.threshold = threshold
        self.bond_dim_max_value = max_bonddim
        self.max_dims = None

    def set_bonddim(self, length):  # configs.py:192-194
        if self.max_dims is None:
            self.max_dims = np.full(length, self.bond_dim_max_value, dtype=int)

    def compute_m_trunc(self, sigma, idx, left):  # configs.py:196-219
        def thr():
            normed = sigma / scipy.linalg.norm(sigma)
            return int(np.sum(normed > self.threshold))

        def fixed():
            return min(self.max_dims[idx + 1 if left else idx], len(sigma))

        if self.criteria == "threshold":
            return thr()
        if self.criteria == "fixed":
            return fixed()
        return min(thr(), fixed())

    @property
    def bonddim_should_set(self):
        return self.criteria != "threshold" and self.max_dims is None


# --------------------------------------------------------------------------
# mp.py / mps.py -- the MPS container and its sweep-time methods
# --------------------------------------------------------------------------
class OMps:
    """Minimal MatrixProduct (mp.py:34-1227) for the sweep path."""

    def __init__(self, sites, qn, qnidx, qntot, to_right, sigmaqn, compress=None, coeff=1.0):
        self.ms = [np.asarray(s) for s in sites]
        self.qn = [np.asarray(q, dtype=int).reshape(len(q), -1) for q in qn]
        self.qnidx = int(qnidx)
        self.qntot = np.asarray(qntot, dtype=int).reshape(-1)
        self.to_right = bool(to_right)
        self.sigmaqn = [np.asarray(s, dtype=int).reshape(len(s), -1) for s in sigmaqn]
        self.compress = compress or Compress()
        self.coeff = coeff

    def __len__(self):
        return len(self.ms)

    def copy(self):
        return _copy.deepcopy(self)

    def to_complex(self):  # mp.py:996-1007
        new = self.copy()
        new.ms = [m.astype(np.complex128) for m in new.ms]
        new.coeff = complex(new.coeff)
        return new

    def iter_idx_list(self, full, stop_idx=None):  # mp.py:230-243
        n = len(self)
        if self.to_right:
            last = stop_idx if stop_idx is not None else (n if full else n - 1)
            return range(self.qnidx, last)
        last = stop_idx if stop_idx is not None else (-1 if full else 0)
        return range(self.qnidx, last, -1)

    def move_qnidx(self, dstidx):  # mp.py:159-172
        n = len(self)
        for idx in range(self.qnidx + 1, n + 1):
            self.qn[idx] = self.qntot - self.qn[idx]
        for idx in range(n, dstidx, -1):
            self.qn[idx] = self.qntot - self.qn[idx]
        self.qnidx = dstidx

    def _switch_direction(self):  # mp.py:297-306
        if self.to_right:
            self.qnidx = len(self) - 1
            self.to_right = False
        else:
            self.qnidx = 0
            self.to_right = True

    def _get_big_qn(self, cidx):  # mp.py:308-352
        if len(cidx) == 2:
            cidx = sorted(cidx)
            assert cidx[0] + 1 == cidx[1]
        assert self.qnidx in cidx
        sig = [self.sigmaqn[i] for i in cidx]
        qnl = np.array(self.qn[cidx[0]])
        qnr = np.array(self.qn[cidx[-1] + 1])
        if len(cidx) == 1:
            if self.to_right:
                qnbigl, qnbigr = add_outer(qnl, sig[0]), qnr
            else:
                qnbigl, qnbigr = qnl, add_outer(sig[0], qnr)
        else:
            qnbigl, qnbigr = add_outer(qnl, sig[0]), add_outer(sig[1], qnr)
        return qnbigl, qnbigr, add_outer(qnbigl, qnbigr)

    def _update_ms(self, idx, u, vt, qnlset=None, qnrset=None):  # mp.py:245-295 (sigma=None, MPS)
        m_trunc = u.shape[1]
        u = u[:, :m_trunc]
        vt = vt[:m_trunc, :]
        pd = self.ms[idx].shape[1:-1]
        pprod = int(np.prod(pd))
        if self.to_right:
            self.ms[idx + 1] = np.tensordot(vt, self.ms[idx + 1], axes=1)
            ret = u.reshape([u.shape[0] // pprod] + list(pd) + [m_trunc])
            if qnlset is not None:
                self.qn[idx + 1] = np.array(qnlset[:m_trunc])
                self.qnidx = idx + 1
        else:
            self.ms[idx - 1] = np.tensordot(self.ms[idx - 1], u, axes=1)
            ret = vt.reshape([m_trunc] + list(pd) + [vt.shape[1] // pprod])
            if qnrset is not None:
                self.qn[idx] = np.array(qnrset[:m_trunc])
                self.qnidx = idx - 1
        self.ms[idx] = ret

    def _push_cano(self, idx):  # mp.py:890-908
        qnbigl, qnbigr, _ = self._get_big_qn([idx])
        system = "L" if self.to_right else "R"
        u, qnlset, v, qnrset = svd_qn(self.ms[idx], qnbigl, qnbigr, self.qntot, QR=True, system=system,
                                      full_matrices=False)
        self._update_ms(idx, u, v.T, qnlset=qnlset, qnrset=qnrset)

    def canonicalise(self):  # mp.py:910-922
        idx = None
        for idx in self.iter_idx_list(full=False):
            self._push_cano(idx)
        if (not self.to_right and idx == 1) or (self.to_right and idx == len(self) - 2):
            self._switch_direction()
        return self

    def _update_mps(self, cstruct, cidx, qnbigl, qnbigr, percent=0):  # mp.py:651-888 (one root, no OFS)
        system = "L" if self.to_right else "R"
        if self.compress.bonddim_should_set:
            self.compress.set_bonddim(len(self) + 1)
        Uset, SUset, qnlnew, Vset, SVset, qnrnew = svd_qn(cstruct, qnbigl, qnbigr, self.qntot, system=system)
        if self.to_right:
            m_trunc = self.compress.compute_m_trunc(SUset, cidx[0], self.to_right)
            ms, msdim, msqn, compms = select_basis(Uset, SUset, qnlnew, Vset, m_trunc, percent=percent)
            ms = ms.reshape(list(qnbigl.shape[:-1]) + [msdim])
            compms = np.moveaxis(compms.reshape(list(qnbigr.shape[:-1]) + [msdim]), -1, 0)
        else:
            m_trunc = self.compress.compute_m_trunc(SVset, cidx[-1], self.to_right)
            ms, msdim, msqn, compms = select_basis(Vset, SVset, qnrnew, Uset, m_trunc, percent=percent)
            ms = np.moveaxis(ms.reshape(list(qnbigr.shape[:-1]) + [msdim]), -1, 0)
            compms = compms.reshape(list(qnbigl.shape[:-1]) + [msdim])
        n = len(self)
        if len(cidx) == 1:
            c0 = cidx[0]
            self.ms[c0] = ms
            if self.to_right:
                if c0 != n - 1:
                    self.ms[c0 + 1] = np.tensordot(compms, self.ms[c0 + 1], axes=1)
                    self.qn[c0 + 1] = msqn
                    self.qnidx = c0 + 1
                else:
                    self.ms[c0] = np.tensordot(self.ms[c0], compms, axes=1)
                    self.qnidx = n - 1
            else:
                if c0 != 0:
                    self.ms[c0 - 1] = np.tensordot(self.ms[c0 - 1], compms, axes=1)
                    self.qn[c0] = msqn
                    self.qnidx = c0 - 1
                else:
                    self.ms[c0] = np.tensordot(compms, self.ms[c0], axes=1)
                    self.qnidx = 0
        else:
            if self.to_right:
                self.ms[cidx[0]], self.ms[cidx[1]] = ms, compms
                self.qnidx = cidx[1]
            else:
                self.ms[cidx[1]], self.ms[cidx[0]] = ms, compms
                self.qnidx = cidx[0]
            self.qn[cidx[1]] = msqn


def dot(bra_conj_sites, ket_sites):
    """mp.py:933-956 : <bra|ket> with bra given already conjugated."""
    e0 = np.eye(1, 1)
    for mt1, mt2 in zip(bra_conj_sites, ket_sites):
        e0 = np.tensordot(e0, mt2, 1)
        e0 = np.tensordot(e0, mt1, ([0, 1], [0, 1])).T
    return complex(e0[0, 0])


def mp_norm(mps: OMps):
    """mp.py:354-372"""
    res = dot([m.conj() for m in mps.ms], mps.ms).real
    if res < 0:
        assert abs(res) < 1e-8
        res = 0
    return float(np.sqrt(res))


def normalize(mps: OMps, kind="mps_only"):
    """mps.py:2025-2059"""
    n = mp_norm(mps)
    if kind == "mps_and_coeff":
        mps.coeff = mps.coeff / np.linalg.norm(mps.coeff)
    elif kind == "mps_norm_to_coeff":
        mps.coeff = mps.coeff * n
    mps.ms[mps.qnidx] = mps.ms[mps.qnidx] * (1.0 / n)
    return mps


class OEnviron:
    """lib.py:12-118 Environ, one MPO, sentinel ones((1,1,1))."""

    def __init__(self, mps: OMps, mpo, domain=None, mps_conj=None):
        self.disk = {}
        self.sentinel = np.ones((1, 1, 1))
        conj = [m.conj() for m in mps.ms] if mps_conj is None else mps_conj
        for dom in (["L", "R"] if domain is None else [domain]):
            self.disk[("L", -1)] = self.sentinel
            self.disk[("R", len(mps))] = self.sentinel
            if dom == "L":
                rng = range(0, len(mps) - 1)
            else:
                rng = range(len(mps) - 1, 0, -1)
            t = self.sentinel
            for idx in rng:
                t = contract_one_site(t, mps.ms[idx], mpo[idx], dom, ms_conj=conj[idx])
                self.disk[(dom, idx)] = t

    def read(self, domain, idx):
        return self.disk[(domain, idx)]

    def write(self, domain, idx, t):
        self.disk[(domain, idx)] = t

    def GetLR(self, domain, siteidx, mps, mpo, itensor=None, method="System"):  # lib.py:62-112
        if siteidx not in range(len(mps)):
            return self.sentinel
        if method == "Enviro":
            return self.read(domain, siteidx)
        assert method == "System"
        if itensor is None:
            itensor = self.read(domain, siteidx + (-1 if domain == "L" else 1))
        itensor = contract_one_site(itensor, mps.ms[siteidx], mpo[siteidx], domain)
        self.write(domain, siteidx, itensor)
        return itensor


# --------------------------------------------------------------------------
# mps.py:1267-1404 -- one-site TDVP projector splitting
# --------------------------------------------------------------------------
def evolve_tdvp_ps(mps_in: OMps, mpo, evolve_dt, normalize_after=True, stats=None):
    mps = mps_in.copy() if np.iscomplex(evolve_dt) else mps_in.to_complex()
    environ = OEnviron(mps, mpo)
    for _ in range(2):
        for imps in mps.iter_idx_list(full=True):
            system = "L" if mps.to_right else "R"
            l_array = environ.read("L", imps - 1)
            r_array = environ.read("R", imps + 1)
            shape = list(mps.ms[imps].shape)
            W = mpo[imps]
            mps_t, j = expm_krylov(lambda y: hop(l_array, [W], r_array, y.reshape(shape)).ravel(),
                                   -1j * evolve_dt / 2, mps.ms[imps].ravel())
            if stats is not None:
                stats.append(j)
            mps_t = mps_t.reshape(shape)
            qnbigl, qnbigr, _ = mps._get_big_qn([imps])
            u, qnlset, v, qnrset = svd_qn(mps_t, qnbigl, qnbigr, mps.qntot, QR=True, system=system,
                                          full_matrices=False)
            vt = v.T
            if not mps.to_right and imps != 0:
                mps.ms[imps] = vt.reshape([-1] + shape[1:])
                mps.qn[imps] = np.array(qnrset)
                mps.qnidx = imps - 1
                r_array = environ.GetLR("R", imps, mps, mpo, itensor=r_array, method="System")
                shape_u = u.shape
                mps_t, j = expm_krylov(lambda y: hop(l_array, [], r_array, y.reshape(shape_u)).ravel(),
                                       1j * evolve_dt / 2, u.ravel())
                if stats is not None:
                    stats.append(j)
                mps.ms[imps - 1] = np.tensordot(mps.ms[imps - 1], mps_t.reshape(shape_u), axes=(-1, 0))
            elif mps.to_right and imps != len(mps) - 1:
                mps.ms[imps] = u.reshape(shape[:-1] + [-1])
                mps.qn[imps + 1] = np.array(qnlset)
                mps.qnidx = imps + 1
                l_array = environ.GetLR("L", imps, mps, mpo, itensor=l_array, method="System")
                shape_svt = vt.shape
                mps_t, j = expm_krylov(lambda y: hop(l_array, [], r_array, y.reshape(shape_svt)).ravel(),
                                       1j * evolve_dt / 2, vt.ravel())
                if stats is not None:
                    stats.append(j)
                mps.ms[imps + 1] = np.tensordot(mps_t.reshape(shape_svt), mps.ms[imps + 1], axes=(1, 0))
            else:
                mps.ms[imps] = mps_t
        mps._switch_direction()
    if normalize_after:
        normalize(mps, "mps_and_coeff" if np.iscomplex(evolve_dt) else "mps_only")
    return mps


# --------------------------------------------------------------------------
# mps.py:1406-1517 -- two-site TDVP projector splitting
# --------------------------------------------------------------------------
def evolve_tdvp_ps2(mps_in: OMps, mpo, evolve_dt, normalize_after=True, stats=None):
    mps = mps_in.copy() if np.iscomplex(evolve_dt) else mps_in.to_complex()
    environ = OEnviron(mps, mpo)
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
            ms2 = np.tensordot(mps.ms[cidx0], mps.ms[cidx1], axes=1)
            W1, W2 = mpo[cidx0], mpo[cidx1]
            shp = ms2.shape
            mps_t, j = expm_krylov(lambda y: hop(l_array, [W1, W2], r_array, y.reshape(shp)).ravel(),
                                   -1j * evolve_dt / 2, ms2.ravel())
            if stats is not None:
                stats.append(j)
            mps_t = mps_t.reshape(shp)
            qnbigl, qnbigr, _ = mps._get_big_qn([cidx0, cidx1])
            mps._update_mps(mps_t, [cidx0, cidx1], qnbigl, qnbigr)
            if imps == last_idx:
                continue
            if mps.to_right:
                l_array = environ.GetLR("L", lidx + 1, mps, mpo, itensor=l_array, method="System")
            else:
                r_array = environ.GetLR("R", ridx - 1, mps, mpo, itensor=r_array, method="System")
            ms1 = mps.ms[cidx2]
            W = mpo[cidx2]
            shp1 = ms1.shape
            mps_t, j = expm_krylov(lambda y: hop(l_array, [W], r_array, y.reshape(shp1)).ravel(),
                                   1j * evolve_dt / 2, ms1.ravel())
            if stats is not None:
                stats.append(j)
            mps.ms[cidx2] = mps_t.reshape(shp1)
            mps._push_cano(cidx2)
        mps._switch_direction()
    if normalize_after:
        normalize(mps, "mps_and_coeff" if np.iscomplex(evolve_dt) else "mps_only")
    return mps


# --------------------------------------------------------------------------
# mps.py:471-609 -- expectation values
# --------------------------------------------------------------------------
def expectation(mps: OMps, mpo):
    """<psi|O|psi> through an R-environment sweep (mps.py:471-525)."""
    conj = [m.conj() for m in mps.ms]
    t = np.ones((1, 1, 1))
    for idx in range(len(mps) - 1, -1, -1):
        t = contract_one_site(t, mps.ms[idx], mpo[idx], "R", ms_conj=conj[idx])
    val = complex(t.ravel()[0])
    return val.real if np.isclose(val.imag, 0) else val


def site_expectations(mps: OMps, site_ops: dict):
    """<psi| O_i |psi> for one-site operators {site: matrix (d_out, d_in)}, the
    quantity Mps.e_occupations returns (mps.py:595-609) for O_i = a^dagger a."""
    n = len(mps)
    conj = [m.conj() for m in mps.ms]
    eye = [np.eye(m.shape[1]).reshape(1, m.shape[1], m.shape[1], 1) for m in mps.ms]
    left = [np.ones((1, 1, 1))]
    for i in range(n - 1):
        left.append(contract_one_site(left[-1], mps.ms[i], eye[i], "L", ms_conj=conj[i]))
    right = [None] * (n + 1)
    right[n] = np.ones((1, 1, 1))
    for i in range(n - 1, 0, -1):
        right[i] = contract_one_site(right[i + 1], mps.ms[i], eye[i], "R", ms_conj=conj[i])
    out = {}
    for i, op in site_ops.items():
        W = np.asarray(op).reshape(1, op.shape[0], op.shape[1], 1)
        t = contract_one_site(left[i], mps.ms[i], W, "L", ms_conj=conj[i])
        out[i] = complex(np.tensordot(t, right[i + 1], axes=3)).real
    return out


def calc_1site_rdm(mps: OMps):
    """mps.py:1547-1598: rho_i[p, q] = sum L[a, a'] conj(ms[a, p, b]) R[b, b'] ms[a', q, b']
    with the overlap (identity-MPO) environments on both sides."""
    n = len(mps)
    conj = [m.conj() for m in mps.ms]
    eye = [np.eye(m.shape[1]).reshape(1, m.shape[1], m.shape[1], 1) for m in mps.ms]
    left = [np.ones((1, 1, 1))]
    for i in range(n - 1):
        left.append(contract_one_site(left[-1], mps.ms[i], eye[i], "L", ms_conj=conj[i]))
    right = [None] * (n + 1)
    right[n] = np.ones((1, 1, 1))
    for i in range(n - 1, 0, -1):
        right[i] = contract_one_site(right[i + 1], mps.ms[i], eye[i], "R", ms_conj=conj[i])
    rdm = {}
    for i, ms in enumerate(mps.ms):
        lt = left[i].reshape(left[i].shape[0], left[i].shape[-1])
        rt = right[i + 1].reshape(right[i + 1].shape[0], right[i + 1].shape[-1])
        t = np.tensordot(lt, ms.conj(), ([0], [0]))
        t = np.tensordot(t, rt, ([-1], [0]))
        rdm[i] = np.tensordot(t, ms, ([0, -1], [0, -1]))
    return rdm


def calc_bond_singular_values(mps: OMps):
    """mps.py:1759-1772 with compress(temp_m_trunc=inf, ret_s=True) (mp.py:437-511):
    right-canonicalise a copy, then an untruncated SVD sweep to the right with
    sigma moved into the next site; the per-bond sigma lists (globally sorted,
    svd_qn.py:231-239) padded with zeros to a rectangle."""
    m = mps.copy()
    m.move_qnidx(len(m) - 1)
    m.to_right = False
    m.canonicalise()
    s_list = []
    for idx in m.iter_idx_list(full=False):
        qnbigl, qnbigr, _ = m._get_big_qn([idx])
        u, sigma, qnlset, v, _, qnrset = svd_qn(m.ms[idx], qnbigl, qnbigr, m.qntot, system="L", full_matrices=False)
        s_list.append(np.asarray(sigma))
        vt = np.einsum("i,ij->ij", sigma, v.T)
        m._update_ms(idx, u, vt, qnlset=qnlset, qnrset=qnrset)
    m._switch_direction()
    width = max(len(x) for x in s_list)
    return np.array([np.pad(x, (0, width - len(x))) for x in s_list])


def calc_vn_entropy(p):
    """utils/utils.py:41-48"""
    p = np.asarray(p, dtype=float)
    p = p / p.sum()
    p = p[p > 0]
    return float(-(p * np.log(p)).sum())


def calc_bond_entropy(mps: OMps, s_array=None):
    """mps.py:1774-1793"""
    if s_array is None:
        s_array = calc_bond_singular_values(mps)
    return np.array([calc_vn_entropy(sig ** 2) for sig in s_array])


def expectations(mps: OMps, mpos):
    """mps.py:527-575 with opt=False: one R-environment sweep per operator."""
    res = np.array([expectation(mps, m) for m in mpos], dtype=complex)
    return res.real if np.allclose(res.imag, 0) else res


# --------------------------------------------------------------------------
# lib/davidson/davidson.py:154-476 -- Davidson, one root (pyscf-derived)
# --------------------------------------------------------------------------
class LinearDependenceError(RuntimeError):
    pass


def _qr(xs, lindep=1e-14):
    nvec = len(xs)
    qs = np.empty((nvec, xs[0].size), dtype=xs[0].dtype)
    nv = 0
    for i in range(nvec):
        xi = np.array(xs[i], copy=True)
        for j in range(nv):
            xi -= qs[j] * np.dot(qs[j].conj(), xi)
        innerprod = np.dot(xi.conj(), xi).real
        if innerprod > lindep:
            qs[nv] = xi / np.sqrt(innerprod)
            nv += 1
    return qs[:nv]


def davidson(aop, x0, precond, tol=1e-12, max_cycle=100, max_space=12, lindep=1e-14):
    """davidson.py:73-151 with nroots=1 (follow_state False, in-core)."""
    toloose = np.sqrt(tol)
    x0 = [x0] if isinstance(x0, np.ndarray) and x0.ndim == 1 else list(x0)
    heff = None
    fresh_start = True
    e = 0.0
    v = None
    conv = False
    for icyc in range(max_cycle):
        if fresh_start:
            xs, ax = [], []
            space = 0
            xt = _qr(x0, lindep)
            if len(xt) == 0:
                raise LinearDependenceError("Initial guess is empty or zero")
            x0 = None
        elif len(xt) > 1:
            xt = _qr(xt, lindep)[:40]
        axt = [aop(x) for x in xt]
        for k in range(len(xt)):
            xs.append(xt[k])
            ax.append(axt[k])
        rnow = len(xt)
        head, space = space, space + rnow
        dtype = np.result_type(axt[0], xt[0])
        if heff is None:
            heff = np.empty((max_space + 1, max_space + 1), dtype=dtype)
        else:
            heff = np.asarray(heff, dtype=dtype)
        elast = e
        # _fill_heff_hermitian (davidson.py:52-70)
        row1 = len(ax)
        row0 = row1 - rnow
        for ip, i in enumerate(range(row0, row1)):
            for jp, j in enumerate(range(row0, i)):
                heff[i, j] = np.dot(xt[ip].conj(), axt[jp])
                heff[j, i] = heff[i, j].conj()
            heff[i, i] = np.dot(xt[ip].conj(), axt[ip]).real
        for i in range(row0):
            axi = ax[i]
            for jp, j in enumerate(range(row0, row1)):
                heff[j, i] = np.dot(xt[jp].conj(), axi)
                heff[i, j] = heff[j, i].conj()
        w, v = scipy.linalg.eigh(heff[:space, :space])
        e = w[0]
        vv = v[:, 0]
        # _gen_x0 (davidson.py:478-485): start from the last vector, add the rest in reverse
        x0 = vv[space - 1] * xs[space - 1]
        for i in reversed(range(space - 1)):
            x0 = x0 + vv[i] * xs[i]
        ax0 = vv[space - 1] * ax[space - 1]
        for i in reversed(range(space - 1)):
            ax0 = ax0 + vv[i] * ax[i]
        de = e - elast
        r = ax0 - e * x0
        dx_norm = np.sqrt(np.dot(r.conj(), r).real)
        conv = abs(de) < tol and dx_norm < toloose
        if conv:
            break
        xt = []
        if dx_norm ** 2 > lindep:
            t = precond(r, e, x0)
            t *= 1 / np.sqrt(np.dot(t.conj(), t).real)
            xt = [t]
        for i in range(space):
            for xi in xt:
                xi -= xs[i] * np.dot(xs[i].conj(), xi)
        nxt = []
        for xi in xt:
            norm = np.sqrt(np.dot(xi.conj(), xi).real)
            if norm ** 2 > lindep:
                nxt.append(xi * (1 / norm))
        xt = nxt
        if len(xt) == 0:
            conv = dx_norm < toloose
            break
        fresh_start = space + 1 > max_space
        if fresh_start:
            x0 = [x0]
    return e, x0


def sign_fix(c):
    """gs.py:370-380 (one root)."""
    return c / np.sign(c[np.abs(c).argmax()])


def cvec2cmat(c, qn_mask):
    """lib.py:442-457 (one root)."""
    cstruct = np.zeros(qn_mask.shape, dtype=c.dtype)
    np.place(cstruct, qn_mask, c)
    return cstruct


def hdiag_of(L, Ws, R):
    """gs.py:419-445 diagonal of H_eff (1 or 2 sites)."""
    tl = np.einsum("aba->ba", L)
    tr = np.einsum("aba->ba", R)
    if len(Ws) == 1:
        t0 = np.einsum("abbc->abc", Ws[0])
        return np.einsum("ba,bcg,gf->acf", tl, t0, tr)
    t0 = np.einsum("abbc->abc", Ws[0])
    t1 = np.einsum("abbc->abc", Ws[1])
    return np.einsum("ba,bce,edg,gf->acdf", tl, t0, t1, tr)


def optimize_mps(mps: OMps, mpo, procedure, method="2site", e_rtol=1e-6, e_atol=1e-8):
    """gs.py:54-171 + single_sweep gs.py:174-304 (one root, no omega).

    procedure: list of (max_bonddim, percent).  Returns (energies, mps)."""
    assert method in ("1site", "2site")
    mps.qn = [q.copy() for q in mps.qn]
    # gs.py:97-102: a left-canonical start is right-canonicalised first and
    # the environment is built from the right; any other start the other way
    # (ensure_*_canonical, mp.py:206-228, always re-canonicalising)
    if mps.qnidx == len(mps) - 1:
        mps.move_qnidx(len(mps) - 1)
        mps.to_right = False
        mps.canonicalise()
        env_dom = "R"
    else:
        mps.move_qnidx(0)
        mps.to_right = True
        mps.canonicalise()
        env_dom = "L"
    environ = OEnviron(mps, mpo, env_dom)
    energies = []
    opt_e_idx = None
    res_mps = None
    for isweep, (mmax, percent) in enumerate(procedure):
        mps.compress = Compress("fixed", max_bonddim=mmax)
        micro = []
        for imps in mps.iter_idx_list(full=True):
            if method == "2site" and ((mps.to_right and imps == len(mps) - 1) or (not mps.to_right and imps == 0)):
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
            if np.prod(cshape) < 1000:
                # eigh_direct (gs.py:307-407)
                if len(cmo) == 1:
                    ham = np.einsum("abc,bdef,lfk->adlcek", ltensor, cmo[0], rtensor)
                    ham = ham[:, :, :, qn_mask][qn_mask, :]
                else:
                    ham = np.einsum("abc,bdef,fghj,ljk->adglcehk", ltensor, cmo[0], cmo[1], rtensor)
                    ham = ham[:, :, :, :, qn_mask][qn_mask, :]
                w, v = scipy.linalg.eigh(ham)
                e, c = w[0], sign_fix(v[:, 0])
            else:
                raw = mps.ms[cidx[0]] if len(cidx) == 1 else np.tensordot(mps.ms[cidx[0]], mps.ms[cidx[1]], axes=1)
                cguess = [raw[qn_mask]]
                hdiag = hdiag_of(ltensor, cmo, rtensor)[qn_mask]

                def aop(x):
                    return hop(ltensor, cmo, rtensor, cvec2cmat(x, qn_mask))[qn_mask]

                e, c = davidson(aop, cguess, lambda x, e0, *a: x / (hdiag - e0 + 1e-4), max_cycle=100)
                c = sign_fix(c)
            micro.append((e, cidx))
            cstruct = cvec2cmat(c, qn_mask)
            if cidx == opt_e_idx:
                res_mps = mps.copy()
                res_mps._update_mps(cstruct, cidx, qnbigl, qnbigr, percent)
            mps._update_mps(cstruct, cidx, qnbigl, qnbigr, percent)
        mps._switch_direction()
        opt = min(micro, key=lambda t: t[0])
        energies.append(opt[0])
        opt_e_idx = opt[1]
        if isweep > 0 and percent == 0:
            v1, v2 = sorted(energies)[:2]
            if np.allclose(v1, v2, rtol=e_rtol, atol=e_atol):
                break
    return energies, res_mps
