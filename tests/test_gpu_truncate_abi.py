"""reno_qn_svd_truncate: the sweeps' QN-blocked truncation behind one C-ABI
call, against the engine's Python-driven truncation (svd_qn.svd_truncate,
full_matrices=False, percent 0 -- the path the reference's compress and
_update_mps take when no zero-sigma completion is selected): same kept
count, singular values within 1e-12, same QN labels, and the same truncated
product left @ right."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(rows, cols, cplx, seed, decay):
    g = torch.Generator(device="cuda").manual_seed(seed)
    rng = np.random.default_rng(seed)
    ql = rng.integers(0, 3, rows).reshape(-1, 1)
    qr = 1 - rng.integers(0, 2, cols).reshape(-1, 1)     # right labels 0 / 1, qntot = 1
    X = torch.randn(rows, cols, dtype=torch.float64, device="cuda", generator=g)
    if cplx:
        X = torch.complex(X, torch.randn(rows, cols, dtype=torch.float64, device="cuda", generator=g))
    # graded columns so that the spectrum decays (and the threshold rule bites)
    X = X * torch.as_tensor(decay ** np.arange(cols), device="cuda").to(X.dtype)
    mask = torch.as_tensor((ql + qr.reshape(1, -1)) == 1, device="cuda")
    return X * mask, ql, qr


def _c_truncate(X, ql, qr, keep_left, mode, m_max, thr, sectors):
    from renormalizer_b200._native import Engine, TruncDesc, load_library
    lib = load_library()
    eng = Engine.get(0)
    rows, cols = X.shape
    qlr = np.ascontiguousarray(ql, dtype=np.int32)
    qrr = np.ascontiguousarray(qr, dtype=np.int32)
    qt = np.array([1], dtype=np.int32)
    sec = np.ascontiguousarray(np.array(sectors, dtype=np.int32).reshape(-1, 1))
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    d = TruncDesc(rows, cols, 1, 1 if X.is_complex() else 0, int(keep_left), mode, m_max, len(sectors), thr,
                  vp(qlr), vp(qrr), vp(qt), vp(sec))
    n = ctypes.c_size_t()
    assert lib.reno_qn_svd_truncate_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    ldm = min(rows, cols)
    left = torch.empty((rows, ldm), dtype=X.dtype, device="cuda")
    right = torch.empty((ldm, cols), dtype=X.dtype, device="cuda")
    sig = np.zeros(ldm)
    qn = np.zeros((ldm, 1), dtype=np.int32)
    m = ctypes.c_int32(0)
    st = lib.reno_qn_svd_truncate(eng.ctx, ctypes.byref(d), ctypes.c_void_p(X.data_ptr()),
                                  ctypes.c_void_p(left.data_ptr()), ctypes.c_void_p(right.data_ptr()), ldm,
                                  vp(sig), vp(qn), ctypes.byref(m), ctypes.c_void_p(ws.data_ptr()), n.value)
    assert st == 0, lib.reno_last_error(eng.ctx)
    torch.cuda.synchronize()
    k = m.value
    return left[:, :k], right[:k], sig[:k], qn[:k], left[:, k:], right[k:]


@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("keep_left", [True, False])
@pytest.mark.parametrize("shape,mode,m_max,thr", [((300, 220), 0, 40, 0.0), ((96, 400), 0, 30, 0.0),
                                                   ((200, 200), 1, 0, 1e-3), ((150, 260), 2, 25, 1e-4)])
def test_c_truncation_matches_python_path(shape, mode, m_max, thr, keep_left, cplx):
    from renormalizer_b200.svd_qn import qn_sectors, svd_truncate
    X, ql, qr = _case(*shape, cplx, seed=shape[0] + mode, decay=0.97)

    def rule(s):
        n_thr = int(np.sum(s / np.linalg.norm(s) > thr)) if mode in (1, 2) else len(s)
        return min(n_thr, m_max, len(s)) if mode in (0, 2) else n_thr

    ref = svd_truncate(X, ql, qr, np.array([1]), keep_left, rule, full_matrices=False,
                       kcap=m_max if mode == 0 else None)
    sectors = [q[0] for q in qn_sectors(ql)]
    left, right, sig, qn, left_rest, right_rest = _c_truncate(X, ql, qr, keep_left, mode, m_max, thr, sectors)
    assert len(sig) == ref.mdim
    np.testing.assert_allclose(sig, ref.sigma, rtol=1e-12, atol=1e-14 * ref.sigma[0])
    assert np.array_equal(qn.reshape(-1), np.asarray(ref.qn).reshape(-1))
    assert torch.allclose(left @ right, ref.left @ ref.right, atol=1e-12 * float(ref.sigma[0]))
    kept = left if keep_left else right.mH
    eye = torch.eye(kept.shape[1], dtype=kept.dtype, device="cuda")
    assert float((kept.mH @ kept - eye).abs().max()) < 1e-12
    assert float(left_rest.abs().max()) == 0.0 if left_rest.numel() else True
