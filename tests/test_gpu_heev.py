"""The device Hermitian eigensolver of the truncation (renormalizer_b200.heev,
csrc/heev.cu) against cuSOLVER's dense eigh (torch.linalg.eigh).

On Gram matrices G = X X^H of complex and real blocks, with a generic
spectrum and with a nearly product one (one dominant singular value, a
decaying tail and an exactly rank-deficient remainder), the kt leading
eigenvalues must match eigvalsh to 1e-13 max|lambda|, the eigenvectors must
have residuals ||G k - lambda k|| below 1e-12 max|lambda| and be
orthonormal to 1e-12, the acceptance check must pass, and two calls on the
same input must agree bit for bit.  Through svd_truncate (fixed cap, blocks
above the solver's size threshold), the kept singular values must match the
cuSOLVER path to 1e-12 sigma_1, the truncated coefficient to 1e-10 of its
norm, and the QN labels exactly."""
import importlib

import numpy as np
import pytest
import torch


def _gram(n, cplx, kind, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = lambda: torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    X = torch.complex(r(), r()) if cplx else r()
    if kind == "generic":
        return X @ X.mH / n
    U, _ = torch.linalg.qr(X)
    s = torch.exp(-torch.arange(n, dtype=torch.float64, device="cuda") / (n / 16))
    s[n // 3:] *= 1e-7
    s[n // 2:] = 0.0
    s[0] = 1.0
    return (U * s ** 2) @ U.mH


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("kind", ["generic", "nearly_product"])
@pytest.mark.parametrize("n,kt", [(96, 40), (256, 128), (700, 128), (2048, 320)])
def test_heev_top_matches_eigh(n, kt, kind, cplx):
    from renormalizer_b200._native import Engine
    from renormalizer_b200.heev import accepted, heev_opts, heev_top
    G = _gram(n, cplx, kind, seed=n + (7 if cplx else 0))
    eng = Engine.get(G.device)
    w, K, chk = heev_top(eng, G, kt)
    w2, K2, chk2 = heev_top(eng, G, kt)
    torch.cuda.synchronize()
    assert accepted(chk.cpu().numpy()), chk.cpu().numpy()
    assert torch.equal(w, w2) and torch.equal(K, K2)
    ref = torch.flip(torch.linalg.eigvalsh(G), dims=[0])[:kt]
    scale = float(ref.abs().max())
    assert float((w - ref).abs().max()) <= 1e-13 * scale
    Kc = K.to(torch.complex128)
    Gc = G.to(torch.complex128)
    assert float((Gc @ Kc - Kc * w).abs().max()) <= 1e-12 * scale
    eye = torch.eye(kt, dtype=torch.complex128, device="cuda")
    assert float((Kc.mH @ Kc - eye).abs().max()) <= 1e-12
    if not cplx:
        assert float(K.imag.abs().max()) == 0.0
    assert heev_opts.tol >= 1e-12


def _two_sector(nblk, seed=5):
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = 2 * nblk
    ql = np.array([0] * nblk + [1] * nblk).reshape(n, 1)
    qr = np.array([1] * nblk + [0] * nblk).reshape(n, 1)
    coef = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    for b, sl in enumerate((slice(0, nblk), slice(nblk, n))):
        X = torch.complex(torch.randn(nblk, nblk, dtype=torch.float64, device="cuda", generator=g),
                          torch.randn(nblk, nblk, dtype=torch.float64, device="cuda", generator=g))
        U, _ = torch.linalg.qr(X)
        V, _ = torch.linalg.qr(X.mT)
        s = torch.exp(-torch.arange(nblk, dtype=torch.float64, device="cuda") / 40.0) * (1.0 + 0.3 * b)
        coef[sl, sl] = (U * s) @ V.mH
    return coef, ql, qr


@pytest.mark.gpu
@pytest.mark.parametrize("keep_left", [True, False])
def test_svd_truncate_device_eigensolver_matches_cusolver(keep_left):
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    from renormalizer_b200.heev import heev_opts
    coef, ql, qr = _two_sector(640)
    kcap = 128
    saved = heev_opts.enabled
    try:
        heev_opts.enabled = False
        ref = svd_qn.svd_truncate(coef, ql, qr, np.array([1]), keep_left, lambda s: min(kcap, len(s)), kcap=kcap)
        heev_opts.enabled = True
        c0, f0 = heev_opts.calls, heev_opts.fallbacks
        got = svd_qn.svd_truncate(coef, ql, qr, np.array([1]), keep_left, lambda s: min(kcap, len(s)), kcap=kcap)
        assert heev_opts.calls - c0 == 2 and heev_opts.fallbacks == f0
    finally:
        heev_opts.enabled = saved
    assert got.mdim == ref.mdim == kcap
    np.testing.assert_array_equal(np.asarray(got.qn), np.asarray(ref.qn))
    np.testing.assert_allclose(got.sigma, ref.sigma, rtol=0, atol=1e-12 * ref.sigma.max())
    a, b = got.left @ got.right, ref.left @ ref.right
    assert float((a - b).abs().max() / b.abs().max()) < 1e-10
    kept = got.left if keep_left else got.right.mH
    eye = torch.eye(kcap, dtype=kept.dtype, device=kept.device)
    assert float((kept.mH @ kept - eye).abs().max()) < 1e-12


@pytest.mark.gpu
def test_heev_batched_mixed_sizes_lower_triangle_reduction():
    """a batch whose largest matrix takes the lower-triangle reduction kernel
    (n >= 3072) with smaller ones sharing the launch: every matrix meets the
    single-matrix bounds, and the batch is reproducible bit for bit"""
    from renormalizer_b200._native import Engine
    from renormalizer_b200.heev import accepted, heev_top_batched
    sizes, kts = (3200, 400, 2100, 300), (320, 100, 320, 64)
    Gs = [_gram(n, True, "generic" if i % 2 == 0 else "nearly_product", seed=31 + i) for i, n in enumerate(sizes)]
    eng = Engine.get(Gs[0].device)
    res = heev_top_batched(eng, Gs, list(kts))
    res2 = heev_top_batched(eng, Gs, list(kts))
    torch.cuda.synchronize()
    for G, kt, (w, K, chk), (w2, K2, _) in zip(Gs, kts, res, res2):
        assert accepted(chk.cpu().numpy()), chk.cpu().numpy()
        assert torch.equal(w, w2) and torch.equal(K, K2)
        ref = torch.flip(torch.linalg.eigvalsh(G), dims=[0])[:kt]
        scale = float(ref.abs().max())
        assert float((w - ref).abs().max()) <= 1e-13 * scale
        assert float((G @ K - K * w).abs().max()) <= 1e-12 * scale
        eye = torch.eye(kt, dtype=torch.complex128, device="cuda")
        assert float((K.mH @ K - eye).abs().max()) <= 1e-12
