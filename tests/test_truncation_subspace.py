"""The top-k subspace path of svd_truncate against its full Gram
eigendecomposition path on the same QN-blocked coefficient.

Both keep the bond's cap k = kcap; with a decaying spectrum (ratio of the
k-th to the (k + oversample)-th singular value well above one) the kept
singular values must agree to 1e-12 relative to sigma_1, the truncated
coefficients left @ right to 1e-10 relative to its norm, the QN labels and
selection exactly, and the kept side must be orthonormal to 1e-12.  A zero
residual tolerance forces the fallback, which must reproduce the full path
bit for bit.  CPU cases run on the test stand-in engine with a lowered size
threshold; the GPU case uses the workload's block size (2048 per QN sector,
k = 256)."""
import importlib

import numpy as np
import pytest
import torch


def _case(dev, nblk, decay, seed=3):
    """two QN sectors of nblk x nblk each: rows/cols labelled 0/1 with qntot 1"""
    g = torch.Generator(device=dev).manual_seed(seed)
    n = 2 * nblk
    ql = np.array([0] * nblk + [1] * nblk).reshape(n, 1)
    qr = np.array([1] * nblk + [0] * nblk).reshape(n, 1)
    coef = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    for b, sl in enumerate((slice(0, nblk), slice(nblk, n))):
        X = torch.complex(torch.randn(nblk, nblk, dtype=torch.float64, device=dev, generator=g),
                          torch.randn(nblk, nblk, dtype=torch.float64, device=dev, generator=g))
        U, _ = torch.linalg.qr(X)
        V, _ = torch.linalg.qr(X.mT)
        s = torch.exp(-torch.arange(nblk, dtype=torch.float64, device=dev) / decay) * (1.0 + 0.5 * b)
        coef[sl, sl] = (U * s) @ V.mH
    # rows of sector 0 pair with columns of sector 0 (labels 0 + 1 = qntot)
    return coef, ql, qr


def _run(coef, ql, qr, keep_left, kcap, percent=0.0):
    from renormalizer_b200.svd_qn import svd_truncate
    return svd_truncate(coef, ql, qr, np.array([1]), keep_left, lambda s: min(kcap, len(s)), percent=percent,
                        kcap=kcap)


def _compare(coef, ql, qr, keep_left, kcap, percent=0.0):
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    from renormalizer_b200.svd_qn import svd_truncate
    full = svd_truncate(coef, ql, qr, np.array([1]), keep_left, lambda s: min(kcap, len(s)), percent=percent)
    sub = _run(coef, ql, qr, keep_left, kcap, percent)
    assert sub.mdim == full.mdim == kcap
    np.testing.assert_array_equal(np.asarray(sub.qn), np.asarray(full.qn))
    np.testing.assert_allclose(sub.sigma, full.sigma, rtol=0, atol=1e-12 * full.sigma.max())
    a = (sub.left @ sub.right)
    b = (full.left @ full.right)
    assert float((a - b).abs().max() / b.abs().max()) < 1e-10
    kept = sub.left if keep_left else sub.right.mH
    eye = torch.eye(kcap, dtype=kept.dtype, device=kept.device)
    assert float((kept.mH @ kept - eye).abs().max()) < 1e-12
    return sub, full


@pytest.mark.parametrize("keep_left", [True, False])
def test_subspace_matches_full_path_cpu(cpu_engine, keep_left):
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    saved = (svd_qn.subspace.min_dim, svd_qn.subspace.oversample)
    svd_qn.subspace.min_dim, svd_qn.subspace.oversample = 64, 16
    c0, f0 = svd_qn.subspace.calls, svd_qn.subspace.fallbacks
    try:
        coef, ql, qr = _case("cpu", 160, 6.0)
        _compare(coef, ql, qr, keep_left, 24)
        _compare(coef, ql, qr, keep_left, 24, percent=0.4)
        assert svd_qn.subspace.calls - c0 == 4 and svd_qn.subspace.fallbacks == f0
    finally:
        svd_qn.subspace.min_dim, svd_qn.subspace.oversample = saved


def test_subspace_fallback_reproduces_full_path_cpu(cpu_engine):
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    saved = (svd_qn.subspace.min_dim, svd_qn.subspace.oversample, svd_qn.subspace.rtol)
    svd_qn.subspace.min_dim, svd_qn.subspace.oversample, svd_qn.subspace.rtol = 64, 16, 0.0
    f0 = svd_qn.subspace.fallbacks
    try:
        coef, ql, qr = _case("cpu", 160, 6.0)
        sub, full = _compare(coef, ql, qr, True, 24)
        assert svd_qn.subspace.fallbacks - f0 == 2
        assert torch.equal(sub.left, full.left) and torch.equal(sub.right, full.right)
    finally:
        svd_qn.subspace.min_dim, svd_qn.subspace.oversample, svd_qn.subspace.rtol = saved


@pytest.mark.gpu
@pytest.mark.parametrize("keep_left", [True, False])
def test_subspace_matches_full_path_gpu(keep_left):
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    saved = svd_qn.subspace.min_dim
    svd_qn.subspace.min_dim = 1024
    f0 = svd_qn.subspace.fallbacks
    try:
        coef, ql, qr = _case("cuda", 2048, 45.0)
        _compare(coef, ql, qr, keep_left, 256)
        assert svd_qn.subspace.fallbacks == f0
    finally:
        svd_qn.subspace.min_dim = saved


@pytest.mark.parametrize("keep_left", [True, False])
@pytest.mark.parametrize("shape", [(160, 160), (160, 96), (96, 160)])
def test_capped_projection_matches_full_cpu(cpu_engine, keep_left, shape):
    """with a fixed cap the full decomposition projects only the leading
    cap + 64 vectors; the selection, the kept factors and the leading sigma
    are those of the uncapped call"""
    from renormalizer_b200.svd_qn import svd_truncate
    g = torch.Generator().manual_seed(1)
    m, n = shape
    X = torch.complex(torch.randn(m, n, dtype=torch.float64, generator=g),
                      torch.randn(m, n, dtype=torch.float64, generator=g))
    U, _ = torch.linalg.qr(X)
    V, _ = torch.linalg.qr(X.mH)
    k = min(m, n)
    s = torch.exp(-torch.arange(k, dtype=torch.float64) / 9.0)
    coef = (U[:, :k] * s) @ V[:, :k].mH
    ql = np.zeros((m, 1), dtype=int)
    qr = np.zeros((n, 1), dtype=int)
    kcap = 16
    full = svd_truncate(coef, ql, qr, np.array([0]), keep_left, lambda sg: min(kcap, len(sg)))
    capped = svd_truncate(coef, ql, qr, np.array([0]), keep_left, lambda sg: min(kcap, len(sg)), kcap=kcap)
    assert capped.mdim == full.mdim == kcap
    np.testing.assert_allclose(capped.sigma, full.sigma, rtol=1e-12)
    assert torch.allclose(capped.left @ capped.right, full.left @ full.right, atol=1e-12)


@pytest.mark.parametrize("keep_left", [True, False])
@pytest.mark.parametrize("shape", [(160, 160), (160, 96), (96, 160)])
def test_capped_projection_nearly_product_cpu(cpu_engine, keep_left, shape):
    """a nearly product block (sigma = 1, then 1e-10 and below, as in a
    bond-expanded product state in FP64): the Gram eigenvalues past the
    first are rounding noise (~1e-16, sqrt ~1e-8, above the true sigma), so
    the unprojected tail must never outrank the projected head -- the
    selection stays within the projected vectors, the kept side is
    orthonormal and left @ right reproduces the block to 1e-9"""
    from renormalizer_b200.svd_qn import svd_truncate
    g = torch.Generator().manual_seed(4)
    m, n = shape
    X = torch.complex(torch.randn(m, n, dtype=torch.float64, generator=g),
                      torch.randn(m, n, dtype=torch.float64, generator=g))
    U, _ = torch.linalg.qr(X)
    V, _ = torch.linalg.qr(X.mH)
    k = min(m, n)
    s = torch.cat([torch.ones(1, dtype=torch.float64),
                   1e-10 * torch.exp(-torch.arange(k - 1, dtype=torch.float64) / 4.0)])
    coef = (U[:, :k] * s) @ V[:, :k].mH
    ql = np.zeros((m, 1), dtype=int)
    qr = np.zeros((n, 1), dtype=int)
    kcap = 4  # projects 68 of the 95 or 159 tiny directions: the rest of the positive noise is tail
    capped = svd_truncate(coef, ql, qr, np.array([0]), keep_left, lambda sg: min(kcap, len(sg)), kcap=kcap)
    assert capped.mdim == kcap
    assert abs(capped.sigma[0] - 1.0) < 1e-12 and np.all(capped.sigma[1:] < 1e-9)
    kept = capped.left if keep_left else capped.right.mH
    eye = torch.eye(kcap, dtype=kept.dtype)
    assert float((kept.mH @ kept - eye).abs().max()) < 1e-12
    assert float((capped.left @ capped.right - coef).abs().max()) < 1e-9


def test_device_eigensolver_fallback_host_logic(cpu_engine, monkeypatch):
    """svd_truncate's handling of the device eigensolver's acceptance triple:
    a stand-in returns only the leading kt eigenpairs with a check that passes
    for one block and fails for the other; the failing block must be redone by
    the full decomposition and the result must equal the all-full path"""
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    heev = importlib.import_module("renormalizer_b200.heev")
    coef, ql, qr = _case("cpu", 160, 12.0)
    kcap = 24
    full = svd_qn.svd_truncate(coef, ql, qr, np.array([1]), True, lambda s: min(kcap, len(s)), kcap=kcap)
    calls = []

    def fake_heev_top_batched(eng, Gs, kts):
        out = []
        for G, kt in zip(Gs, kts):
            w, V = torch.linalg.eigh(G)
            w, V = torch.flip(w, dims=[0]), torch.flip(V, dims=[1])
            calls.append(kt)
            bad = 1.0 if len(calls) == 1 else 0.0
            out.append((w[:kt], V[:, :kt], torch.tensor([0.0, bad, 0.0], dtype=torch.float64)))
        return out

    monkeypatch.setattr(svd_qn, "_device_eig_ok", lambda G: True)
    monkeypatch.setattr(heev, "heev_top_batched", fake_heev_top_batched)
    f0 = heev.heev_opts.fallbacks
    got = svd_qn.svd_truncate(coef, ql, qr, np.array([1]), True, lambda s: min(kcap, len(s)), kcap=kcap)
    assert len(calls) == 2 and heev.heev_opts.fallbacks == f0 + 1
    assert got.mdim == full.mdim == kcap
    np.testing.assert_array_equal(np.asarray(got.qn), np.asarray(full.qn))
    np.testing.assert_allclose(got.sigma, full.sigma, rtol=1e-12)
    assert torch.allclose(got.left @ got.right, full.left @ full.right, atol=1e-12)


@pytest.mark.parametrize("percent", [0, 0.1, 0.3])
def test_select_basis_indices_matches_oracle(percent):
    """the vectorised basis selection returns exactly the reference rule's
    indices (oracle select_basis, lib.py:253-298), ties included"""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    import reno_oracle
    from renormalizer_b200.svd_qn import select_basis_indices
    rng = np.random.default_rng(6)
    for trial in range(40):
        n = int(rng.integers(1, 300))
        nq = int(rng.integers(1, 5))
        sig = np.round(rng.random(n), 2) * (rng.random(n) > 0.2)   # many ties and zeros
        qns = [(int(q),) for q in rng.integers(0, nq, n)]
        M = int(rng.integers(1, n + 20))
        got = select_basis_indices(sig, qns, M, percent)
        vset = np.eye(n)
        ms, mpsdim, mpsqn, _ = reno_oracle.select_basis(vset, sig, qns, None, M, percent)
        ref = [int(np.argmax(ms[:, j])) for j in range(mpsdim)]
        assert got == ref, (trial, n, M)
