"""Singular values far below sqrt(eps) sigma_1 through svd_truncate.

The truncation diagonalises Gram matrices, whose eigenvectors for sigma below
~1e-8 sigma_1 are mixed by rounding; the cluster refinement (svd_qn.refine)
recovers those sigma.  A two-sector coefficient with a graded spectrum
(1 down to 1e-14, with near-degenerate pairs in the tail) is truncated with
every entry kept, as calc_bond_singular_values does (mps.py:1759-1772 in the
reference: numpy's SVD of each block): the sigma must match LAPACK's to 1e-12
absolute, left @ right must rebuild the coefficient, and the kept side must
be orthonormal.  Without the pass (tau = 0) the same sigma are off by more
than 1e-10, which is what the test guards against."""
import importlib

import numpy as np
import pytest
import torch


def _graded(dev, nblk, seed=11):
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = 2 * nblk
    ql = np.array([0] * nblk + [1] * nblk).reshape(n, 1)
    qr = np.array([1] * nblk + [0] * nblk).reshape(n, 1)
    coef = torch.zeros((n, n), dtype=torch.complex128)
    ref = []
    for b, sl in enumerate((slice(0, nblk), slice(nblk, n))):
        X = torch.complex(torch.randn(nblk, nblk, dtype=torch.float64, generator=g),
                          torch.randn(nblk, nblk, dtype=torch.float64, generator=g))
        U, _ = torch.linalg.qr(X)
        V, _ = torch.linalg.qr(X.mT)
        s = torch.logspace(0, -14, nblk, dtype=torch.float64) * (1.0 + 0.25 * b)
        s[nblk // 2::2] *= 1.0 + 1e-3       # near-degenerate pairs in the tail
        coef[sl, sl] = (U * s) @ V.mH
        ref.append(np.linalg.svd(coef[sl, sl].numpy(), compute_uv=False))
    return coef.to(dev), ql, qr, np.sort(np.concatenate(ref))[::-1]


def _truncate_all(coef, ql, qr, keep_left):
    from renormalizer_b200.svd_qn import svd_truncate
    return svd_truncate(coef, ql, qr, np.array([1]), keep_left, lambda s: len(s), full_matrices=False)


def _check(dev, keep_left, nblk=96):
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    coef, ql, qr, ref = _graded(dev, nblk)
    b0 = svd_qn.refine.blocks
    res = _truncate_all(coef, ql, qr, keep_left)
    assert svd_qn.refine.blocks - b0 == 2
    got = np.sort(np.asarray(res.sigma))[::-1]
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)
    rebuilt = res.left @ res.right
    assert float((rebuilt - coef).abs().max()) < 1e-13
    kept = res.left if keep_left else res.right.mH
    eye = torch.eye(kept.shape[1], dtype=kept.dtype, device=kept.device)
    assert float((kept.mH @ kept - eye).abs().max()) < 1e-12
    saved = svd_qn.refine.tau
    svd_qn.refine.tau = 0.0
    try:
        raw = np.sort(np.asarray(_truncate_all(coef, ql, qr, keep_left).sigma))[::-1]
    finally:
        svd_qn.refine.tau = saved
    assert np.abs(raw - ref).max() > 1e-10


@pytest.mark.parametrize("keep_left", [True, False])
def test_small_sigma_refined_cpu(cpu_engine, keep_left):
    _check("cpu", keep_left)


@pytest.mark.gpu
@pytest.mark.parametrize("keep_left", [True, False])
def test_small_sigma_refined_gpu(keep_left):
    _check("cuda", keep_left)
