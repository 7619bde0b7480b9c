"""Batched Householder QR (reno_qr_blocks) against LAPACK through SciPy.

The per-block QR of svd_qn.py:195-204 is scipy.linalg.qr(mode="economic");
the engine's kernel follows LAPACK's conventions, so Q and R must agree with
SciPy entry by entry, signs included (not only up to a diagonal unitary), for
tall, square and wide blocks, real and complex, several blocks per call."""
import numpy as np
import pytest
import scipy.linalg as sla
import torch

pytestmark = pytest.mark.gpu


def _mat(rng, m, k, cplx):
    a = rng.standard_normal((m, k))
    if cplx:
        a = a + 1j * rng.standard_normal((m, k))
    return a


@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("shapes", [
    [(7, 3)], [(5, 5)], [(3, 8)], [(1, 1)], [(1, 6)], [(9, 1)],
    [(64, 40), (33, 57), (128, 128)],
    [(2048, 128), (2048, 128)],
    [(4096, 256)],
    [(300, 200), (17, 5), (260, 260), (5, 300)],
])
def test_qr_blocks_match_lapack(shapes, cplx):
    from renormalizer_b200._native import Engine
    eng = Engine.get(0)
    rng = np.random.default_rng(len(shapes) * 101 + sum(m * 7 + k for m, k in shapes) + cplx)
    hs = [_mat(rng, m, k, cplx) for m, k in shapes]
    ds = [torch.from_numpy(h).cuda() for h in hs]
    Qs, Rs = eng.qr_blocks(ds)
    for h, d, Q, R in zip(hs, ds, Qs, Rs):
        q_ref, r_ref = sla.qr(h, mode="economic")
        q, r = Q.cpu().numpy(), R.cpu().numpy()
        scale = max(1.0, np.abs(h).max())
        assert np.abs(q - q_ref).max() < 1e-12 * max(h.shape), (h.shape, np.abs(q - q_ref).max())
        assert np.abs(r - r_ref).max() < 1e-12 * scale * max(h.shape), (h.shape, np.abs(r - r_ref).max())
        assert np.abs(np.triu(r) - r).max() == 0.0
        # the input is left untouched
        assert torch.equal(d.cpu(), torch.from_numpy(h))


def test_qr_rank_deficient_block_is_orthonormal_and_exact():
    """A rank-deficient block (a bond-expanded state's site tensor has columns
    of weight 1e-10 and exact zeros): Q stays orthonormal and Q R = A."""
    from renormalizer_b200._native import Engine
    eng = Engine.get(0)
    rng = np.random.default_rng(3)
    u = _mat(rng, 512, 4, True)
    a = u @ _mat(rng, 4, 96, True)
    a[:, 50:60] *= 1e-10
    a[:, 70] = 0.0
    Q, R = eng.qr_blocks([torch.from_numpy(a).cuda()])
    q, r = Q[0].cpu().numpy(), R[0].cpu().numpy()
    assert np.abs(q.conj().T @ q - np.eye(q.shape[1])).max() < 1e-13
    assert np.abs(q @ r - a).max() < 1e-13 * np.abs(a).max()


def test_qr_rejects_mixed_dtypes():
    from renormalizer_b200._native import Engine
    eng = Engine.get(0)
    with pytest.raises(AssertionError):
        eng.qr_blocks([torch.zeros((4, 3), dtype=torch.float64, device="cuda"),
                       torch.zeros((4, 3), dtype=torch.complex128, device="cuda")])
