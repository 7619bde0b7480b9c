"""GPU parity of the contraction and vector kernels against the reference
fixtures and the oracle, through the C ABI.

Tolerances: FP64 path 1e-12 relative to max|y| (rounding only);
split-precision paths use the bound stated per mode in SPLIT_TOL."""
import numpy as np
import pytest
import torch

from conftest import golden_cases, load_golden
from oracle import reno_oracle as O

pytestmark = pytest.mark.gpu

HEFF = load_golden("heff_cases.npz")
ENV = load_golden("env_cases.npz")
KRY = load_golden("krylov_cases.npz")

FP64_TOL = 1e-12
# relative to max|y|: BF16 hi/lo keeps ~16 significant bits per operand,
# TF32 hi/lo ~21; the error grows with sqrt(K) under FP32 accumulation
SPLIT_TOL = {"bf16x3": 2e-4, "tf32x3": 2e-5}


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("case", golden_cases(HEFF))
def test_heff_fp64_matches_reference(case):
    from renormalizer_b200.hop_expr import HeffOperator
    n = int(HEFF[f"{case}/nsite"])
    Ws = [HEFF[f"{case}/W{i + 1}"] for i in range(n)]
    psi = HEFF[f"{case}/psi"]
    op = HeffOperator(HEFF[f"{case}/L"], HEFF[f"{case}/R"], Ws, psi.shape, prec="fp64")
    y = op(_dev(psi)).cpu().numpy()
    ref = HEFF[f"{case}/y"]
    assert y.shape == ref.shape and y.dtype == ref.dtype
    err = np.abs(y - ref).max() / np.abs(ref).max()
    assert err < FP64_TOL, err


@pytest.mark.parametrize("case", golden_cases(ENV))
def test_env_fp64_matches_reference(case):
    from renormalizer_b200.lib import contract_one_site
    bra = ENV[f"{case}/bra"] if f"{case}/bra" in ENV.files else None
    out = contract_one_site(ENV[f"{case}/E"], ENV[f"{case}/ms"], ENV[f"{case}/W"], str(ENV[f"{case}/domain"]),
                            ms_conj=bra, prec="fp64").cpu().numpy()
    ref = ENV[f"{case}/out"]
    assert out.shape == ref.shape
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err < FP64_TOL, err


@pytest.mark.parametrize("k", range(int(KRY["count"])))
def test_krylov_matches_reference(k):
    from renormalizer_b200.krylov import expm_krylov
    A = KRY[f"k{k}/A"]
    dt = KRY[f"k{k}/dt"][()]
    Ad = _dev(A)
    res, n = expm_krylov(lambda x: Ad.to(x.dtype) @ x, dt, KRY[f"k{k}/v"].copy())
    assert n == int(KRY[f"k{k}/n"])
    np.testing.assert_allclose(res.cpu().numpy(), KRY[f"k{k}/res"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 3, 1), (7, 2, 5), (64, 10, 64), (130, 3, 67)])
@pytest.mark.parametrize("cplx", [True, False])
def test_heff_1site_shapes_vs_oracle(shape, cplx):
    """ragged and minimal shapes (M in {1,2,5,...}, odd d), tile-edge sizes"""
    from renormalizer_b200.hop_expr import HeffOperator
    rng = np.random.default_rng(7)
    ml, d, mr = shape
    wl, wr = 3, 4
    mk = lambda s: rng.standard_normal(s) + (1j * rng.standard_normal(s) if cplx else 0)
    L, R, psi = mk((ml, wl, ml)), mk((mr, wr, mr)), mk((ml, d, mr))
    W = rng.standard_normal((wl, d, d, wr))
    ref = O.hop(L, [W], R, psi)
    y = HeffOperator(L, R, [W], psi.shape, prec="fp64")(_dev(psi)).cpu().numpy()
    assert np.abs(y - ref).max() <= FP64_TOL * max(np.abs(ref).max(), 1e-300)


def test_heff_2site_c2_block_vs_oracle():
    """a 2-site block with the Holstein config's local dims (d1=2, d2=16, w=5)"""
    from renormalizer_b200.hop_expr import HeffOperator
    rng = np.random.default_rng(11)
    ml, mr, d1, d2, w = 40, 36, 2, 16, 5
    mk = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    L, R, psi = mk((ml, w, ml)), mk((mr, w, mr)), mk((ml, d1, d2, mr))
    W1, W2 = rng.standard_normal((w, d1, d1, w)), rng.standard_normal((w, d2, d2, w))
    ref = O.hop(L, [W1, W2], R, psi)
    y = HeffOperator(L, R, [W1, W2], psi.shape, prec="fp64")(_dev(psi)).cpu().numpy()
    assert np.abs(y - ref).max() / np.abs(ref).max() < FP64_TOL


def test_heff_diag_vs_oracle():
    from renormalizer_b200.hop_expr import HeffOperator
    rng = np.random.default_rng(3)
    L, R = rng.standard_normal((6, 3, 6)), rng.standard_normal((5, 2, 5))
    W1, W2 = rng.standard_normal((3, 4, 4, 3)), rng.standard_normal((3, 2, 2, 2))
    op = HeffOperator(L, R, [W1, W2], (6, 4, 2, 5), prec="fp64")
    np.testing.assert_allclose(op.diag().cpu().numpy(), O.hdiag_of(L, [W1, W2], R), rtol=1e-12, atol=1e-12)
    op1 = HeffOperator(L, R, [rng.standard_normal((3, 4, 4, 2))], (6, 4, 5), prec="fp64")
    np.testing.assert_allclose(op1.diag().cpu().numpy(), O.hdiag_of(L, [op1.W[0].cpu().numpy()], R), rtol=1e-12,
                               atol=1e-12)


def test_vector_kernels_vs_numpy():
    from renormalizer_b200._native import Engine, ptr
    eng = Engine.get(0)
    rng = np.random.default_rng(5)
    for n in (1, 7, 1000, 300001):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        xd, yd = _dev(x), _dev(y)
        out = torch.zeros(4, dtype=torch.float64, device="cuda")
        ws = eng.vec_workspace()
        eng.check(eng.lib.reno_vec_dotc(eng.ctx, n, 1, ptr(xd), ptr(yd), ptr(out), ptr(ws), ws.numel()), "dotc")
        ref = np.vdot(x, y)
        got = out[0].item() + 1j * out[1].item()
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)) * np.sqrt(n)
        eng.check(eng.lib.reno_vec_norm(eng.ctx, n, 1, ptr(xd), ptr(out), ptr(ws), ws.numel()), "norm")
        assert out[0].item() == pytest.approx(np.linalg.norm(x), rel=1e-13)
        # deterministic: same bits twice
        eng.check(eng.lib.reno_vec_norm(eng.ctx, n, 1, ptr(xd), ptr(out[1:]), ptr(ws), ws.numel()), "norm")
        assert out[0].item() == out[1].item()


def test_heff_invalid_shapes_raise():
    from renormalizer_b200.hop_expr import HeffOperator
    with pytest.raises(AssertionError):
        HeffOperator(np.ones((3, 2, 3)), np.ones((4, 2, 4)), [np.ones((2, 3, 3, 2))], (3, 2, 4))
