"""Split-precision tensor-core path (tcgen05 + TMA, BF16x3 / TF32x3 with FP32
accumulation) against FP64 references.

Tolerances (relative to max|C|): a BF16 hi/lo pair keeps ~17 significant
bits of each operand, a TF32 pair ~22; with the dropped lo*lo term and FP32
accumulation the products agree with FP64 to ~1e-5 (BF16x3) and ~1e-6
(TF32x3).  The bounds below leave a 3-5x margin."""
import numpy as np
import pytest
import torch

from conftest import golden_cases, load_golden
from oracle import reno_oracle as O

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 5e-5, "tf32x3": 5e-6}
HEFF = load_golden("heff_cases.npz")
ENV = load_golden("env_cases.npz")


def _chain_tol(prec, ks):
    """bound for a chain of split GEMMs relative to max|y|: 4 x the per-GEMM
    TOL, grown with sqrt(K / 256) for the longest contraction -- beyond a
    few hundred terms the FP32 accumulation, not the hi/lo split, sets the
    error (which is why TF32x3 is then no more accurate than BF16x3)"""
    return 4 * TOL[prec] * max(1.0, np.sqrt(max(ks) / 256.0))


def _eng():
    from renormalizer_b200._native import Engine
    return Engine.get(0)


def _rand(shape, cplx, g):
    if cplx:
        return torch.complex(torch.randn(shape, dtype=torch.float64, device="cuda", generator=g),
                             torch.randn(shape, dtype=torch.float64, device="cuda", generator=g))
    return torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("ac,bc", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("M,N,K", [(200, 300, 150), (7, 1000, 33), (1000, 9, 260)])
def test_split_gemm_matches_fp64(prec, ac, bc, M, N, K):
    eng = _eng()
    g = torch.Generator(device="cuda").manual_seed(M + 7 * N + K)
    A, B = _rand((M, K), ac, g), _rand((K, N), bc, g)
    C = eng.matmul(A, B, prec=prec)
    ref = A.to(C.dtype) @ B.to(C.dtype)
    err = float((C - ref).abs().max() / ref.abs().max())
    assert err < TOL[prec], err
    assert eng.device_error() == 0


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_split_gemm_strided_conj(prec):
    eng = _eng()
    g = torch.Generator(device="cuda").manual_seed(5)
    A = _rand((300, 129), True, g).transpose(0, 1)  # (129, 300) column-major view
    B = _rand((300, 77), True, g)
    C = eng.matmul(A, B, conj_a=True, prec=prec)
    ref = A.conj() @ B
    assert float((C - ref).abs().max() / ref.abs().max()) < TOL[prec]


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("case", golden_cases(HEFF))
def test_split_heff_matches_reference(prec, case):
    from renormalizer_b200.hop_expr import HeffOperator
    n = int(HEFF[f"{case}/nsite"])
    Ws = [HEFF[f"{case}/W{i + 1}"] for i in range(n)]
    psi = HEFF[f"{case}/psi"]
    op = HeffOperator(HEFF[f"{case}/L"], HEFF[f"{case}/R"], Ws, psi.shape, prec=prec)
    y = op(torch.from_numpy(psi).cuda()).cpu().numpy()
    ref = HEFF[f"{case}/y"]
    # a chain of 2-4 split GEMM stages
    assert np.abs(y - ref).max() / np.abs(ref).max() < 4 * TOL[prec]


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("case", golden_cases(ENV))
def test_split_env_matches_reference(prec, case):
    from renormalizer_b200.lib import contract_one_site
    bra = ENV[f"{case}/bra"] if f"{case}/bra" in ENV.files else None
    out = contract_one_site(ENV[f"{case}/E"], ENV[f"{case}/ms"], ENV[f"{case}/W"], str(ENV[f"{case}/domain"]),
                            ms_conj=bra, prec=prec).cpu().numpy()
    ref = ENV[f"{case}/out"]
    assert np.abs(out - ref).max() / np.abs(ref).max() < 3 * TOL[prec]


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_split_heff_2site_holstein_block(prec):
    """the config's 2-site block shape at reduced M (d1=16, d2=16, w=5)"""
    from renormalizer_b200.hop_expr import HeffOperator
    rng = np.random.default_rng(11)
    ml, mr, d1, d2, w = 64, 48, 16, 16, 5
    mk = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    L, R, psi = mk((ml, w, ml)), mk((mr, w, mr)), mk((ml, d1, d2, mr))
    W1, W2 = rng.standard_normal((w, d1, d1, w)), rng.standard_normal((w, d2, d2, w))
    ref = O.hop(L, [W1, W2], R, psi)
    y = HeffOperator(L, R, [W1, W2], psi.shape, prec=prec)(torch.from_numpy(psi).cuda()).cpu().numpy()
    assert np.abs(y - ref).max() / np.abs(ref).max() < 4 * TOL[prec]


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("ml,mr,d1,d2,wl,wm,wr", [(64, 48, 2, 16, 5, 5, 4), (48, 40, 16, 2, 4, 5, 5),
                                                   (33, 17, 3, 5, 3, 4, 2), (128, 128, 16, 16, 5, 5, 4)])
def test_split_heff_2site_fused_shapes(prec, cplx, ml, mr, d1, d2, wl, wm, wr):
    """the fused 2-site chain (epilogues writing the next stage's packed
    operand): electron-phonon and phonon-electron blocks (runs along K of 2
    elements take the scalar stores), ragged bonds, the real (DMRG) form"""
    from renormalizer_b200.hop_expr import HeffOperator
    rng = np.random.default_rng(ml + d1)
    mk = lambda s: rng.standard_normal(s) + (1j * rng.standard_normal(s) if cplx else 0)
    L, R, psi = mk((ml, wl, ml)), mk((mr, wr, mr)), mk((ml, d1, d2, mr))
    W1, W2 = rng.standard_normal((wl, d1, d1, wm)), rng.standard_normal((wm, d2, d2, wr))
    ref = O.hop(L, [W1, W2], R, psi)
    op = HeffOperator(L, R, [W1, W2], psi.shape, prec=prec)
    y = op(torch.from_numpy(psi).cuda()).cpu().numpy()
    assert y.dtype == ref.dtype
    assert np.abs(y - ref).max() / np.abs(ref).max() < _chain_tol(prec, [2 * ml, wl * d1, wm * d2, 2 * wr * mr])


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("ml,mr,d,wl,wr", [(64, 48, 16, 5, 4), (48, 40, 2, 4, 5), (33, 17, 3, 3, 2),
                                           (256, 256, 16, 5, 5)])
def test_split_heff_1site_fused_shapes(prec, cplx, ml, mr, d, wl, wr):
    """the fused 1-site chain: phonon and electron sites, ragged bonds, the
    real (DMRG) form, the workload's M = 256 phonon site"""
    from renormalizer_b200.hop_expr import HeffOperator
    rng = np.random.default_rng(ml + d)
    mk = lambda s: rng.standard_normal(s) + (1j * rng.standard_normal(s) if cplx else 0)
    L, R, psi = mk((ml, wl, ml)), mk((mr, wr, mr)), mk((ml, d, mr))
    W = rng.standard_normal((wl, d, d, wr))
    ref = O.hop(L, [W], R, psi)
    y = HeffOperator(L, R, [W], psi.shape, prec=prec)(torch.from_numpy(psi).cuda()).cpu().numpy()
    assert y.dtype == ref.dtype
    assert np.abs(y - ref).max() / np.abs(ref).max() < _chain_tol(prec, [2 * ml, wl * d, 2 * wr * mr])


@pytest.mark.parametrize("prec,atol", [("bf16x3", 2e-5), ("tf32x3", 2e-6)])
def test_split_tdvp_short_trajectory(prec, atol):
    from renormalizer_b200 import EvolveConfig, EvolveMethod, backend
    from test_gpu_tdvp import TDVP, engine_state
    backend.prec = prec
    try:
        mps, mpo = engine_state("ps_hol4")
        mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps)
        pops = [mps.e_occupations]
        for _ in range(8):
            mps = mps.evolve(mpo, float(TDVP["ps_hol4/dt"]))
            pops.append(mps.e_occupations)
    finally:
        backend.prec = "fp64"
    dev = np.abs(np.array(pops) - TDVP["ps_hol4/pops"]).max()
    assert dev < atol, dev


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_split_promoted_accumulation(prec):
    """reno_set_split_accumulation_chunk: on operands the split represents
    exactly (so only the accumulation rounds), all-positive, K = 4096, the
    tensor cores' accumulation leaves every output too small (truncation);
    promoting every 128 K elements into round-to-nearest FP32 cuts the bias by
    more than 8x, keeps complex / tile-edge products within the split
    tolerance, and switching it off restores the default kernel's results
    bit for bit."""
    from renormalizer_b200._native import Engine, load_library
    eng, lib = Engine.get(0), load_library()
    g = torch.Generator(device="cuda").manual_seed(2)

    def exact(x):
        if prec == "bf16x3":
            return x.to(torch.bfloat16).to(torch.float64)
        f = x.to(torch.float32)
        return (f.view(torch.int32) & ~((1 << 13) - 1)).view(torch.float32).to(torch.float64)

    A = exact(torch.rand(256, 4096, dtype=torch.float64, device="cuda", generator=g)).contiguous()
    B = exact(torch.rand(4096, 256, dtype=torch.float64, device="cuda", generator=g)).contiguous()
    ref = eng.matmul(A, B, prec="fp64")
    try:
        plain = eng.matmul(A, B, prec=prec)
        assert lib.reno_set_split_accumulation_chunk(128) == 0
        prom = eng.matmul(A, B, prec=prec)
        bias_plain = float((plain - ref).mean() / ref.mean())
        bias_prom = float((prom - ref).mean() / ref.mean())
        assert bias_plain < 0 and bool(((plain - ref) < 0).all())
        assert abs(bias_prom) * 8 < abs(bias_plain), (bias_plain, bias_prom)
        # general operands through the promoted kernel: complex, ragged tiles
        Ac = torch.complex(torch.randn(300, 777, dtype=torch.float64, device="cuda", generator=g),
                           torch.randn(300, 777, dtype=torch.float64, device="cuda", generator=g))
        Bc = torch.randn(777, 190, dtype=torch.float64, device="cuda", generator=g)
        c_ref = eng.matmul(Ac, Bc, prec="fp64")
        c_prom = eng.matmul(Ac, Bc, prec=prec)
        tol = 5e-5 if prec == "bf16x3" else 5e-6
        assert float((c_prom - c_ref).abs().max() / c_ref.abs().max()) < tol
    finally:
        assert lib.reno_set_split_accumulation_chunk(0) == 0
    assert torch.equal(eng.matmul(A, B, prec=prec), plain)
    assert eng.device_error() == 0
