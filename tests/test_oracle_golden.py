"""Pin the CPU oracle to fixtures produced by the Renormalizer reference.

These run without a GPU: they prove that oracle/reno_oracle.py restates the
reference faithfully, so that the GPU parity tests can trust it.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden, mpo_from_golden, mps_from_golden
from oracle import reno_oracle as O

HEFF = load_golden("heff_cases.npz")
ENV = load_golden("env_cases.npz")
KRY = load_golden("krylov_cases.npz")
SVD = load_golden("svd_cases.npz")
TDVP = load_golden("tdvp_cases.npz")
DMRG = load_golden("dmrg_cases.npz")


@pytest.mark.parametrize("case", golden_cases(HEFF))
def test_oracle_hop_matches_reference(case):
    n = int(HEFF[f"{case}/nsite"])
    Ws = [HEFF[f"{case}/W{i + 1}"] for i in range(n)]
    y = O.hop(HEFF[f"{case}/L"], Ws, HEFF[f"{case}/R"], HEFF[f"{case}/psi"])
    ref = HEFF[f"{case}/y"]
    assert y.shape == ref.shape
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("case", golden_cases(ENV))
def test_oracle_env_matches_reference(case):
    bra = ENV[f"{case}/bra"] if f"{case}/bra" in ENV.files else None
    out = O.contract_one_site(ENV[f"{case}/E"], ENV[f"{case}/ms"], ENV[f"{case}/W"], str(ENV[f"{case}/domain"]),
                              ms_conj=bra)
    ref = ENV[f"{case}/out"]
    assert out.shape == ref.shape
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("k", range(int(KRY["count"])))
def test_oracle_krylov_matches_reference(k):
    A = KRY[f"k{k}/A"]
    dt = KRY[f"k{k}/dt"][()]
    res, n = O.expm_krylov(lambda x: A.dot(x), dt, KRY[f"k{k}/v"].copy())
    assert n == int(KRY[f"k{k}/n"])
    np.testing.assert_allclose(res, KRY[f"k{k}/res"], rtol=1e-11, atol=1e-12)


def test_oracle_svd_qn_matches_reference():
    c, ql, qr, qt = SVD["c"], SVD["qnbigl"], SVD["qnbigr"], SVD["qntot"]
    for fm, tag in ((True, "full"), (False, "econ")):
        np.random.seed(5)
        u, su, qnl, v, sv, qnr = O.svd_qn(c, ql, qr, qt, full_matrices=fm)
        assert u.shape[1] == int(SVD[f"{tag}/ucols"]) and v.shape[1] == int(SVD[f"{tag}/vcols"])
        np.testing.assert_allclose(np.sort(su), np.sort(SVD[f"{tag}/su"]), atol=1e-12)
        np.testing.assert_allclose(np.sort(sv), np.sort(SVD[f"{tag}/sv"]), atol=1e-12)
        # QN labels of the nonzero singular triplets agree as multisets
        assert sorted(map(tuple, np.array(qnl))) == sorted(map(tuple, SVD[f"{tag}/qnl"]))
        if fm:
            ms, mdim, mqn, comp = O.select_basis(u, su, qnl, v, 7, percent=0)
            assert mdim == int(SVD["sel/mdim"])
            np.testing.assert_allclose(ms @ comp.T, SVD["sel/recon"], atol=1e-12)
            ms2, _, mqn2, comp2 = O.select_basis(u, su, qnl, v, 7, percent=0.4)
            np.testing.assert_allclose(ms2 @ comp2.T, SVD["sel40/recon"], atol=1e-12)
    for system in ("L", "R"):
        u, qnl, v, qnr = O.svd_qn(c, ql, qr, qt, QR=True, system=system, full_matrices=False)
        np.testing.assert_allclose(u @ v.T, SVD[f"qr{system}/recon"], atol=1e-12)
        # the QR factors reconstruct the QN-masked coefficient
        np.testing.assert_allclose(u @ v.T, c.reshape(u.shape[0], v.shape[0]), atol=1e-12)


def _traj(tag, fn, src=None, nsteps=None):
    src = TDVP if src is None else src
    init = mps_from_golden(src, f"{tag}/init", compress=O.Compress("fixed", max_bonddim=int(src[f"{tag}/mmax"])))
    mpo = mpo_from_golden(src, f"{tag}/mpo", len(init))
    dt = float(src[f"{tag}/dt"])
    e_sites = [i for i, s in enumerate(init.sigmaqn) if s.shape[0] == 2 and s[1, 0] == 1]
    op = np.diag([0.0, 1.0])
    pops = [[O.site_expectations(init, {i: op for i in e_sites})[i] for i in e_sites]]
    mps = init
    for _ in range(src[f"{tag}/pops"].shape[0] - 1 if nsteps is None else nsteps):
        mps = fn(mps, mpo, dt)
        ex = O.site_expectations(mps, {i: op for i in e_sites})
        pops.append([ex[i] for i in e_sites])
    return np.array(pops)


@pytest.mark.parametrize("tag", ["ps_exact3", "ps_hol4"])
def test_oracle_tdvp_ps_matches_reference(tag):
    pops = _traj(tag, O.evolve_tdvp_ps)
    ref = TDVP[f"{tag}/pops"]
    # short trajectories reproduce the reference to rounding-noise level
    np.testing.assert_allclose(pops, ref, atol=1e-9)


@pytest.mark.parametrize("tag", ["ps2_exact3", "ps2_hol2m2"])
def test_oracle_tdvp_ps2_matches_reference(tag):
    pops = _traj(tag, O.evolve_tdvp_ps2)
    ref = TDVP[f"{tag}/pops"]
    np.testing.assert_allclose(pops, ref, atol=1e-8)


def test_oracle_config1_first_steps_match_reference():
    """Config 1 (10-molecule Holstein chain, M = 32, TDVP-PS, dt = 0.05) from
    the reference's own hint-expanded start: the oracle's first five steps
    reproduce the reference's populations to 1e-10 (the reference moves by
    2e-12 between 1 and 4 BLAS threads over these steps)."""
    cfg = load_golden("config_cases.npz")
    pops = _traj("c1", O.evolve_tdvp_ps, src=cfg, nsteps=5)
    np.testing.assert_allclose(pops, cfg["c1/pops"][:6], atol=1e-10)
    env = np.abs(cfg["c1/pops"] - cfg["c1/pops_t4"]).max(axis=1)
    assert env[5] < 1e-10 < env[30]


def test_oracle_dense_exact_dynamics():
    """TDVP-PS of the 3-site model against dense exact propagation (stands in
    for the qutip oracle of mps/tests/test_evolve.py:128-131, mean dev < 1e-4)."""
    pops = _traj("ps_exact3", O.evolve_tdvp_ps)
    assert np.abs(pops - TDVP["ps_exact3/exact_pops"]).mean() < 1e-4


@pytest.mark.parametrize("tag", ["hol_test_gs", "sbm6x4"])
def test_oracle_dmrg_matches_reference(tag):
    init = mps_from_golden(DMRG, f"{tag}/init")
    mpo = mpo_from_golden(DMRG, f"{tag}/mpo", len(init))
    ref = DMRG[f"{tag}/energies"]
    proc = {"hol_test_gs": [[10, 0.4], [20, 0.2], [30, 0.1], [40, 0], [40, 0]],
            "sbm6x4": [[12, 0.4], [12, 0.2], [12, 0.1], [12, 0], [12, 0], [12, 0]]}[tag]
    energies, _ = O.optimize_mps(init, mpo, proc, e_atol=1e-8 if tag == "hol_test_gs" else 1e-9)
    # every sweep's energy, and the number of sweeps before convergence
    assert len(energies) == len(ref)
    np.testing.assert_allclose(energies, ref, rtol=1e-11)
    if tag == "hol_test_gs":
        assert min(energies) == pytest.approx(float(DMRG["hol_test_gs/GS_E"]), rel=1e-5)
