"""GPU TDVP sweeps (Mps.evolve with tdvp_ps / tdvp_ps2) against the
reference's own trajectories (tests/golden/tdvp_cases.npz) and the oracle.

Both engines start from the reference's dumped initial MPS and MPO tensors.
The plain FP64 engine must reproduce the reference populations within 1e-9
(PS) / 1e-8 (PS2) over these short trajectories: the trajectories amplify
rounding noise (reference vs itself at 1 vs 4 BLAS threads: 2e-12 after 5
steps), and TDVP-PS2 picks gauge-arbitrary zero-weight padding vectors."""
import numpy as np
import pytest
import torch

from conftest import engine_chain, load_golden

pytestmark = pytest.mark.gpu

TDVP = load_golden("tdvp_cases.npz")


def engine_state(tag):
    from renormalizer_b200 import CompressConfig, CompressCriteria
    mps, mpo = engine_chain(TDVP, tag)
    mmax = int(TDVP[f"{tag}/mmax"])
    if mmax > 0:
        mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=mmax)
    return mps, mpo


def run(tag, method):
    from renormalizer_b200 import EvolveConfig, EvolveMethod, backend
    backend.prec = "fp64"
    mps, mpo = engine_state(tag)
    mps.evolve_config = EvolveConfig(getattr(EvolveMethod, method))
    dt = float(TDVP[f"{tag}/dt"])
    pops = [mps.e_occupations]
    for _ in range(TDVP[f"{tag}/pops"].shape[0] - 1):
        mps = mps.evolve(mpo, dt)
        pops.append(mps.e_occupations)
    return np.array(pops), mps


@pytest.mark.parametrize("tag", ["ps_exact3", "ps_hol4"])
def test_tdvp_ps_matches_reference(tag):
    pops, mps = run(tag, "tdvp_ps")
    np.testing.assert_allclose(pops, TDVP[f"{tag}/pops"], atol=1e-9)
    assert abs(mps.mp_norm - 1.0) < 1e-12


@pytest.mark.parametrize("tag", ["ps2_exact3", "ps2_hol2m2"])
def test_tdvp_ps2_matches_reference(tag):
    pops, mps = run(tag, "tdvp_ps2")
    np.testing.assert_allclose(pops, TDVP[f"{tag}/pops"], atol=1e-8)
    assert max(mps.bond_dims) <= int(TDVP[f"{tag}/mmax"])


CFG = load_golden("config_cases.npz")


def _config_run(tag, method, nsteps):
    from renormalizer_b200 import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, backend
    backend.prec = "fp64"
    mps, mpo = engine_chain(CFG, tag)
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=int(CFG[f"{tag}/mmax"]))
    mps.evolve_config = EvolveConfig(getattr(EvolveMethod, method))
    dt = float(CFG[f"{tag}/dt"])
    pops = [mps.e_occupations]
    for _ in range(nsteps):
        mps = mps.evolve(mpo, dt)
        pops.append(mps.e_occupations)
    return np.abs(np.array(pops) - CFG[f"{tag}/pops"][:nsteps + 1]).max(axis=1), mps


def test_config1_matches_reference():
    """Config 1 exactly: 10-molecule Holstein chain (omega = 1, g = 1, 10
    levels), the reference's hint-expanded start at M = 32, 100 steps of
    one-site TDVP-PS at dt = 0.05.  The first five steps agree with the
    reference to 1e-10; after that the trajectory amplifies rounding (the
    reference against itself at 1 vs 4 BLAS threads: 2e-12 after 5 steps,
    5e-10 after 15, 1e-5 after 80), and the engine must stay within 100 times
    the reference's own spread so far."""
    dev, _ = _config_run("c1", "tdvp_ps", 100)
    env = np.maximum.accumulate(np.abs(CFG["c1/pops"] - CFG["c1/pops_t4"]).max(axis=1))
    assert dev[:6].max() <= 1e-10, dev[:6]
    bound = np.maximum(100 * env, 1e-10)
    assert np.all(dev <= bound), [(i, dev[i], env[i]) for i in np.nonzero(dev > bound)[0][:5]]


def test_config2_reduced_matches_reference():
    """Config 2 at reduced size: 4 molecules with two modes (omega = 1 / 0.5,
    g = 1 / 0.7), 16 levels, M = 32, two-site TDVP-PS at dt = 0.025 from the
    reference's hint-expanded start: 1e-10 over the first five steps, 1e-8 to
    step 10, and the reference's final bond dimensions."""
    dev, mps = _config_run("c2red", "tdvp_ps2", 10)
    assert dev[:6].max() <= 1e-10, dev
    assert dev.max() <= 1e-8, dev
    assert list(mps.bond_dims) == list(CFG["c2red/bond_dims_final"])


def test_tdvp_ps_energy_conserved():
    from renormalizer_b200 import EvolveConfig, EvolveMethod
    mps, mpo = engine_state("ps_hol4")
    mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps)
    e0 = mps.expectation(mpo)
    np.testing.assert_allclose(e0, TDVP["ps_hol4/energy"][0], rtol=1e-12)
    for _ in range(3):
        mps = mps.evolve(mpo, 0.05)
    # one-site TDVP conserves energy exactly up to Krylov accuracy
    assert abs(mps.expectation(mpo) - e0) < 1e-7


def test_dense_exact_dynamics():
    """test_evolve.py:128-131 with dense exact propagation in place of qutip."""
    pops, _ = run("ps_exact3", "tdvp_ps")
    assert np.abs(pops - TDVP["ps_exact3/exact_pops"]).mean() < 1e-4


def test_hartree_expand_and_evolve_holstein():
    """the configs' initial-state idiom: Hartree product, random bond expansion, PS2"""
    from renormalizer_b200 import (CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, HolsteinModel, Mol,
                                   Mpo, Mps, Phonon, Quantity)
    ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), 6)]
    model = HolsteinModel([Mol(Quantity(0), ph)] * 4, Quantity(1.0), 3)
    mpo = Mpo(model)
    mps = Mps.hartree_product_state(model, {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=12)
    mps = mps.expand_bond_dimension()
    assert max(mps.bond_dims) == 12
    assert abs(mps.e_occupations[0] - 1.0) < 1e-8
    mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps2)
    e0 = mps.expectation(mpo)
    for _ in range(3):
        mps = mps.evolve(mpo, 0.05)
    occ = mps.e_occupations
    assert abs(occ.sum() - 1.0) < 1e-8
    assert occ[0] < 1.0 - 1e-4  # the exciton moved
    assert abs(mps.expectation(mpo) - e0) < 1e-4
