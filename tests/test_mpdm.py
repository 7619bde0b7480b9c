"""Finite temperature on the engine: MpDm and ThermalProp against the
reference (tests/golden/mpdm_cases.npz, written by make_golden.py from
renormalizer/mps/mpdm.py and thermalprop.py).

The T = infinity one-exciton density operator of a 3-molecule Holstein chain
(3 levels per mode, M = 10) evolves in imaginary time (6 steps of beta / 4000
at 298 K, TDVP-PS and TDVP-PS2, energy offset updated every step as
ThermalProp does).  From the reference's expanded start the engine must give
the same energies, electronic and phonon occupations and bond entropies
after every step: 1e-10 for TDVP-PS2, and for TDVP-PS 2e-7, twice the
reference's own spread on this run (the reference against itself from a
start perturbed by one ulp per entry, three draws: up to 1.1e-8 in the
energies, 2.7e-8 in the electronic and 1.0e-7 in the phonon occupations after
6 steps; 3e-15 for TDVP-PS2: the one-site sweep keeps the start's
1e-10-weight expansion directions, whose rounding the imaginary-time steps
amplify).  The engine's own start (MpDm.max_entangled_ex, ThermalProp's
canonicalisation and Hamiltonian-hint bond expansion) must reproduce the
reference's TDVP-PS2 trajectory to 5e-10.

The ancilla contractions themselves (W (x) 1 on the combined index) are
checked against the reference's ancilla einsums (hop_expr.py:80-116,
lib.py:206-211, 238-243) on random tensors."""
import numpy as np
import pytest
import torch

from conftest import load_golden

MPDM = load_golden("mpdm_cases.npz")


def _model():
    from renormalizer_b200 import HolsteinModel, Mol, Phonon, Quantity
    ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), 3)]
    return HolsteinModel([Mol(Quantity(0), ph)] * 3, Quantity(1.0), 3)


def _start(tag, model):
    from renormalizer_b200 import MpDm
    pre = f"{tag}/init"
    n = int(MPDM[f"{pre}/nsites"])
    sites = [MPDM[f"{pre}/mt_{i}"] for i in range(n)]
    qn = [MPDM[f"{pre}/qn_{i}"] for i in range(n + 1)]
    return MpDm.from_arrays(model, sites, qn, int(MPDM[f"{pre}/qnidx"]), MPDM[f"{pre}/qntot"],
                            bool(MPDM[f"{pre}/to_right"]))


def _run(tag, tol):
    """ThermalProp's step (thermalprop.py:74-109) from the reference's expanded
    start: record, then evolve with the last energy as the MPO offset"""
    from renormalizer_b200 import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, Mpo, Quantity
    model = _model()
    mps = _start(tag, model)
    mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps if tag == "ps" else EvolveMethod.tdvp_ps2)
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=int(MPDM[f"{tag}/mmax"]))
    h_mpo = Mpo(model)
    nsteps = len(MPDM[f"{tag}/energies"]) - 1
    energies, e_occ, ph_occ, ent = [], [], [], []
    for step in range(nsteps + 1):
        energies.append(mps.expectation(h_mpo))
        e_occ.append(mps.e_occupations)
        ph_occ.append(mps.ph_occupations)
        ent.append(mps.calc_bond_entropy())
        if step < nsteps:
            mps = mps.evolve(Mpo(model, offset=Quantity(energies[-1])), complex(MPDM[f"{tag}/dbeta"]))
    np.testing.assert_allclose(energies, MPDM[f"{tag}/energies"], rtol=0, atol=tol)
    np.testing.assert_allclose(e_occ, MPDM[f"{tag}/e_occ"], rtol=0, atol=tol)
    np.testing.assert_allclose(ph_occ, MPDM[f"{tag}/ph_occ"], rtol=0, atol=tol)
    np.testing.assert_allclose(ent, MPDM[f"{tag}/entropy"], rtol=0, atol=10 * tol)
    assert list(mps.bond_dims) == list(MPDM[f"{tag}/bond_dims_final"])


def _own_start(tol):
    """MpDm.max_entangled_ex, ThermalProp's canonicalisation and hint
    expansion and its TDVP-PS2 steps, all in the engine.  (The engine's start
    equals the reference's up to the gauge of each bond -- the kept singular
    vectors' phases -- and rounding; TDVP-PS, which keeps the start's bond
    spaces, amplifies that to ~1e-4 here, so the comparison uses TDVP-PS2.)"""
    from renormalizer_b200 import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, MpDm, ThermalProp
    model = _model()
    np.random.seed(7)  # the completion columns come from numpy's global RNG, as in the reference
    init = MpDm.max_entangled_ex(model)
    init.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=int(MPDM["ps2/mmax"]))
    tp = ThermalProp(init, evolve_config=EvolveConfig(EvolveMethod.tdvp_ps2))
    assert list(tp.latest_mps.bond_dims) == [int(x) for x in _bond_dims("ps2")]
    tp.evolve(evolve_dt=complex(MPDM["ps2/dbeta"]), nsteps=len(MPDM["ps2/energies"]) - 1)
    np.testing.assert_allclose(tp.energies, MPDM["ps2/energies"], rtol=0, atol=tol)
    np.testing.assert_allclose(tp.e_occupations_array, MPDM["ps2/e_occ"], rtol=0, atol=tol)
    np.testing.assert_allclose(tp.ph_occupations_array, MPDM["ps2/ph_occ"], rtol=0, atol=tol)
    np.testing.assert_allclose(tp.vn_entropy_array, MPDM["ps2/entropy"], rtol=0, atol=10 * tol)


def _bond_dims(tag):
    pre = f"{tag}/init"
    n = int(MPDM[f"{pre}/nsites"])
    return [MPDM[f"{pre}/mt_0"].shape[0]] + [MPDM[f"{pre}/mt_{i}"].shape[-1] for i in range(n)]


def _ancilla_contractions(dev):
    """the engine's matvec / environment update with W (x) 1 against the
    reference's ancilla einsums"""
    from renormalizer_b200.hop_expr import HeffOperator
    from renormalizer_b200.lib import contract_one_site
    from renormalizer_b200.mpdm import ancilla_tensor
    rng = np.random.default_rng(4)
    c = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    ml, mr, wl, wm, wr, d1, d2 = 5, 4, 3, 2, 3, 3, 2
    L, R = c(ml, wl, ml), c(mr, wr, mr)
    W1, W2 = rng.standard_normal((wl, d1, d1, wm)), rng.standard_normal((wm, d2, d2, wr))
    Wb = rng.standard_normal((wl, d1, d1, wr))
    psi1 = c(ml, d1, d1, mr)
    ref1 = np.einsum("abc, bdef, lfk, cegk -> adgl", L, Wb, R, psi1)
    y1 = HeffOperator(L, R, [ancilla_tensor(Wb, d1)], (ml, d1 * d1, mr), prec="fp64")(
        torch.as_tensor(psi1.reshape(ml, d1 * d1, mr), device=dev))
    np.testing.assert_allclose(y1.cpu().numpy().reshape(ref1.shape), ref1, rtol=0, atol=1e-12 * np.abs(ref1).max())
    psi2 = c(ml, d1, d1, d2, d2, mr)
    ref2 = np.einsum("abc, bdef, fghj, ljk, cemhnk -> admgnl", L, W1, W2, R, psi2)
    y2 = HeffOperator(L, R, [ancilla_tensor(W1, d1), ancilla_tensor(W2, d2)], (ml, d1 * d1, d2 * d2, mr),
                      prec="fp64")(torch.as_tensor(psi2.reshape(ml, d1 * d1, d2 * d2, mr), device=dev))
    np.testing.assert_allclose(y2.cpu().numpy().reshape(ref2.shape), ref2, rtol=0, atol=1e-12 * np.abs(ref2).max())
    ms = c(ml, d1, d1, mr)
    E = c(ml, wl, ml)
    # lib.py:206-211: the ancilla bond (g) is traced between bra and ket
    refL = np.einsum("abc, adgf, bdeh, cegk -> fhk", E, ms.conj(), Wb, ms)
    outL = contract_one_site(torch.as_tensor(E, device=dev), torch.as_tensor(ms.reshape(ml, d1 * d1, mr), device=dev),
                             torch.as_tensor(ancilla_tensor(Wb, d1), device=dev), "L", prec="fp64")
    np.testing.assert_allclose(outL.cpu().numpy(), refL, rtol=0, atol=1e-12 * np.abs(refL).max())
    Er = c(mr, wr, mr)
    refR = np.einsum("fdga, abc, hdeb, kegc -> fhk", ms.conj(), Er, Wb, ms)
    outR = contract_one_site(torch.as_tensor(Er, device=dev), torch.as_tensor(ms.reshape(ml, d1 * d1, mr), device=dev),
                             torch.as_tensor(ancilla_tensor(Wb, d1), device=dev), "R", prec="fp64")
    np.testing.assert_allclose(outR.cpu().numpy(), refR, rtol=0, atol=1e-12 * np.abs(refR).max())


def test_mpdm_host_logic(cpu_engine):
    _ancilla_contractions("cpu")
    _run("ps2", 1e-10)
    _run("ps", 2e-7)
    _own_start(5e-10)


@pytest.mark.gpu
def test_ancilla_contractions_gpu():
    from renormalizer_b200 import backend
    backend.prec = "fp64"
    _ancilla_contractions("cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("tag,tol", [("ps", 2e-7), ("ps2", 1e-10)])
def test_thermal_prop_matches_reference_gpu(tag, tol):
    from renormalizer_b200 import backend
    backend.prec = "fp64"
    _run(tag, tol)


@pytest.mark.gpu
def test_thermal_prop_own_start_gpu():
    from renormalizer_b200 import backend
    backend.prec = "fp64"
    _own_start(5e-10)
