"""Host logic of the sweep engine on the CPU stand-in engine (no GPU):
QN bookkeeping, QN-blocked truncation order, TDVP-PS / PS2 control flow and
the Krylov driver, checked against the reference's own trajectories."""
import numpy as np
import pytest

from conftest import load_golden
from test_gpu_tdvp import TDVP, engine_state


def _run(tag, method, steps=None):
    from renormalizer_b200 import EvolveConfig, EvolveMethod
    mps, mpo = engine_state(tag)
    mps.evolve_config = EvolveConfig(getattr(EvolveMethod, method))
    dt = float(TDVP[f"{tag}/dt"])
    pops = [mps.e_occupations]
    n = TDVP[f"{tag}/pops"].shape[0] - 1 if steps is None else steps
    for _ in range(n):
        mps = mps.evolve(mpo, dt)
        pops.append(mps.e_occupations)
    return np.array(pops), mps


@pytest.mark.parametrize("tag", ["ps_exact3", "ps_hol4"])
def test_host_tdvp_ps(cpu_engine, tag):
    pops, mps = _run(tag, "tdvp_ps")
    np.testing.assert_allclose(pops, TDVP[f"{tag}/pops"], atol=1e-9)


@pytest.mark.parametrize("tag", ["ps2_exact3", "ps2_hol2m2"])
def test_host_tdvp_ps2(cpu_engine, tag):
    pops, mps = _run(tag, "tdvp_ps2")
    np.testing.assert_allclose(pops, TDVP[f"{tag}/pops"], atol=1e-8)
    assert list(mps.bond_dims) == list(TDVP[f"{tag}/bond_dims_final"])


def test_host_expand_and_canonical(cpu_engine):
    from renormalizer_b200 import (CompressConfig, CompressCriteria, HolsteinModel, Mol, Mpo, Mps, Phonon,
                                   Quantity)
    ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), 5)]
    model = HolsteinModel([Mol(Quantity(0), ph)] * 3, Quantity(1.0), 3)
    mps = Mps.hartree_product_state(model, {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=7)
    np.random.seed(3)
    mps = mps.expand_bond_dimension()
    assert max(mps.bond_dims) == 7
    assert abs(mps.mp_norm - 1.0) < 1e-12
    assert abs(mps.e_occupations[0] - 1.0) < 1e-8
    assert mps.check_left_canonical() or mps.check_right_canonical()


def _hartree_of(tag):
    """The reference chain's model with the Hartree product it expanded
    (exciton on the first electronic site)."""
    from conftest import engine_chain
    from renormalizer_b200 import Mps
    ref, mpo = engine_chain(TDVP, tag)
    model = ref.model
    first_e = next(b for b in model.basis if getattr(b, "is_electron", False))
    return ref, mpo, Mps.hartree_product_state(model, {first_e.dof: 1})


@pytest.mark.parametrize("tag", ["ps_hol4", "ps2_hol2m2"])
def test_host_expand_with_hint_mpo_matches_reference(cpu_engine, tag):
    """expand_bond_dimension(mpo, include_ex=False) (mps.py:1934-2023) gives
    the reference's expanded start state: same bond dimensions and, with the
    product-state component divided out, the same 1e-10-weight expansion
    directions (dense comparison)."""
    from renormalizer_b200 import CompressConfig, CompressCriteria
    ref, mpo, h = _hartree_of(tag)
    h.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=int(TDVP[f"{tag}/mmax"]))
    ours = h.expand_bond_dimension(mpo, include_ex=False)
    assert list(ours.bond_dims) == list(ref.bond_dims)
    psi0 = h.todense().ravel()
    psi0 = psi0 / np.linalg.norm(psi0)
    parts = []
    for m in (ours, ref):
        v = m.todense().ravel() * complex(m.coeff)
        parts.append(v / np.vdot(psi0, v) - psi0)
    assert 5e-11 < np.linalg.norm(parts[1]) < 1e-9
    assert np.linalg.norm(parts[0] - parts[1]) < 1e-13


def test_host_mpo_times_mps_conserves_qn(cpu_engine):
    """Mpo @ Mps (mpo.py:331-389): the product's QN labels describe its
    tensors -- every entry whose left label + site QN differs from its right
    label is zero -- and the Hamiltonian keeps the total QN."""
    from renormalizer_b200 import (CompressConfig, CompressCriteria, HolsteinModel, Mol, Mpo, Mps, Phonon,
                                   Quantity)
    from renormalizer_b200.svd_qn import add_outer
    ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), 3)]
    model = HolsteinModel([Mol(Quantity(0), ph)] * 3, Quantity(1.0), 3)
    mpo = Mpo(model)
    assert list(mpo.qntot) == [0]
    np.random.seed(5)
    mps = Mps.random(model, 1, 6)
    out = mpo @ mps
    assert list(out.qntot) == [1]
    out.move_qnidx(len(out) - 1)
    for i, t in enumerate(out):
        a = t.cpu().numpy()
        lab = add_outer(out.qn[i], np.asarray(model.basis[i].sigmaqn).reshape(-1, 1)).reshape(-1)
        right = out.qn[i + 1].reshape(-1) if i < len(out) - 1 else out.qntot
        mask = lab[:, None] != np.asarray(right).reshape(1, -1)
        assert np.all(np.abs(a.reshape(-1, a.shape[-1])[mask]) < 1e-14)
    # the dense product equals H |psi>
    np.testing.assert_allclose(out.todense(), mpo.todense() @ mps.todense(), atol=1e-12)
