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
