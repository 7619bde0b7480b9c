"""Gradient of a site population after a TDVP-PS trajectory with respect to
per-molecule Holstein couplings g_i (renormalizer_b200.tdvp_grad), on a
3-molecule chain (6 MPS sites, 3 levels, M = 4, 4 steps of dt = 0.1).

* the engine gradient (hand-written H_eff and contraction backwards,
  checkpointed steps) against the same trajectory differentiated by torch
  autograd through FP64 tensordot / einsum: 1e-10 relative;
* against central finite differences of the trajectory evaluated with the
  MPO rebuilt at g0 +- h e_j (h = 1e-5): 1e-7 absolute;
* the trajectory value against the engine's own TDVP-PS (adaptive Krylov,
  QN-blocked QR) from the same start: 1e-6 (the fixed Lanczos order is the
  only difference)."""
import numpy as np
import pytest
import torch


def _setup(dev):
    from renormalizer_b200 import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, HolsteinModel, Mol, \
        Mpo, Mps, Phonon, Quantity
    def model(g):
        mols = [Mol(Quantity(0.1 * i), [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0) * gi), 3)])
                for i, gi in enumerate(g)]
        return HolsteinModel(mols, Quantity(1.0), 3)
    g0 = np.array([0.8, 1.1, 1.3])
    build = lambda g: [Mpo(model(g)).numpy(i) for i in range(6)]
    np.random.seed(11)
    mps = Mps.hartree_product_state(model(g0), {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=4)
    mps = mps.expand_bond_dimension()
    mps.ensure_right_canonical()
    mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps)
    return model, build, g0, mps


def _run(dev):
    from renormalizer_b200 import Mpo, backend
    from renormalizer_b200.tdvp_grad import coupling_gradient, trajectory_value
    backend.prec = "fp64"
    model, build, g0, mps = _setup(dev)
    sites0 = [mps[i] for i in range(len(mps))]
    op = np.diag([0.0, 1.0])
    dt, nsteps, k = 0.1, 4, 8
    val, grad = coupling_gradient(build, g0, sites0, dt, nsteps, 0, op, krylov=k, checkpoint_every=2)
    val_e, grad_e = coupling_gradient(build, g0, [s.cpu() for s in sites0], dt, nsteps, 0, op, krylov=k,
                                      checkpoint_every=0, contract="einsum")
    assert abs(val - val_e) < 1e-12
    assert np.abs(grad - grad_e).max() <= 1e-10 * np.abs(grad_e).max()
    h = 1e-5
    for j in range(len(g0)):
        e = np.zeros(len(g0))
        e[j] = h
        fp = trajectory_value(build(g0 + e), sites0, dt, nsteps, 0, op, krylov=k)
        fm = trajectory_value(build(g0 - e), sites0, dt, nsteps, 0, op, krylov=k)
        assert abs((fp - fm) / (2 * h) - grad[j]) < 1e-7, (j, (fp - fm) / (2 * h), grad[j])
    # the engine's own TDVP-PS from the same right-canonical start
    m = mps.copy()
    mpo = Mpo(model(g0))
    for _ in range(nsteps):
        m = m.evolve(mpo, dt)
    assert abs(m.e_occupations[0] - val) < 1e-6
    return val, grad


def test_tdvp_gradient_host_logic(cpu_engine):
    _run("cpu")


@pytest.mark.gpu
def test_tdvp_gradient_gpu():
    _run("cuda")


def test_batched_trajectory_values_match_single_cpu(cpu_engine):
    """trajectory_values (batched FP64 torch contractions, the finite-difference
    helper) equals trajectory_value(contract="einsum") per coupling set"""
    from renormalizer_b200.tdvp_grad import trajectory_value, trajectory_values
    _, build, g0, mps = _setup("cpu")
    sites0 = [mps[i].cpu() for i in range(len(mps))]
    op = np.diag([0.0, 1.0])
    gs = [g0, g0 + np.array([1e-3, 0, 0]), g0 - np.array([0, 0, 2e-3])]
    got = trajectory_values([build(g) for g in gs], sites0, 0.1, 3, 0, op, krylov=8)
    for g, v in zip(gs, got):
        ref = trajectory_value(build(g), sites0, 0.1, 3, 0, op, krylov=8, contract="einsum")
        assert abs(v - ref) < 1e-13, (v, ref)


def test_batched_lanczos_mixed_breakdown():
    """an instance whose Krylov space is exhausted earlier than the others'
    gets the result of its own run"""
    from renormalizer_b200.tdvp_grad import expm_krylov_fixed
    rng = np.random.default_rng(2)
    h = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    H = torch.as_tensor(h + h.conj().T)
    low = torch.zeros((6, 6), dtype=torch.complex128)
    low[:2, :2] = H[:2, :2]                       # Krylov space of dimension 2 from e_0
    v = torch.zeros(6, dtype=torch.complex128)
    v[0], v[1] = 1.0, 0.5j
    Hs = torch.stack([H, low])
    out = expm_krylov_fixed(lambda x: torch.einsum("bij,bj->bi", Hs, x), -0.3j, torch.stack([v, v]), 5, nb=1)
    for i, M in enumerate((H, low)):
        ref = expm_krylov_fixed(lambda x: M @ x, -0.3j, v, 5)
        assert float((out[i] - ref).abs().max()) < 1e-13
