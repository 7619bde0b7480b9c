"""The engine's own Holstein / spin-boson models and MPO builder reproduce the
reference's Hamiltonians (dense H of the reference Mpo(model), with and
without an energy offset).  CPU only."""
import numpy as np
import pytest

from conftest import load_golden

MPO = load_golden("mpo_cases.npz")


def holstein(nmol, nlev, modes, J=1.0):
    from renormalizer_b200.model import HolsteinModel, Mol, Phonon, Quantity
    ph = [Phonon.simple_phonon(Quantity(w), Quantity(np.sqrt(2.0) * g / np.sqrt(w)), nlev) for (w, g) in modes]
    return HolsteinModel([Mol(Quantity(0), ph)] * nmol, Quantity(J), 3)


def sbm(omega, c, nlev, delta=1.0, eps=0.0):
    from renormalizer_b200.model import Phonon, Quantity, SpinBosonModel
    ph = [Phonon.simple_phonon(Quantity(w), Quantity(ci / w ** 2), nlev) for w, ci in zip(omega, c)]
    return SpinBosonModel(Quantity(eps), Quantity(delta), ph)


MODELS = {
    "hol3x2": lambda: holstein(3, 2, [(1.0, 1.0 / np.sqrt(2.0))]),
    "hol4x3": lambda: holstein(4, 3, [(1.0, 1.0)]),
    "hol2m2x3": lambda: holstein(2, 3, [(1.0, 1.0), (0.5, 0.7)]),
    "sbm3x3": lambda: sbm(MPO["sbm3x3/omega"], MPO["sbm3x3/c"], 3),
}


@pytest.mark.parametrize("name", sorted(MODELS))
def test_mpo_dense_matches_reference(name):
    from renormalizer_b200.mpo import build_mpo_tensors
    from renormalizer_b200.model import Quantity
    model = MODELS[name]()
    assert list(model.pbond_list) == list(MPO[f"{name}/pdims"])
    Ws = build_mpo_tensors(model, model.ham_terms, 0.0)
    H = _dense(Ws)
    np.testing.assert_allclose(H, MPO[f"{name}/H"], atol=1e-12)
    Ws_off = build_mpo_tensors(model, model.ham_terms, Quantity(0.37).as_au())
    np.testing.assert_allclose(_dense(Ws_off), MPO[f"{name}/H_off"], atol=1e-12)


def test_mpo_bond_dims_match_reference_scale():
    from renormalizer_b200.mpo import build_mpo_tensors
    m = holstein(4, 4, [(1.0, 1.0), (0.5, 0.7)])
    Ws = build_mpo_tensors(m, m.ham_terms)
    assert max(W.shape[3] for W in Ws) <= 5
    from renormalizer_b200.model import SpectralDensityFunction, Quantity
    w, c2 = SpectralDensityFunction(0.5, Quantity(10.0)).Wang1(8)
    s = sbm(w, np.sqrt(c2), 4)
    Ws = build_mpo_tensors(s, s.ham_terms)
    assert max(W.shape[3] for W in Ws) == 3


def _dense(Ws):
    t = Ws[0]
    for W in Ws[1:]:
        t = np.tensordot(t, W, axes=([-1], [0]))
    t = t[0, ..., 0]
    n = len(Ws)
    t = t.transpose([2 * i for i in range(n)] + [2 * i + 1 for i in range(n)])
    d = int(np.prod(t.shape[:n]))
    return t.reshape(d, d)
