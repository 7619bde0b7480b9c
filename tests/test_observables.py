"""On-device observables against the reference (tests/golden/obs_cases.npz,
a 3-molecule two-mode Holstein chain after 4 TDVP-PS2 steps):
calc_1site_rdm (mps.py:1547-1598), calc_bond_singular_values /
calc_bond_entropy (mps.py:1759-1793, compress with ret_s) and expectations
with the shared-environment path (mps.py:527-575, 2103-2169).

Tolerances: RDMs and expectations are contractions (1e-12 relative to the
largest entry); the bond singular values go through an SVD sweep of a
re-canonicalised copy, compared as sorted lists to 1e-12 absolute (sigma <= 1;
the values below sqrt(eps) go through the truncation's cluster refinement);
entropies to 1e-10."""
import numpy as np
import pytest

from conftest import engine_chain, load_golden, mpo_from_golden, mps_from_golden
from oracle import reno_oracle as O

OBS = load_golden("obs_cases.npz")


def _engine_state():
    from renormalizer_b200 import Mpo
    mps, _ = engine_chain(OBS, "obs", mps_key="mps", mpo_key=None)
    ops = [Mpo.from_tensors(mps.model, mpo_from_golden(OBS, f"obs/op{k}", len(mps)))
           for k in range(int(OBS["obs/nops"]))]
    return mps, ops


def _check(mps, ops):
    n = len(mps)
    rdm = mps.calc_1site_rdm()
    for i in range(n):
        ref = OBS[f"obs/rdm_{i}"]
        assert np.abs(rdm[i] - ref).max() <= 1e-12 * np.abs(ref).max()
    sv = mps.calc_bond_singular_values()
    ref = OBS["obs/bond_sv"]
    assert sv.shape == ref.shape
    np.testing.assert_allclose(np.sort(sv, axis=1), np.sort(ref, axis=1), rtol=0, atol=1e-12)
    np.testing.assert_allclose(mps.calc_bond_entropy(sv), OBS["obs/bond_entropy"], atol=1e-10)
    ref = OBS["obs/expectations"]
    for opt in (True, False):
        got = mps.expectations(ops, opt=opt)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_observables_match_reference():
    m = mps_from_golden(OBS, "obs/mps")
    rdm = O.calc_1site_rdm(m)
    for i in range(len(m)):
        np.testing.assert_allclose(rdm[i], OBS[f"obs/rdm_{i}"], atol=1e-14)
    sv = O.calc_bond_singular_values(m)
    np.testing.assert_allclose(np.sort(sv, axis=1), np.sort(OBS["obs/bond_sv"], axis=1), atol=1e-13)
    np.testing.assert_allclose(O.calc_bond_entropy(m, sv), OBS["obs/bond_entropy"], atol=1e-12)
    ops = [mpo_from_golden(OBS, f"obs/op{k}", len(m)) for k in range(int(OBS["obs/nops"]))]
    np.testing.assert_allclose(O.expectations(m, ops), OBS["obs/expectations"], atol=1e-12)


def test_observables_host_logic(cpu_engine):
    _check(*_engine_state())


@pytest.mark.gpu
def test_observables_gpu():
    from renormalizer_b200 import backend
    backend.prec = "fp64"
    _check(*_engine_state())
