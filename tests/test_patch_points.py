"""The engine dropped into the reference's own sweep through its patch
points (renormalizer.mps.mps.{hop_expr, Environ, expm_krylov}), on the CPU
stand-in engine: the reference's unmodified Mps.evolve (one-site TDVP-PS and
two-site TDVP-PS2) must give the populations it gives on its own, and must
really call the engine.  Needs the reference package (the build container);
skipped where it is absent."""
import sys
from pathlib import Path

import numpy as np
import pytest

REF = Path("/root/reference")
SHIMS = Path(__file__).resolve().parents[1] / "oracle" / "_shims"


@pytest.fixture
def reference(monkeypatch):
    if not (REF / "renormalizer").is_dir():
        pytest.skip("the reference package is not present here")
    import torch
    # torch.einsum (the CPU stand-in engine) would route through the reference's
    # opt_einsum stand-in, which has no contract_path
    monkeypatch.setattr(torch.backends.opt_einsum, "enabled", False)
    for p in (str(SHIMS), str(REF)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import logging
    logging.disable(logging.WARNING)
    import renormalizer  # noqa: F401
    return renormalizer


def _chain(method):
    from renormalizer.model import HolsteinModel, Mol, Phonon
    from renormalizer.mps import Mpo, Mps
    from renormalizer.utils import CompressConfig, CompressCriteria, EvolveConfig, Quantity
    ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), 4)]
    model = HolsteinModel([Mol(Quantity(0), ph)] * 3, Quantity(1.0), 3)
    mpo = Mpo(model)
    np.random.seed(5)
    mps = Mps.hartree_product_state(model, {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=6)
    mps = mps.expand_bond_dimension(mpo, include_ex=False)
    mps.evolve_config = EvolveConfig(method)
    return mps, mpo


@pytest.mark.parametrize("method", ["tdvp_ps", "tdvp_ps2"])
def test_reference_evolve_with_engine_patched_in(reference, cpu_engine, method):
    from renormalizer.utils import EvolveMethod
    from renormalizer_b200 import patch
    m = getattr(EvolveMethod, method)
    mps, mpo = _chain(m)
    ref = mps.copy()
    for _ in range(3):
        np.random.seed(0)
        ref = ref.evolve(mpo, 0.05)
    n0 = cpu_engine.launches
    calls = {"heff": 0}
    orig = cpu_engine.heff_apply

    def counting(*a, **k):
        calls["heff"] += 1
        return orig(*a, **k)

    cpu_engine.heff_apply = counting
    patch.install()
    try:
        import renormalizer.mps.mps as M
        assert M.hop_expr is patch.hop_expr and M.Environ is patch.Environ
        got = mps.copy()
        for _ in range(3):
            np.random.seed(0)
            got = got.evolve(mpo, 0.05)
    finally:
        patch.uninstall()
    import renormalizer.mps.mps as M
    assert M.hop_expr is not patch.hop_expr
    assert calls["heff"] > 0
    np.testing.assert_allclose(np.asarray(got.e_occupations), np.asarray(ref.e_occupations), atol=1e-11)
