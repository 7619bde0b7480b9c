"""npz 0.4 dump / load (mp.py:1085-1113, mps.py:352-386) and the TdMpsJob
checkpoint files (utils/tdmps.py:181-207), on the CPU stand-in engine.  With
the reference package present, files cross in both directions: the
reference's Mps.load reads the engine's dumps and the engine reads the
reference's."""
import sys
from pathlib import Path

import numpy as np
import pytest

REF = Path("/root/reference")
SHIMS = Path(__file__).resolve().parents[1] / "oracle" / "_shims"


def _model():
    from renormalizer_b200 import HolsteinModel, Mol, Phonon, Quantity
    ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), 4)]
    return HolsteinModel([Mol(Quantity(0), ph)] * 3, Quantity(1.0), 3)


def _job_class():
    from renormalizer_b200 import (CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, Mpo, Mps,
                                   TdMpsJob)

    class Job(TdMpsJob):
        def __init__(self, model, **kw):
            self.model = model
            self.mpo = Mpo(model)
            self.pops = []
            super().__init__(EvolveConfig(EvolveMethod.tdvp_ps2), **kw)

        def init_mps(self):
            mps = Mps.hartree_product_state(self.model, {0: 1})
            mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=6)
            mps = mps.expand_bond_dimension(self.mpo, include_ex=False)
            mps.evolve_config = self.evolve_config
            return mps

        def process_mps(self, mps):
            self.pops.append(mps.e_occupations)

        def evolve_single_step(self, evolve_dt):
            return self.latest_mps.evolve(self.mpo, evolve_dt)

        def get_dump_dict(self):
            return {"time series": np.array(self.evolve_times), "population": np.array(self.pops)}

    return Job


def test_tdmpsjob_checkpoints_and_reload(cpu_engine, tmp_path):
    from renormalizer_b200 import Mps
    model = _model()
    job = _job_class()(model, dump_mps="all", dump_dir=str(tmp_path), job_name="hol3")
    job.evolve(evolve_dt=0.05, nsteps=3)
    assert np.allclose(job.evolve_times, [0, 0.05, 0.1, 0.15])
    d = np.load(tmp_path / "hol3.npz")
    assert d["population"].shape == (4, 3) and not (tmp_path / "hol3.npz.bak").exists()
    for step in (1, 2, 3):
        assert (tmp_path / f"hol3_mps_{step}.npz").exists()
    back = Mps.load(model, str(tmp_path / "hol3_mps_3.npz"))
    for a, b in zip(back, job.latest_mps):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
    assert back.qnidx == job.latest_mps.qnidx and back.to_right == job.latest_mps.to_right
    assert back.coeff == job.latest_mps.coeff
    np.testing.assert_allclose(back.e_occupations, job.pops[-1], atol=1e-14)
    # evolve_time / nsteps forms of the driver
    job.evolve(evolve_dt=0.05, evolve_time=0.1)
    assert len(job.evolve_times) == 4 + 3


@pytest.fixture
def reference(monkeypatch):
    if not (REF / "renormalizer").is_dir():
        pytest.skip("the reference package is not present here")
    for p in (str(SHIMS), str(REF)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import logging
    logging.disable(logging.WARNING)
    import renormalizer  # noqa: F401
    return renormalizer


def test_npz_files_cross_with_the_reference(reference, cpu_engine, tmp_path):
    from renormalizer.model import HolsteinModel as RModel, Mol as RMol, Phonon as RPhonon
    from renormalizer.mps import Mpo as RMpo, Mps as RMps
    from renormalizer.utils import CompressConfig as RCC, CompressCriteria as RCrit, Quantity as RQ
    from renormalizer_b200 import Mps
    # a reference-written dump, read by the engine
    ph = [RPhonon.simple_phonon(RQ(1.0), RQ(np.sqrt(2.0)), 4)]
    rmodel = RModel([RMol(RQ(0), ph)] * 3, RQ(1.0), 3)
    rmps = RMps.hartree_product_state(rmodel, {0: 1})
    rmps.compress_config = RCC(RCrit.fixed, max_bonddim=6)
    rmps = rmps.expand_bond_dimension(RMpo(rmodel), include_ex=False)
    rmps.dump(str(tmp_path / "ref.npz"))
    ours = Mps.load(_model(), str(tmp_path / "ref.npz"))
    np.testing.assert_allclose(ours.todense(), np.asarray(rmps.todense()), atol=1e-15)
    assert ours.qnidx == rmps.qnidx and list(ours.qntot) == list(rmps.qntot)
    # an engine-written dump, read by the reference
    ours.dump(str(tmp_path / "ours.npz"))
    back = RMps.load(rmodel, str(tmp_path / "ours.npz"))
    np.testing.assert_allclose(np.asarray(back.todense()), ours.todense(), atol=1e-15)
    assert back.qnidx == ours.qnidx and back.to_right == ours.to_right
    for qa, qb in zip(back.qn, ours.qn):
        assert np.array_equal(np.asarray(qa), np.asarray(qb))
