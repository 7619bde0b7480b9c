"""Imaginary-time propagation of a density operator on the sweep engine.

Drop-in for renormalizer/mps/thermalprop.py:13-150 (``ThermalProp``) and
thermalprop.py:153-168 (``load_thermal_state``).  The density operator
(mpdm.MpDm, usually the T = infinity state) is evolved in imaginary time
with the TDVP sweeps of Mps.evolve; at every step the Hamiltonian carries the
previous step's energy as its offset (thermalprop.py:107-109), so the norm
stays representable.  After every step the energy, the electronic and phonon
occupations and the bond entropies are recorded (thermalprop.py:75-96).

Not part of the engine: the exact (local-Hamiltonian) propagator
(``exact=True``, Mpo.exact_propagator) and the ``properties`` hook.
"""
from __future__ import annotations

import logging

import numpy as np

from .configs import EvolveConfig
from .model import Model, Quantity
from .mpdm import MpDm
from .mpo import Mpo
from .tdmps import TdMpsJob

logger = logging.getLogger(__name__)


class ThermalProp(TdMpsJob):
    def __init__(self, init_mpdm: MpDm, h_mpo_model: Model = None, exact: bool = False, space: str = "GS",
                 evolve_config: EvolveConfig = None, dump_mps: bool = None, dump_dir: str = None,
                 job_name: str = None, properties=None, auto_expand: bool = True):
        if exact:
            raise NotImplementedError("the exact local propagator is outside the sweep engine")
        if properties is not None:
            raise NotImplementedError("the Property hook is outside the sweep engine")
        assert space in ("GS", "EX")
        self.init_mpdm: MpDm = init_mpdm.canonicalise()
        if h_mpo_model is None:
            h_mpo_model = self.init_mpdm.model
        self.h_mpo = Mpo(h_mpo_model)
        self.exact = exact
        self.space = space
        self.energies = []
        self._e_occupations_array = []
        self._ph_occupations_array = []
        self._vn_entropy_array = []
        self.properties = properties
        self.auto_expand = auto_expand
        super().__init__(evolve_config=evolve_config, dump_mps=dump_mps, dump_dir=dump_dir, job_name=job_name)

    def init_mps(self):
        """thermalprop.py:68-72"""
        self.init_mpdm.evolve_config = self.evolve_config
        if self.evolve_config.is_tdvp and self.auto_expand:
            self.init_mpdm = self.init_mpdm.expand_bond_dimension(self.h_mpo)
        return self.init_mpdm

    def process_mps(self, mps):
        """thermalprop.py:74-96"""
        self.energies.append(mps.expectation(self.h_mpo))
        self._e_occupations_array.append(mps.e_occupations)
        self._ph_occupations_array.append(mps.ph_occupations)
        self._vn_entropy_array.append(mps.calc_bond_entropy())
        logger.info(f"Energy: {self.energies[-1]}, total electron: {self._e_occupations_array[-1].sum()}")

    def evolve_prop(self, old_mpdm, evolve_dt):
        """thermalprop.py:107-109"""
        h_mpo = Mpo(self.h_mpo.model, offset=Quantity(self.energies[-1]))
        return old_mpdm.evolve(h_mpo, evolve_dt)

    def evolve_single_step(self, evolve_dt):
        return self.evolve_prop(self.latest_mps, evolve_dt)

    def evolve(self, evolve_dt=None, nsteps=None, evolve_time=None):
        """thermalprop.py:119-124: imaginary steps only"""
        if evolve_dt is not None:
            assert np.iscomplex(evolve_dt) and evolve_dt.imag < 0
        if evolve_time is not None:
            assert np.iscomplex(evolve_time) and evolve_time.imag < 0
        return super().evolve(evolve_dt, nsteps, evolve_time)

    @property
    def e_occupations_array(self):
        return np.array(self._e_occupations_array)

    @property
    def ph_occupations_array(self):
        return np.array(self._ph_occupations_array)

    @property
    def vn_entropy_array(self):
        return np.array(self._vn_entropy_array)

    def get_dump_dict(self):
        """thermalprop.py:138-150"""
        return {"time series": [-t.imag for t in self.evolve_times], "energies": self.energies,
                "electron occupations array": self.e_occupations_array.tolist(),
                "phonon occupations array": self.ph_occupations_array.tolist(),
                "vn entropy array": self.vn_entropy_array.tolist()}


def load_thermal_state(model, path: str):
    """thermalprop.py:153-168: the MpDm stored at ``path``, or None"""
    try:
        logger.info(f"Try load from {path}")
        return MpDm.load(model, path)
    except FileNotFoundError:
        logger.info(f"No file found in {path}")
        return None
