"""Time-evolution job driver with the reference's checkpoint files.

Drop-in for renormalizer/utils/tdmps.py:19-223 (``TdMpsJob``): a subclass
provides ``init_mps``, ``process_mps``, ``evolve_single_step`` and
``get_dump_dict``; ``evolve(evolve_dt, nsteps, evolve_time)`` runs the steps.
When ``dump_dir`` and ``job_name`` are set, every step writes the properties
to ``<dump_dir>/<job_name>.npz`` (the previous file is kept as ``.bak``
until the new one is complete, so an interrupted dump leaves one intact
file, tdmps.py:181-195) and, with ``dump_mps`` "one" / "all", the latest MPS
as ``<job_name>_mps.npz`` / ``<job_name>_mps_<step>.npz`` in the npz 0.4
protocol (tdmps.py:197-206) -- files the reference's ``Mps.load`` reads, and
this engine's ``Mps.load`` reads the reference's.
"""
from __future__ import annotations

import logging
import os
from datetime import datetime

import numpy as np

from .configs import EvolveConfig

logger = logging.getLogger(__name__)


class TdMpsJob:
    def __init__(self, evolve_config: EvolveConfig = None, dump_mps: str = None, dump_dir: str = None,
                 job_name: str = None):
        self.evolve_config = evolve_config if evolve_config is not None else EvolveConfig()
        self.evolve_times = [0]
        self.info_interval = 1
        if dump_mps not in (None, "all", "one"):
            raise ValueError(f"dump_mps should be None, 'all', 'one'. Got {dump_mps}")
        self.dump_mps = dump_mps
        self._dump_mps = None
        self.dump_dir = dump_dir
        self.job_name = job_name
        mps = self.init_mps()
        if mps is None:
            raise ValueError("init_mps should return an mps. Got None")
        self.latest_mps = mps
        self.process_mps(mps)

    # ---------------------------------------------------------------- to override
    def init_mps(self):
        raise NotImplementedError

    def process_mps(self, mps):
        raise NotImplementedError

    def evolve_single_step(self, evolve_dt):
        raise NotImplementedError

    def get_dump_dict(self):
        raise NotImplementedError

    def stop_evolve_criteria(self):
        return False

    # ---------------------------------------------------------------- driver
    def evolve(self, evolve_dt=None, nsteps=None, evolve_time=None):
        """tdmps.py:68-165: nsteps steps of evolve_dt; evolve_dt from
        evolve_time / nsteps, or nsteps from evolve_time // evolve_dt + 1,
        or (evolve_dt alone) until stop_evolve_criteria."""
        if evolve_dt is not None and nsteps is not None:
            pass
        elif evolve_dt is None and nsteps is not None and evolve_time is not None:
            evolve_dt = evolve_time / float(nsteps)
        elif evolve_dt is not None and nsteps is None and evolve_time is not None:
            nsteps = int(abs(evolve_time) // abs(evolve_dt)) + 1
        elif evolve_dt is not None and nsteps is None and evolve_time is None:
            nsteps = int(1e10)
        else:
            raise ValueError(f"The input parameters evolve_dt:{evolve_dt}, nsteps:{nsteps}, "
                             f"evolve_time:{evolve_time} do not meet the requirements!")
        t0 = datetime.now()
        for i in range(nsteps):
            if self.stop_evolve_criteria():
                logger.info("Criteria to stop the evolution has met. Stop the evolution")
                break
            new_mps = self.evolve_single_step(evolve_dt)
            self.evolve_times.append(self.latest_evolve_time + evolve_dt)
            self.process_mps(new_mps)
            self.latest_mps = new_mps
            self._dump_mps = self.dump_mps if (self.info_interval is not None and i % self.info_interval == 0) \
                else None
            if self._defined_output_path:
                try:
                    self.dump_dict()
                except IOError:  # a failed dump never ends the calculation
                    logger.exception("dumping dict failed with IOError")
        logger.info(f"evolution finished in {datetime.now() - t0}")
        return self

    def dump_dict(self):
        """tdmps.py:181-206"""
        if not self._defined_output_path:
            raise ValueError("Dump dir or job name not set")
        d = self.get_dump_dict()
        os.makedirs(self.dump_dir, exist_ok=True)
        file_path = os.path.join(self.dump_dir, self.job_name + ".npz")
        bak_path = file_path + ".bak"
        if os.path.exists(file_path):
            if os.path.exists(bak_path):
                os.remove(bak_path)
            os.rename(file_path, bak_path)
        np.savez(file_path, **d)
        if os.path.exists(bak_path):
            os.remove(bak_path)
        if self._dump_mps is not None:
            if self._dump_mps == "all":
                name = f"{self.job_name}_mps_{len(self.evolve_times) - 1}.npz"
            else:
                name = f"{self.job_name}_mps.npz"
            self.latest_mps.dump(os.path.join(self.dump_dir, name))

    @property
    def latest_evolve_time(self):
        return self.evolve_times[-1]

    @property
    def evolve_times_array(self):
        return np.array(self.evolve_times)

    @property
    def _defined_output_path(self):
        return self.dump_dir is not None and self.job_name is not None
