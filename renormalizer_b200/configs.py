"""Configuration objects of the sweep path, mirroring
renormalizer/utils/configs.py (CompressCriteria 13-24, CompressConfig 41-264,
OptimizeConfig 267-300, EvolveMethod 302-321, EvolveConfig 342-416).

Only the fields that the TDVP / DMRG sweep reads are kept; the truncation
rule ``compute_m_trunc`` follows configs.py:196-219 exactly:
threshold keeps sigma / ||sigma|| > threshold, fixed keeps
min(max_dims[bond], len(sigma)), both takes the smaller count.
"""
from __future__ import annotations

from enum import Enum
from typing import Union

import numpy as np


class CompressCriteria(Enum):
    threshold = "threshold"
    fixed = "fixed"
    both = "both"


class CompressConfig:
    def __init__(self, criteria: Union[CompressCriteria, str] = CompressCriteria.threshold, threshold: float = 1e-3,
                 max_bonddim: int = 32):
        if isinstance(criteria, str):
            criteria = CompressCriteria[criteria]
        self.criteria = criteria
        self._threshold = None
        self.threshold = threshold
        self.bond_dim_max_value = max_bonddim
        self.max_dims = None

    @property
    def threshold(self):
        return self._threshold

    @threshold.setter
    def threshold(self, v):
        if v <= 0:
            raise ValueError("non-positive threshold")
        if v == 1:
            raise ValueError("1 is an ambiguous threshold")
        if v > 1:
            raise ValueError("Can't set threshold to be larger than 1")
        self._threshold = v

    def set_bonddim(self, length):
        if self.max_dims is None:
            self.max_dims = np.full(length, self.bond_dim_max_value, dtype=int)

    @property
    def bonddim_should_set(self):
        return self.criteria is not CompressCriteria.threshold and self.max_dims is None

    def _threshold_m_trunc(self, sigma: np.ndarray) -> int:
        assert 0 < self.threshold < 1
        normed = sigma / np.linalg.norm(sigma)
        return int(np.sum(normed > self.threshold))

    def _fixed_m_trunc(self, sigma: np.ndarray, idx: int, left: bool) -> int:
        assert self.max_dims is not None
        return int(min(self.max_dims[idx + 1 if left else idx], len(sigma)))

    def fixed_cap(self, idx: int, left: bool):
        """The kept dimension's upper bound when the rule is ``fixed`` (the
        same bond index as compute_m_trunc); None for threshold-based rules,
        whose count depends on the whole spectrum."""
        if self.criteria is not CompressCriteria.fixed or self.max_dims is None:
            return None
        return int(self.max_dims[idx + 1 if left else idx])

    def compute_m_trunc(self, sigma: np.ndarray, idx: int, left: bool) -> int:
        if self.criteria is CompressCriteria.threshold:
            return self._threshold_m_trunc(sigma)
        if self.criteria is CompressCriteria.fixed:
            return self._fixed_m_trunc(sigma, idx, left)
        return min(self._threshold_m_trunc(sigma), self._fixed_m_trunc(sigma, idx, left))

    def copy(self) -> "CompressConfig":
        new = self.__class__.__new__(self.__class__)
        new.__dict__ = self.__dict__.copy()
        if self.max_dims is not None:
            new.max_dims = self.max_dims.copy()
        return new

    def __str__(self):
        return f"CompressConfig(criteria={self.criteria}, threshold={self.threshold}, " \
               f"max_bonddim={self.bond_dim_max_value})"


class OptimizeConfig:
    def __init__(self, procedure=None):
        self.procedure = procedure if procedure is not None else [[10, 0.4], [20, 0.2], [30, 0.1], [40, 0], [40, 0]]
        self.method = "2site"
        self.algo = "davidson"
        self.nroots = 1
        self.e_rtol = 1e-6
        self.e_atol = 1e-8
        self.inverse = 1.0

    def copy(self):
        new = self.__class__.__new__(self.__class__)
        new.__dict__ = self.__dict__.copy()
        new.procedure = list(self.procedure)
        return new


class EvolveMethod(Enum):
    prop_and_compress = "P&C"
    prop_and_compress_tdrk4 = "P&C TD RK4"
    prop_and_compress_tdrk = "P&C TD RK"
    tdvp_ps = "TDVP PS one-site"
    tdvp_ps2 = "TDVP PS two-site"
    tdvp_vmf = "TDVP Variable Mean Field"
    tdvp_mu_cmf = "TDVP Matrix Unfolding Constant Mean Field"
    tdvp_mu_vmf = "TDVP Matrix Unfolding Variable Mean Field"


class EvolveConfig:
    """The sweep engine implements the projector-splitting TDVP schemes
    (tdvp_ps, tdvp_ps2) with the Krylov propagator (ivp_solver='krylov')."""

    def __init__(self, method: Union[EvolveMethod, str] = EvolveMethod.tdvp_ps, adaptive=False, guess_dt=1e-1,
                 adaptive_rtol=5e-4, ivp_rtol=1e-5, ivp_atol=1e-8, ivp_solver="krylov", fixed_krylov=None):
        if isinstance(method, str):
            method = EvolveMethod[method]
        self.method = method
        self.adaptive = adaptive
        self.guess_dt = guess_dt
        self.adaptive_rtol = adaptive_rtol
        self.ivp_rtol = ivp_rtol
        self.ivp_atol = ivp_atol
        self.ivp_solver = ivp_solver
        # engine extension: run every local exponential with exactly this
        # many Krylov vectors (no data-dependent exit), used for graph capture
        self.fixed_krylov = fixed_krylov
        self.stat = None

    @property
    def is_tdvp(self):
        return self.method not in (EvolveMethod.prop_and_compress, EvolveMethod.prop_and_compress_tdrk4,
                                   EvolveMethod.prop_and_compress_tdrk)

    def copy(self):
        new = self.__class__.__new__(self.__class__)
        new.__dict__ = self.__dict__.copy()
        return new
