"""B200-native sweep engine for Renormalizer's MPS hot path.

The effective-Hamiltonian matvec (hop_expr), the environment updates
(Environ / contract_one_site), the Lanczos exponential, the Davidson
eigensolver and the QN-blocked truncation of TDVP-PS / TDVP-PS2 time
evolution and DMRG run in hand-written sm_100a CUDA (libreno_b200.so) behind
the reference's own interface: Mps, Mpo, Model, Mps.evolve, optimize_mps,
Environ, hop_expr, expm_krylov, svd_qn.
"""
from .backend import backend
from .configs import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, OptimizeConfig
from .model import (BasisHalfSpin, BasisSHO, BasisSimpleElectron, HolsteinModel, Model, Mol, Op, Phonon, Quantity,
                    SpectralDensityFunction, SpinBosonModel)
from .mpo import Mpo
from .mps import Mps, compressed_sum, evolve_batch
from .lib import Environ, contract_one_site
from .hop_expr import hop_expr
from .krylov import expm_krylov
from .svd_qn import svd_qn
from .davidson import davidson
from .gs import optimize_mps
from .autodiff import heff as heff_autograd
from .tdmps import TdMpsJob
from .mpdm import MpDm
from .thermalprop import ThermalProp, load_thermal_state

__all__ = ["backend", "evolve_batch", "compressed_sum", "CompressConfig", "CompressCriteria", "EvolveConfig", "EvolveMethod", "OptimizeConfig",
           "BasisHalfSpin", "BasisSHO", "BasisSimpleElectron", "HolsteinModel", "Model", "Mol", "Op", "Phonon",
           "Quantity", "SpectralDensityFunction", "SpinBosonModel", "Mpo", "Mps", "Environ", "contract_one_site",
           "hop_expr", "expm_krylov", "svd_qn", "davidson", "optimize_mps", "heff_autograd", "TdMpsJob", "MpDm",
           "ThermalProp", "load_thermal_state"]
