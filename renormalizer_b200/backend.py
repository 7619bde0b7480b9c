"""Device, dtype and arithmetic policy of the B200 sweep engine.

Mirrors renormalizer/mps/backend.py:97-216 (the ``Backend`` singleton: real
and complex dtypes, canonical tolerances) and adds the engine's contraction
arithmetic:

* ``"fp64"``   -- FP64 tensor-core (DMMA) contractions, the plain engine;
* ``"bf16x3"`` -- BF16 hi/lo operand split, three products, FP32 accumulate;
* ``"tf32x3"`` -- TF32 hi/lo operand split, three products, FP32 accumulate.

Krylov / Davidson orthogonalisation, the small tridiagonal and projected
eigenproblems, SVD/QR and all norms and energies stay FP64 in every mode.
"""
from __future__ import annotations

import os

import numpy as np
import torch

PRECISIONS = ("fp64", "bf16x3", "tf32x3")


class Backend:
    def __init__(self):
        self.real_dtype = torch.float64
        self.complex_dtype = torch.complex128
        self._prec = os.environ.get("RENO_PREC", "fp64")
        if self._prec not in PRECISIONS:
            raise ValueError(f"RENO_PREC must be one of {PRECISIONS}")
        gpu = os.environ.get("RENO_GPU")
        self._device_index = int(gpu) if gpu is not None else None
        self.canonical_atol = 1e-8
        self.canonical_rtol = 1e-5

    @property
    def device(self) -> torch.device:
        if not torch.cuda.is_available():
            raise RuntimeError("renormalizer_b200 needs a CUDA device (B200, sm_100a); none is visible")
        idx = self._device_index if self._device_index is not None else torch.cuda.current_device()
        return torch.device("cuda", idx)

    @property
    def prec(self) -> str:
        return self._prec

    @prec.setter
    def prec(self, v: str):
        if v not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}, got {v}")
        self._prec = v

    def sync(self):
        torch.cuda.synchronize(self.device)


backend = Backend()

# global seeds (backend.py:68-74): the engine's own random choices (random MPS,
# orthonormal padding) draw from numpy's global RNG like the reference
np.random.seed(9012)
