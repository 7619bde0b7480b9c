import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


def load_golden(name):
    return np.load(GOLDEN / name, allow_pickle=False)


def golden_cases(npz, prefix_filter=None):
    names = sorted({k.split("/")[0] for k in npz.files if "/" in k})
    if prefix_filter:
        names = [n for n in names if n.startswith(prefix_filter)]
    return names


def mps_from_golden(d, prefix, compress=None):
    """Build the oracle's MPS container from a dumped reference MPS."""
    from oracle.reno_oracle import OMps
    n = int(d[f"{prefix}/nsites"])
    sites = [d[f"{prefix}/mt_{i}"] for i in range(n)]
    qn = [d[f"{prefix}/qn_{i}"] for i in range(n + 1)]
    sig = [d[f"{prefix}/sigmaqn_{i}"] for i in range(n)]
    return OMps(sites, qn, int(d[f"{prefix}/qnidx"]), d[f"{prefix}/qntot"], bool(d[f"{prefix}/to_right"]), sig,
                compress=compress)


def mpo_from_golden(d, prefix, n):
    return [d[f"{prefix}/W_{i}"] for i in range(n)]


def engine_chain(d, tag, mps_key="init", mpo_key="mpo"):
    """The engine's Mps / Mpo from a dumped reference chain ``{tag}/{mps_key}``
    and ``{tag}/{mpo_key}`` (None: no Mpo): a model with the same local
    dimensions and QNs (electron sites carry QN (0, 1), the others QN 0) and
    the dumped tensors."""
    from renormalizer_b200 import Mpo, Mps
    from renormalizer_b200.model import BasisSHO, BasisSimpleElectron, Model
    pre = f"{tag}/{mps_key}"
    n = int(d[f"{pre}/nsites"])
    basis = []
    ie = 0
    for i in range(n):
        sq = d[f"{pre}/sigmaqn_{i}"]
        if sq.shape[0] == 2 and sq[1, 0] == 1:
            basis.append(BasisSimpleElectron(ie))
            ie += 1
        else:
            basis.append(BasisSHO(("ph", i), 1.0, int(sq.shape[0])))
    model = Model(basis, [])
    sites = [d[f"{pre}/mt_{i}"] for i in range(n)]
    qn = [d[f"{pre}/qn_{i}"] for i in range(n + 1)]
    mps = Mps.from_arrays(model, sites, qn, int(d[f"{pre}/qnidx"]), d[f"{pre}/qntot"], bool(d[f"{pre}/to_right"]))
    mpo = Mpo.from_tensors(model, [d[f"{tag}/{mpo_key}/W_{i}"] for i in range(n)]) if mpo_key else None
    return mps, mpo


@pytest.fixture
def cpu_engine(monkeypatch):
    """Run the engine's host logic on the CPU stand-in (tests/fake_engine.py)."""
    import torch
    from fake_engine import FakeEngine
    from renormalizer_b200 import _native
    from renormalizer_b200.backend import Backend
    fake = FakeEngine()
    monkeypatch.setattr(_native.Engine, "get", classmethod(lambda cls, device=None: fake))
    monkeypatch.setattr(Backend, "device", property(lambda self: torch.device("cpu")))
    return fake
