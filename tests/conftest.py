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
