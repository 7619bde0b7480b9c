"""C-ABI checks that need no GPU: the library loads, and it exports every
entry point that include/reno_b200.h declares (and the ctypes shim binds)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "reno_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(reno_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from renormalizer_b200 import build
    path = build.build_library()
    return ctypes.CDLL(str(path))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "reno_heff_apply" in syms and "reno_env_update" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_shim_binds_exactly_the_header(lib):
    from renormalizer_b200 import _native
    assert sorted(_native.exported_symbols()) == declared_symbols()
    _native.load_library()


def test_workspace_queries_without_gpu(lib):
    from renormalizer_b200._native import HeffDesc, EnvDesc, load_library
    L = load_library()
    d = HeffDesc(nsite=2, ml=256, mr=256, wl=5, wm=5, wr=5, d1=16, d2=16, psi_dtype=1, env_dtype=1, mpo_dtype=0,
                 prec=0)
    n = ctypes.c_size_t()
    assert L.reno_heff_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == 0
    # T1/T3 + T2 intermediates: 2 x (256*5*16*16*256) complex128 plus the MPO transposes
    assert n.value >= 2 * 256 * 5 * 256 * 256 * 16
    bad = HeffDesc(nsite=3)
    assert L.reno_heff_workspace_bytes(ctypes.byref(bad), ctypes.byref(n)) == 1
    e = EnvDesc(side=1, d=10, w_in=5, w_out=4, mk_in=32, mk_out=30, mb_in=32, mb_out=30, env_dtype=1, ket_dtype=1,
                bra_dtype=1, mpo_dtype=0, prec=0)
    assert L.reno_env_workspace_bytes(ctypes.byref(e), ctypes.byref(n)) == 0 and n.value > 0


def test_version_and_null_context(lib):
    from renormalizer_b200._native import load_library
    L = load_library()
    assert L.reno_version() >= 100
    assert L.reno_ctx_set_stream(None, None) == 1
    assert L.reno_last_error(None) == b"null context"


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from renormalizer_b200.hop_expr import hop_expr
    import numpy as np
    with pytest.raises(RuntimeError):
        hop_expr(np.ones((2, 1, 2)), np.ones((2, 1, 2)), [], (2, 2))(np.ones((2, 2)))
