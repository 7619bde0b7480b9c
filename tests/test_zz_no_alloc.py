"""The allocation-free matvec entry point, reno_heff_apply_noalloc.

Some callers of this library cannot allocate device memory: hosts that keep
the GPU's memory in their own pool and forbid outside code from calling
cudaMalloc, or foreign-language hosts that cannot keep a device allocation
alive between calls.  For them the library carries a fixed scratch array and
this entry point takes only inputs and outputs.  The test drives it through
the C ABI, twice in a row with different inputs (the array keeps the previous
call's contents), and requires the same result as reno_heff_apply with a
caller workspace, within the tolerance the other GPU tests use per
arithmetic.  It also checks that a problem too large for the array is
rejected with a clear message.  The file name sorts last so that a run which
stops at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "bf16x3": 2e-4}
PREC = {"fp64": 0, "bf16x3": 1}


def _setup():
    from renormalizer_b200._native import Engine, HeffDesc, load_library
    lib = load_library()
    eng = Engine.get(0)
    return lib, eng, HeffDesc


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _case(nsite, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    cx = lambda *s: torch.complex(torch.randn(s, dtype=torch.float64, device="cuda", generator=g),
                                  torch.randn(s, dtype=torch.float64, device="cuda", generator=g))
    ml, mr, w, d1, d2 = 24, 20, 5, 10, 2
    L, R = cx(ml, w, ml), cx(mr, w, mr)
    W1 = torch.randn(w, d1, d1, w, dtype=torch.float64, device="cuda", generator=g)
    W2 = torch.randn(w, d2, d2, w, dtype=torch.float64, device="cuda", generator=g) if nsite == 2 else None
    shape = (ml, d1, d2, mr) if nsite == 2 else (ml, d1, mr)
    return L, R, W1, W2, shape, cx


def _fill_scratch_with_other_layout(lib, eng, HeffDesc, nsite, prec):
    """One call of another shape and site count, so that the scratch array
    holds stale data laid out differently from the calls under test."""
    g = torch.Generator(device="cuda").manual_seed(99)
    cx = lambda *s: torch.complex(torch.randn(s, dtype=torch.float64, device="cuda", generator=g),
                                  torch.randn(s, dtype=torch.float64, device="cuda", generator=g))
    other = 2 if nsite == 1 else 1
    ml, mr, w, d1, d2 = 31, 13, 4, 6, 3
    L, R = cx(ml, w, ml), cx(mr, w, mr)
    W1 = torch.randn(w, d1, d1, w, dtype=torch.float64, device="cuda", generator=g)
    W2 = torch.randn(w, d2, d2, w, dtype=torch.float64, device="cuda", generator=g) if other == 2 else None
    shape = (ml, d1, d2, mr) if other == 2 else (ml, d1, mr)
    d = HeffDesc(nsite=other, ml=ml, mr=mr, wl=w, wm=w, wr=w, d1=d1, d2=d2 if other == 2 else 1, psi_dtype=1,
                 env_dtype=1, mpo_dtype=0, prec=PREC[prec])
    psi = cx(*shape)
    y = torch.empty_like(psi)
    st = lib.reno_heff_apply_noalloc(eng.ctx, ctypes.byref(d), _p(L), _p(W1), _p(W2), _p(R), _p(psi), _p(y))
    assert st == 0, lib.reno_last_error(eng.ctx)
    torch.cuda.synchronize()


@pytest.mark.parametrize("prec", ["fp64", "bf16x3"])
@pytest.mark.parametrize("nsite", [2, 1])
def test_noalloc_matches_workspace_entry_twice(nsite, prec):
    lib, eng, HeffDesc = _setup()
    _fill_scratch_with_other_layout(lib, eng, HeffDesc, nsite, prec)
    L, R, W1, W2, shape, cx = _case(nsite, 17 + nsite)
    d = HeffDesc(nsite=nsite, ml=shape[0], mr=shape[-1], wl=5, wm=5, wr=5, d1=shape[1],
                 d2=shape[2] if nsite == 2 else 1, psi_dtype=1, env_dtype=1, mpo_dtype=0, prec=PREC[prec])
    n = ctypes.c_size_t()
    assert lib.reno_heff_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    for call in range(2):
        psi = cx(*shape)
        y_ref = torch.empty_like(psi)
        y = torch.full_like(psi, float("nan"))
        st = lib.reno_heff_apply(eng.ctx, ctypes.byref(d), _p(L), _p(W1), _p(W2), _p(R), _p(psi), _p(y_ref),
                                 _p(ws), ctypes.c_size_t(n.value))
        assert st == 0, lib.reno_last_error(eng.ctx)
        st = lib.reno_heff_apply_noalloc(eng.ctx, ctypes.byref(d), _p(L), _p(W1), _p(W2), _p(R), _p(psi), _p(y))
        assert st == 0, lib.reno_last_error(eng.ctx)
        torch.cuda.synchronize()
        err = float((y - y_ref).abs().max() / y_ref.abs().max())
        assert err <= TOL[prec], (call, err)


def test_noalloc_rejects_problems_larger_than_its_scratch():
    lib, eng, HeffDesc = _setup()
    d = HeffDesc(nsite=2, ml=256, mr=256, wl=5, wm=5, wr=5, d1=16, d2=16, psi_dtype=1, env_dtype=1, mpo_dtype=0,
                 prec=0)
    dummy = torch.zeros(1, dtype=torch.complex128, device="cuda")
    st = lib.reno_heff_apply_noalloc(eng.ctx, ctypes.byref(d), _p(dummy), _p(dummy), _p(dummy), _p(dummy),
                                     _p(dummy), _p(dummy))
    assert st == 4  # RENO_ERR_WORKSPACE
    msg = lib.reno_last_error(eng.ctx).decode()
    assert "scratch" in msg and "reno_heff_apply" in msg
