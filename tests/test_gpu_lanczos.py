"""reno_lanczos_expm: the whole Lanczos exponential behind one C-ABI call.

krylov.py:27-84 (expm_krylov) with the matvec of hop_expr, driven from the
host in C++ so that a host without Python can run a local TDVP update.  The
reference's Krylov fixtures (tests/golden/krylov_cases.npz: a dense
Hermitian A, a start vector and dt, the result and the number of matvecs)
are run through the C ABI with A as a zero-site effective Hamiltonian
(L = A, R = 1, bond dimension 1 on the right), and a two-site H_eff case is
compared with the engine's own expm_krylov."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

KRY = load_golden("krylov_cases.npz")


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _expm_c(desc, L, W1, W2, R, psi, dt, kmax=60):
    from renormalizer_b200._native import Engine, load_library
    lib = load_library()
    eng = Engine.get(0)
    n = ctypes.c_size_t()
    assert lib.reno_lanczos_workspace_bytes(ctypes.byref(desc), kmax, ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    k = ctypes.c_int32(0)
    x = psi.clone()
    st = lib.reno_lanczos_expm(eng.ctx, ctypes.byref(desc), _p(L), _p(W1), _p(W2), _p(R), float(np.real(dt)),
                               float(np.imag(dt)), _p(x), kmax, ctypes.byref(k), _p(ws), n.value)
    assert st == 0, lib.reno_last_error(eng.ctx)
    torch.cuda.synchronize()
    return x, k.value


@pytest.mark.parametrize("case", range(int(KRY["count"])))
def test_lanczos_expm_matches_reference_fixtures(case):
    from renormalizer_b200._native import HeffDesc
    A = np.asarray(KRY[f"k{case}/A"], dtype=complex)
    v = np.asarray(KRY[f"k{case}/v"], dtype=complex)
    dt = complex(KRY[f"k{case}/dt"][()])
    m = A.shape[0]
    L = torch.from_numpy(A.reshape(m, 1, m).copy()).cuda()
    R = torch.ones((1, 1, 1), dtype=torch.complex128, device="cuda")
    psi = torch.from_numpy(v.reshape(m, 1).copy()).cuda()
    d = HeffDesc(nsite=0, ml=m, mr=1, wl=1, wm=1, wr=1, d1=1, d2=1, psi_dtype=1, env_dtype=1, mpo_dtype=0, prec=0)
    x, k = _expm_c(d, L, None, None, R, psi, dt)
    assert k == int(KRY[f"k{case}/n"])
    np.testing.assert_allclose(x.cpu().numpy().reshape(-1), KRY[f"k{case}/res"], rtol=1e-10, atol=1e-12)


def test_lanczos_expm_matches_engine_driver_on_two_site_heff():
    from renormalizer_b200._native import HeffDesc
    from renormalizer_b200.hop_expr import HeffOperator
    from renormalizer_b200.krylov import expm_krylov
    g = torch.Generator(device="cuda").manual_seed(11)
    cx = lambda *s: torch.complex(torch.randn(s, dtype=torch.float64, device="cuda", generator=g),
                                  torch.randn(s, dtype=torch.float64, device="cuda", generator=g))
    ml, mr, d1, d2, wl, wm, wr = 24, 20, 4, 3, 3, 4, 2
    L, R = cx(ml, wl, ml), cx(mr, wr, mr)
    L, R = (L + L.transpose(0, 2).conj()) / 2, (R + R.transpose(0, 2).conj()) / 2
    W1 = torch.randn(wl, d1, d1, wm, dtype=torch.float64, device="cuda", generator=g)
    W2 = torch.randn(wm, d2, d2, wr, dtype=torch.float64, device="cuda", generator=g)
    W1, W2 = (W1 + W1.transpose(1, 2)) / 2, (W2 + W2.transpose(1, 2)) / 2
    psi = cx(ml, d1, d2, mr)
    psi = psi / torch.linalg.vector_norm(psi)
    dt = -0.025j
    op = HeffOperator(L, R, [W1, W2], list(psi.shape), prec="fp64")
    ref, kref = expm_krylov(lambda y: op.apply(y), dt, psi.reshape(-1))
    d = HeffDesc(nsite=2, ml=ml, mr=mr, wl=wl, wm=wm, wr=wr, d1=d1, d2=d2, psi_dtype=1, env_dtype=1, mpo_dtype=0,
                 prec=0)
    x, k = _expm_c(d, L, W1.contiguous(), W2.contiguous(), R, psi, dt)
    assert k == kref
    assert float((x.reshape(-1) - ref).abs().max()) < 1e-12


def test_lanczos_expm_reports_kmax_exceeded():
    from renormalizer_b200._native import HeffDesc, RENO_ERR_WORKSPACE, Engine, load_library
    lib = load_library()
    eng = Engine.get(0)
    m = 40
    g = torch.Generator(device="cuda").manual_seed(2)
    A = torch.randn(m, m, dtype=torch.float64, device="cuda", generator=g)
    A = ((A + A.T) * 10).to(torch.complex128)
    L = A.reshape(m, 1, m).contiguous()
    R = torch.ones((1, 1, 1), dtype=torch.complex128, device="cuda")
    psi = torch.ones((m, 1), dtype=torch.complex128, device="cuda")
    d = HeffDesc(nsite=0, ml=m, mr=1, wl=1, wm=1, wr=1, d1=1, d2=1, psi_dtype=1, env_dtype=1, mpo_dtype=0, prec=0)
    n = ctypes.c_size_t()
    assert lib.reno_lanczos_workspace_bytes(ctypes.byref(d), 6, ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    k = ctypes.c_int32(0)
    st = lib.reno_lanczos_expm(eng.ctx, ctypes.byref(d), _p(L), None, None, _p(R), 0.0, -1.0, _p(psi), 6,
                               ctypes.byref(k), _p(ws), n.value)
    assert st == RENO_ERR_WORKSPACE
    assert b"kmax" in lib.reno_last_error(eng.ctx)
