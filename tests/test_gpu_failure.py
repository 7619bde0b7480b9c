"""Failure detection on the device: bounded waits that run out.

The tensor-core GEMM and the eigensolver's grid-synchronised reduction wait
on barriers that other threads of the GPU complete.  Every such wait has a
wall-clock limit; when one runs out the kernel records where, skips its
remaining work, drains its own copies and frees its tensor memory, so that
the context stays usable.  These tests make one wait run out on purpose with
the library's test hook (reno_test_skip_arrival: CTA 0 of the next launch
leaves one arrival out -- nothing faults), under a 50 ms limit, and check the
reported status, the host-side reaction (the truncation redoes the block with
cuSOLVER) and that the next normal call is correct."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SPLIT_STAGE, HETRD_ARRIVAL = 1, 2


@pytest.fixture
def short_waits():
    from renormalizer_b200._native import load_library
    lib = load_library()
    assert lib.reno_set_wait_limit_ns(50_000_000) == 0
    yield lib
    lib.reno_test_skip_arrival(SPLIT_STAGE, -1)
    lib.reno_test_skip_arrival(HETRD_ARRIVAL, -1)
    assert lib.reno_set_wait_limit_ns(2_000_000_000) == 0


def _gemm_case():
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.complex(torch.randn(300, 700, dtype=torch.float64, device="cuda", generator=g),
                      torch.randn(300, 700, dtype=torch.float64, device="cuda", generator=g))
    B = torch.complex(torch.randn(700, 520, dtype=torch.float64, device="cuda", generator=g),
                      torch.randn(700, 520, dtype=torch.float64, device="cuda", generator=g))
    return A, B


def test_split_gemm_wait_runs_out_and_recovers(short_waits):
    from renormalizer_b200._native import Engine
    lib = short_waits
    eng = Engine.get(0)
    A, B = _gemm_case()
    ref = A @ B
    assert eng.device_error() == 0
    assert lib.reno_test_skip_arrival(SPLIT_STAGE, 0) == 0
    eng.matmul(A, B, prec="bf16x3")          # stage 0 of CTA 0 never lands
    torch.cuda.synchronize()
    code = eng.device_error()
    assert 1001 <= code <= 1009, code        # 1000 + the site whose wait ran out
    assert eng.device_error() == 0           # read clears it
    C = eng.matmul(A, B, prec="bf16x3")      # the context is intact
    torch.cuda.synchronize()
    assert eng.device_error() == 0
    assert float((C - ref).abs().max() / ref.abs().max()) < 2e-4


def _gram(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    X = torch.complex(torch.randn(n, n + 40, dtype=torch.float64, device="cuda", generator=g),
                      torch.randn(n, n + 40, dtype=torch.float64, device="cuda", generator=g))
    return X @ X.mH


def test_reduction_barrier_runs_out_and_recovers(short_waits):
    from renormalizer_b200._native import Engine
    from renormalizer_b200.heev import accepted, heev_top
    lib = short_waits
    eng = Engine.get(0)
    G = _gram(600, 1)                       # above 256: the grid-synchronised reduction
    assert lib.reno_test_skip_arrival(HETRD_ARRIVAL, 3) == 0
    _, _, chk = heev_top(eng, G, 64)
    chk = chk.cpu().numpy()
    assert chk[0] == 1.0 and not accepted(chk)
    w, K, chk = heev_top(eng, G, 64)        # next call: normal
    assert accepted(chk.cpu().numpy())
    ref = torch.flip(torch.linalg.eigvalsh(G), dims=[0])[:64]
    assert float((w - ref).abs().max() / ref.abs().max()) < 1e-13


def test_truncation_redoes_a_block_whose_reduction_timed_out(short_waits):
    """svd_truncate reads the eigensolver's status with the singular values;
    a block whose reduction timed out is redone by cuSOLVER and the result is
    the same as without the fault."""
    import importlib
    svd_qn = importlib.import_module("renormalizer_b200.svd_qn")
    heev = importlib.import_module("renormalizer_b200.heev")
    lib = short_waits
    g = torch.Generator(device="cuda").manual_seed(9)
    coef = torch.complex(torch.randn(700, 900, dtype=torch.float64, device="cuda", generator=g),
                         torch.randn(700, 900, dtype=torch.float64, device="cuda", generator=g))
    ql, qr = np.zeros((700, 1), dtype=int), np.zeros((900, 1), dtype=int)
    fn = lambda s: min(40, len(s))
    clean = svd_qn.svd_truncate(coef, ql, qr, np.array([0]), True, fn, kcap=40)
    f0 = heev.heev_opts.fallbacks
    assert lib.reno_test_skip_arrival(HETRD_ARRIVAL, 5) == 0
    got = svd_qn.svd_truncate(coef, ql, qr, np.array([0]), True, fn, kcap=40)
    assert heev.heev_opts.fallbacks == f0 + 1
    np.testing.assert_allclose(got.sigma, clean.sigma, rtol=1e-12)
    assert torch.allclose(got.left @ got.right, clean.left @ clean.right, atol=1e-12)
