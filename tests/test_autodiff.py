"""The hand-written H_eff backward (renormalizer_b200.autodiff) against torch
autograd through an FP64 einsum of the same contraction (hop_expr.py:57-103)
and against central finite differences.

Every gradient (psi, L, W1, W2, R; complex and real operands; 0, 1 and 2
active sites) must match the einsum reference to 1e-12 relative to its
largest entry (FP64 GEMMs on both sides); a directional derivative of the
real loss Re<c, y> must match central differences (h = 1e-6) to 1e-7."""
import numpy as np
import pytest
import torch

EINSUM = {0: "abc,lbk,ck->al", 1: "abc,bdef,lfk,cek->adl", 2: "abc,bdef,fghj,ljk,cehk->adgl"}


def _case(nsite, cplx, dev, seed=3):
    g = torch.Generator(device=dev).manual_seed(seed + nsite)
    r = lambda *s: torch.randn(s, dtype=torch.float64, device=dev, generator=g)
    c = lambda *s: torch.complex(r(*s), r(*s)) if cplx else r(*s)
    ml, mr, wl, wm, wr, d1, d2 = 5, 4, 3, 2, 3, 3, 2
    if nsite == 0:
        wr = wl
    L, R = c(ml, wl, ml), c(mr, wr, mr)
    Ws = [] if nsite == 0 else ([r(wl, d1, d1, wr)] if nsite == 1 else [r(wl, d1, d1, wm), r(wm, d2, d2, wr)])
    shape = {0: (ml, mr), 1: (ml, d1, mr), 2: (ml, d1, d2, mr)}[nsite]
    psi = c(*shape)
    return L, Ws, R, psi, c


def _reference_grads(L, Ws, R, psi, gy):
    ts = [t.detach().clone().cpu().requires_grad_(True) for t in [L] + Ws + [R, psi]]
    ops = [ts[0]] + ts[1:1 + len(Ws)] + [ts[-2], ts[-1]]
    dt = torch.complex128 if any(t.is_complex() for t in ts) else torch.float64
    y = torch.einsum(EINSUM[len(Ws)], *[t.to(dt) for t in ops])
    y.backward(gy.cpu().to(dt))
    return [t.grad for t in ts]


def _run(nsite, cplx, dev):
    from renormalizer_b200.autodiff import heff
    L, Ws, R, psi, c = _case(nsite, cplx, dev)
    leaves = [t.clone().requires_grad_(True) for t in [L] + Ws + [R, psi]]
    Lg, Wg, Rg, Pg = leaves[0], leaves[1:1 + len(Ws)], leaves[-2], leaves[-1]
    y = heff(Pg, Lg, Wg, Rg, prec="fp64")
    gy = c(*y.shape)
    y.backward(gy)
    ref = _reference_grads(L, Ws, R, psi, gy)
    for got, exp, name in zip([t.grad for t in leaves], ref, ["L"] + [f"W{i + 1}" for i in range(len(Ws))] + ["R", "psi"]):
        assert got is not None and got.shape == exp.shape and got.dtype == exp.dtype, name
        err = float((got.cpu() - exp).abs().max() / exp.abs().max())
        assert err < 1e-12, (name, err)
    # directional derivative of Re<cvec, y> against central differences
    cvec = c(*y.shape)
    dirs = [c(*t.shape) if t.is_complex() else torch.randn_like(t) for t in leaves]
    loss = lambda ts: torch.real(torch.sum(cvec.conj() * heff(ts[-1], ts[0], ts[1:1 + len(Ws)], ts[-2], prec="fp64")))
    for t in leaves:
        t.grad = None
    loss(leaves).backward()
    analytic = sum(float(torch.real(torch.sum(t.grad.conj() * dv))) for t, dv in zip(leaves, dirs))
    h = 1e-6
    with torch.no_grad():
        plus = loss([t.detach() + h * dv for t, dv in zip(leaves, dirs)])
        minus = loss([t.detach() - h * dv for t, dv in zip(leaves, dirs)])
    fd = float(plus - minus) / (2 * h)
    assert abs(fd - analytic) <= 1e-7 * max(1.0, abs(analytic)), (fd, analytic)


@pytest.mark.parametrize("nsite", [0, 1, 2])
@pytest.mark.parametrize("cplx", [True, False])
def test_heff_backward_host_logic(cpu_engine, nsite, cplx):
    _run(nsite, cplx, "cpu")


@pytest.mark.gpu
@pytest.mark.parametrize("nsite", [0, 1, 2])
@pytest.mark.parametrize("cplx", [True, False])
def test_heff_backward_gpu(nsite, cplx):
    _run(nsite, cplx, "cuda")
