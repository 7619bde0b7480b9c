"""Lockstep evolution of independent MPS (evolve_batch, grouped matvecs).

Static-disorder realisations of a Holstein chain (three molecules, per-site
couplings drawn per realisation, different random bond expansions) evolved
together must give, step by step, the states each realisation gets from its
own Mps.evolve, for TDVP-PS2 and TDVP-PS: overlap 1 to 1e-12 and site
populations to 1e-12.  (Entry-wise equality is not expected: zero-weight
completion columns of the truncation are drawn from numpy's global RNG, as in
the reference, and lockstep runs draw them in a different order.)  The grouped
matvec must equal the single one bit for bit on ragged shapes with 0, 1 and 2
active sites."""
import numpy as np
import pytest
import torch


def _realisation(seed, method, nlev=4, M=8):
    from renormalizer_b200 import (CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, HolsteinModel, Mol,
                                   Mpo, Mps, Phonon, Quantity)
    g = np.random.default_rng(seed).uniform(0.5, 1.5, 3)
    mols = [Mol(Quantity(0), [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0) * gi), nlev)]) for gi in g]
    model = HolsteinModel(mols, Quantity(1.0), 3)
    np.random.seed(100 + seed)
    mps = Mps.hartree_product_state(model, {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=M)
    mps = mps.expand_bond_dimension()
    mps.evolve_config = EvolveConfig(method)
    return mps, Mpo(model)


def _run(method_name, steps=2, atol=1e-12):
    from renormalizer_b200 import EvolveMethod, evolve_batch
    method = getattr(EvolveMethod, method_name)
    cases = [_realisation(s, method) for s in range(3)]
    single = []
    for mps, mpo in cases:
        m = mps
        traj = []
        for _ in range(steps):
            m = m.evolve(mpo, 0.05)
            traj.append(m)
        single.append(traj)
    batch = [mps for mps, _ in cases]
    for step in range(steps):
        batch = evolve_batch(batch, [mpo for _, mpo in cases], 0.05)
        for i, m in enumerate(batch):
            ref = single[i][step]
            assert m.bond_dims == ref.bond_dims
            ov = complex(m.conj().dot(ref)) / np.sqrt(abs(complex(m.conj().dot(m))) * abs(complex(ref.conj().dot(ref))))
            assert abs(abs(ov) - 1.0) < atol, (method_name, step, i, ov)
            np.testing.assert_allclose(m.e_occupations, ref.e_occupations, rtol=0, atol=atol)


@pytest.mark.parametrize("method", ["tdvp_ps2", "tdvp_ps"])
def test_evolve_batch_host_logic(cpu_engine, method):
    _run(method)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["tdvp_ps2", "tdvp_ps"])
def test_evolve_batch_gpu(method):
    from renormalizer_b200 import backend
    backend.prec = "fp64"
    _run(method)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_evolve_batch_split_gpu(prec):
    """lockstep TDVP-PS2 in split precision (each problem's fused split chain,
    batched truncations and QRs) against each realisation's own evolve in the
    same precision.  Tolerance 1e-9: the batched eigensolver rounds the
    truncation differently from a single call, and the split operands of the
    next matvec can round to the other side of a BF16 / TF32 boundary."""
    from renormalizer_b200 import backend
    saved = backend.prec
    backend.prec = prec
    try:
        _run("tdvp_ps2", atol=1e-9)
    finally:
        backend.prec = saved


@pytest.mark.gpu
def test_grouped_matvec_matches_single():
    from renormalizer_b200.hop_expr import HeffOperator, apply_grouped
    g = torch.Generator(device="cuda").manual_seed(11)
    r = lambda *s: torch.randn(s, dtype=torch.float64, device="cuda", generator=g)
    c = lambda *s: torch.complex(r(*s), r(*s))
    for nsite in (0, 1, 2):
        ops, psis = [], []
        for ml, mr, wl, wm, wr, d1, d2 in ((5, 7, 3, 2, 3, 2, 3), (40, 33, 5, 4, 5, 4, 2), (70, 64, 4, 3, 4, 3, 3)):
            if nsite == 0:
                wr = wl
            W = [] if nsite == 0 else ([r(wl, d1, d1, wr)] if nsite == 1 else [r(wl, d1, d1, wm), r(wm, d2, d2, wr)])
            shape = {0: (ml, mr), 1: (ml, d1, mr), 2: (ml, d1, d2, mr)}[nsite]
            ops.append(HeffOperator(c(ml, wl, ml), c(mr, wr, mr), W, shape, prec="fp64"))
            psis.append(c(*shape))
        ys = apply_grouped(ops, psis)
        for op, psi, y in zip(ops, psis, ys):
            assert torch.equal(y, op.apply(psi)), nsite


def test_expm_krylov_batch_matches_single(cpu_engine):
    """lockstep Lanczos exponentials of independent problems (different sizes,
    step sizes and stopping points) equal their own expm_krylov results
    exactly, and the grouped operator sees only the still-running problems"""
    from renormalizer_b200.krylov import expm_krylov, expm_krylov_batch
    rng = np.random.default_rng(8)
    mats, vecs, dts = [], [], []
    for n, dt in ((6, -0.3j), (40, -0.05j), (25, 0.2), (3, -1j)):
        h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        mats.append(torch.as_tensor(h + h.conj().T))
        vecs.append(torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n)))
        dts.append(dt)
    # a start vector inside a 3-dimensional invariant subspace: the Lanczos
    # iteration breaks down (beta_2 ~ 0) and stops at the next check point
    d = np.arange(1.0, 31.0)
    mats.append(torch.as_tensor(np.diag(d).astype(complex)))
    v = np.zeros(30, dtype=complex)
    v[[3, 11, 20]] = (1.0, 0.5j, -0.25)
    vecs.append(torch.as_tensor(v))
    dts.append(-0.1j)
    issued = [0] * len(mats)

    def counted(i, x):
        issued[i] += 1
        return mats[i] @ x

    single = [expm_krylov(lambda x, i=i: counted(i, x), dt, v) for i, (dt, v) in enumerate(zip(dts, vecs))]
    assert single[-1][1] == 3
    seen = []

    def group_apply(idx, xs):
        seen.append(list(idx))
        return [mats[i] @ x for i, x in zip(idx, xs)]

    batch = expm_krylov_batch(group_apply, dts, vecs)
    for (vs, js), (vb, jb) in zip(single, batch):
        assert js == jb
        assert torch.equal(vs, vb)
    assert seen[0] == [0, 1, 2, 3, 4]
    assert all(len(a) >= len(b) for a, b in zip(seen, seen[1:]))
    # every problem gets exactly the matvecs its own expm_krylov asks for
    assert [sum(i in s for s in seen) for i in range(len(mats))] == issued


def test_apply_grouped_dispatch_host_logic(cpu_engine, monkeypatch):
    """apply_grouped on the CPU stand-in: FP64 operators (two shapes, 0/1/2
    sites) go to grouped calls of at most 128 problems with one nsite and
    dtype set each, split-precision operators one by one; every result equals
    the operator's own apply"""
    import importlib
    hop_expr = importlib.import_module("renormalizer_b200.hop_expr")
    from renormalizer_b200.hop_expr import HeffOperator, apply_grouped
    rng = np.random.default_rng(2)
    c = lambda *s: torch.as_tensor(rng.standard_normal(s) + 1j * rng.standard_normal(s))
    r = lambda *s: torch.as_tensor(rng.standard_normal(s))
    ops, psis = [], []
    for i in range(133):
        nsite = i % 3
        ml, mr, w, d1, d2 = (3, 4, 2, 2, 2) if i % 2 else (5, 2, 3, 3, 2)
        W = [] if nsite == 0 else ([r(w, d1, d1, w)] if nsite == 1 else [r(w, d1, d1, w), r(w, d2, d2, w)])
        shape = {0: (ml, mr), 1: (ml, d1, mr), 2: (ml, d1, d2, mr)}[nsite]
        prec = "bf16x3" if i % 7 == 0 else "fp64"
        ops.append(HeffOperator(c(ml, w, ml), c(mr, w, mr), W, shape, prec=prec))
        psis.append(c(*shape))
    calls = []
    fake = cpu_engine
    orig = type(fake).heff_apply_grouped

    def spy(self, descs, *rest):
        calls.append([(d.nsite, d.prec) for d in descs])
        return orig(self, descs, *rest)

    monkeypatch.setattr(type(fake), "heff_apply_grouped", spy)
    monkeypatch.setattr(hop_expr, "MAX_GROUP", 20)
    ys = apply_grouped(ops, psis)
    for op, psi, y in zip(ops, psis, ys):
        assert torch.equal(y, op.apply(psi))
    assert all(len(cl) <= 20 for cl in calls)
    assert all(len({ns for ns, _ in cl}) == 1 and all(p == 0 for _, p in cl) for cl in calls)
    assert sum(len(cl) for cl in calls) == sum(1 for op in ops if op.prec == "fp64")


@pytest.mark.parametrize("method", ["tdvp_ps2", "tdvp_ps"])
def test_evolve_batch_per_instance_precision_host_logic(cpu_engine, monkeypatch, method):
    """evolve_batch(precs=...) builds every local operator of an instance in
    that instance's precision (realisations told apart by their phonon
    dimension, 4 and 3) and leaves the backend's precision as it was"""
    import importlib
    from renormalizer_b200 import EvolveMethod, backend, evolve_batch
    hop_expr = importlib.import_module("renormalizer_b200.hop_expr")
    seen = []
    orig = hop_expr.HeffOperator.__init__

    def spy(self, *a, **k):
        orig(self, *a, **k)
        seen.append((tuple(self.cshape[1:-1]), self.prec))

    monkeypatch.setattr(hop_expr.HeffOperator, "__init__", spy)
    m = getattr(EvolveMethod, method)
    (a, mpo_a), (b, mpo_b) = _realisation(0, m, nlev=4), _realisation(1, m, nlev=3)
    backend.prec = "fp64"
    evolve_batch([a, b], [mpo_a, mpo_b], 0.05, precs=["bf16x3", "fp64"])
    assert backend.prec == "fp64"
    by_a = [p for d, p in seen if 4 in d]
    by_b = [p for d, p in seen if 3 in d]
    assert by_a and by_b
    assert set(by_a) == {"bf16x3"} and set(by_b) == {"fp64"}


@pytest.mark.gpu
def test_grouped_vector_ops_match_single():
    """reno_vec_grouped gives every item bitwise the result of the single
    vector call: ragged lengths across the block partition (1 .. 3 x 1184
    blocks), real and complex, every operation."""
    from renormalizer_b200._native import (Engine, VOP_ALLCLOSE, VOP_ALPHA, VOP_LINCOMB, VOP_NORM, VOP_ORTH,
                                           VOP_SCALE_INV, dtype_code)
    eng = Engine.get(0)
    g = torch.Generator(device="cuda").manual_seed(5)
    sizes = (1, 7, 256, 1025, 300_001, 3_700_000)
    vecs = []
    for i, n in enumerate(sizes):
        dt = torch.complex128 if i % 2 else torch.float64
        mk = (lambda: torch.randn(n, dtype=torch.float64, device="cuda", generator=g)) if dt == torch.float64 else \
            (lambda: torch.complex(torch.randn(n, dtype=torch.float64, device="cuda", generator=g),
                                   torch.randn(n, dtype=torch.float64, device="cuda", generator=g)))
        V = torch.stack([mk() for _ in range(4)])
        vecs.append((n, dt, V, mk()))
    j = 2
    single_ab, group_ab = [], []
    single_w, group_w = [], []
    for n, dt, V, w in vecs:
        ab_s = torch.zeros(8, dtype=torch.float64, device="cuda")
        ab_s[2 * j - 1] = 0.37
        ab_g = ab_s.clone()
        ws, wg = w.clone(), w.clone()
        eng.krylov_alpha(ws, V[j], ab_s, j)
        eng.krylov_orth(ws, V[j], V[j - 1], ab_s, j)
        single_ab.append(ab_s), group_ab.append(ab_g), single_w.append(ws), group_w.append(wg)
    items = lambda rows: [(n, dtype_code(V), jj, x, y, out, sc, s, n) for (n, dt, V, w), (jj, x, y, out, sc, s)
                          in zip(vecs, rows)]
    eng.vec_grouped(VOP_ALPHA, items([(j, wg, V[j], None, ab, None)
                                      for (n, dt, V, w), wg, ab in zip(vecs, group_w, group_ab)]))
    eng.vec_grouped(VOP_ORTH, items([(j, V[j], V[j - 1], wg, ab, None)
                                     for (n, dt, V, w), wg, ab in zip(vecs, group_w, group_ab)]))
    for a, b in zip(single_ab, group_ab):
        assert torch.equal(a, b)
    for a, b in zip(single_w, group_w):
        assert torch.equal(a, b)
    # norm, scale_inv, lincomb, allclose
    s_norm = [torch.zeros(4, dtype=torch.float64, device="cuda") for _ in vecs]
    g_norm = [torch.zeros(4, dtype=torch.float64, device="cuda") for _ in vecs]
    for (n, dt, V, w), o in zip(vecs, s_norm):
        eng.vec_norm(V[1], o)
    eng.vec_grouped(VOP_NORM, items([(0, V[1], None, None, o, None) for (n, dt, V, w), o in zip(vecs, g_norm)]))
    assert all(torch.equal(a, b) for a, b in zip(s_norm, g_norm))
    s_sc = [torch.empty_like(w) for _, _, _, w in vecs]
    g_sc = [torch.empty_like(w) for _, _, _, w in vecs]
    for (n, dt, V, w), o, nr in zip(vecs, s_sc, s_norm):
        eng.scale_inv(V[1], nr, o)
    eng.vec_grouped(VOP_SCALE_INV, items([(0, V[1], None, o, None, nr)
                                          for (n, dt, V, w), o, nr in zip(vecs, g_sc, g_norm)]))
    assert all(torch.equal(a, b) for a, b in zip(s_sc, g_sc))
    coef = torch.randn(8, dtype=torch.float64, device="cuda", generator=g)
    s_lc = [torch.empty_like(w) for _, _, _, w in vecs]
    g_lc = [torch.empty_like(w) for _, _, _, w in vecs]
    for (n, dt, V, w), o in zip(vecs, s_lc):
        eng.lincomb(V, 3, coef, o)
    eng.vec_grouped(VOP_LINCOMB, items([(3, V, None, o, None, coef) for (n, dt, V, w), o in zip(vecs, g_lc)]))
    assert all(torch.equal(a, b) for a, b in zip(s_lc, g_lc))
    s_fl = [torch.full((4,), -1.0, dtype=torch.float64, device="cuda") for _ in vecs]
    g_fl = [torch.full((4,), -1.0, dtype=torch.float64, device="cuda") for _ in vecs]
    pert = [w * (1 + 1e-7 * (i % 2)) for i, (_, _, _, w) in enumerate(vecs)]
    for (n, dt, V, w), p, o in zip(vecs, pert, s_fl):
        eng.allclose(w, p, 1e-9, 0.0, o)
    eng.vec_grouped(VOP_ALLCLOSE, items([(0, w, p, None, o, None) for (n, dt, V, w), p, o in zip(vecs, pert, g_fl)]),
                    1e-9, 0.0)
    assert all(torch.equal(a, b) for a, b in zip(s_fl, g_fl))
    assert [float(f[0]) for f in g_fl] == [1.0, 0.0] * 3


@pytest.mark.gpu
def test_expm_krylov_batch_matches_single_gpu():
    """the grouped lockstep Lanczos exponential equals each problem's own
    expm_krylov bit for bit on the GPU (sizes from 3 to 4000, real and
    imaginary steps, early and late convergence)"""
    from renormalizer_b200.krylov import expm_krylov, expm_krylov_batch
    rng = np.random.default_rng(3)
    mats, vecs, dts = [], [], []
    for n, dt in ((3, -1j), (6, -0.3j), (40, -0.05j), (25, 0.2), (700, -0.02j), (4000, -0.01j)):
        h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        mats.append(torch.as_tensor((h + h.conj().T) / np.sqrt(n), device="cuda"))
        vecs.append(torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n), device="cuda"))
        dts.append(dt)
    single = [expm_krylov(lambda x, m=m: m @ x, dt, v) for m, dt, v in zip(mats, dts, vecs)]
    batch = expm_krylov_batch(lambda idx, xs: [mats[i] @ x for i, x in zip(idx, xs)], dts, vecs)
    for (vs, js), (vb, jb) in zip(single, batch):
        assert js == jb
        assert torch.equal(vs, vb)


def test_qr_split_batch_matches_single(cpu_engine):
    """the batched canonicalising QR (the QN blocks of several calls in shared
    reno_qr_blocks launches) returns every call's own qr_split result, for
    QR and RQ, real and complex, several QN sectors"""
    from renormalizer_b200.svd_qn import qr_split, qr_split_batch
    rng = np.random.default_rng(4)
    calls = []
    for rows, cols, cplx, system in ((12, 9, True, "L"), (7, 20, False, "R"), (16, 16, True, "R"), (5, 3, False, "L")):
        a = rng.standard_normal((rows, cols)) + (1j * rng.standard_normal((rows, cols)) if cplx else 0)
        ql = rng.integers(0, 3, rows).reshape(rows, 1)
        qr = (2 - rng.integers(0, 3, cols)).reshape(cols, 1)
        calls.append(dict(coef=torch.as_tensor(a), qnbigl=ql, qnbigr=qr, qntot=np.array([2]), system=system))
    single = [qr_split(**c) for c in calls]
    batch = qr_split_batch(calls)
    for (u1, l1, v1, r1), (u2, l2, v2, r2) in zip(single, batch):
        assert torch.equal(u1, u2) and torch.equal(v1, v2)
        assert l1 == l2 and r1 == r2
