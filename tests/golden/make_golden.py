"""Generate the golden fixtures of the sweep hot path from the Renormalizer
reference itself.

Run in the build container (the reference is importable there, never on the
GPU machine):

    python tests/golden/make_golden.py  [--reference /root/reference]

The reference's missing third-party modules (opt_einsum 3.3, h5py) are
replaced by the stand-ins in oracle/_shims.  Output: tests/golden/*.npz.
Every case seeds numpy's global RNG first, so reruns reproduce the files.
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def _import_reference(path):
    sys.path.insert(0, str(REPO / "oracle" / "_shims"))
    sys.path.insert(0, str(path))
    import logging
    logging.disable(logging.WARNING)
    import renormalizer  # noqa: F401


def _rand(shape, cplx, rng):
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    return a


def gen_heff(out):
    from renormalizer.mps.hop_expr import hop_expr
    rng = np.random.default_rng(1234)
    cases = {}
    specs = [
        ("n0c", 0, True, dict(ml=5, mr=7, wl=3, wr=3)),
        ("n1c", 1, True, dict(ml=5, mr=7, wl=3, wr=2, d1=3)),
        ("n1r", 1, False, dict(ml=6, mr=4, wl=2, wr=3, d1=4)),
        ("n2c", 2, True, dict(ml=5, mr=7, wl=3, wm=4, wr=2, d1=3, d2=2)),
        ("n2r", 2, False, dict(ml=4, mr=6, wl=2, wm=3, wr=4, d1=2, d2=5)),
        ("n1c_big", 1, True, dict(ml=33, mr=17, wl=5, wr=4, d1=10)),
        ("n2c_big", 2, True, dict(ml=19, mr=23, wl=4, wm=5, wr=3, d1=6, d2=4)),
    ]
    for name, nsite, cplx, s in specs:
        L = _rand((s["ml"], s["wl"], s["ml"]), cplx, rng)
        R = _rand((s["mr"], s["wr"], s["mr"]), cplx, rng)
        Ws = []
        if nsite == 0:
            shape = (s["ml"], s["mr"])
        elif nsite == 1:
            Ws = [rng.standard_normal((s["wl"], s["d1"], s["d1"], s["wr"]))]
            shape = (s["ml"], s["d1"], s["mr"])
        else:
            Ws = [rng.standard_normal((s["wl"], s["d1"], s["d1"], s["wm"])),
                  rng.standard_normal((s["wm"], s["d2"], s["d2"], s["wr"]))]
            shape = (s["ml"], s["d1"], s["d2"], s["mr"])
        psi = _rand(shape, cplx, rng)
        expr = hop_expr(L, R, list(Ws), list(shape))
        y = expr(psi)
        cases[f"{name}/L"] = L
        cases[f"{name}/R"] = R
        for i, W in enumerate(Ws):
            cases[f"{name}/W{i + 1}"] = W
        cases[f"{name}/psi"] = psi
        cases[f"{name}/y"] = np.asarray(y)
        cases[f"{name}/nsite"] = np.array(nsite)
    np.savez_compressed(out / "heff_cases.npz", **cases)


def gen_env(out):
    from renormalizer.mps.lib import contract_one_site
    rng = np.random.default_rng(4321)
    cases = {}
    specs = [
        ("Lc", "L", True, False, dict(mi=5, mo=6, d=3, wi=3, wo=2)),
        ("Lr", "L", False, False, dict(mi=4, mo=7, d=2, wi=2, wo=4)),
        ("Rc", "R", True, False, dict(mi=5, mo=6, d=3, wi=3, wo=2)),
        ("Rr", "R", False, False, dict(mi=4, mo=7, d=2, wi=2, wo=4)),
        ("Lc_bra", "L", True, True, dict(mi=5, mo=6, d=3, wi=3, wo=2, bi=4, bo=3)),
        ("Rc_bra", "R", True, True, dict(mi=5, mo=6, d=3, wi=3, wo=2, bi=4, bo=3)),
        ("Lc_big", "L", True, False, dict(mi=37, mo=29, d=10, wi=5, wo=4)),
        ("Rc_big", "R", True, False, dict(mi=37, mo=29, d=10, wi=5, wo=4)),
    ]
    for name, dom, cplx, with_bra, s in specs:
        bi, bo = (s.get("bi", s["mi"]), s.get("bo", s["mo"]))
        if dom == "L":
            E = _rand((bi, s["wi"], s["mi"]), cplx, rng)
            ms = _rand((s["mi"], s["d"], s["mo"]), cplx, rng)
            W = rng.standard_normal((s["wi"], s["d"], s["d"], s["wo"]))
            bra = _rand((bi, s["d"], bo), cplx, rng) if with_bra else None
        else:
            E = _rand((bi, s["wi"], s["mi"]), cplx, rng)
            ms = _rand((s["mo"], s["d"], s["mi"]), cplx, rng)
            W = rng.standard_normal((s["wo"], s["d"], s["d"], s["wi"]))
            bra = _rand((bo, s["d"], bi), cplx, rng) if with_bra else None
        res = contract_one_site(E, ms, W, dom, ms_conj=bra)
        cases[f"{name}/E"] = E
        cases[f"{name}/ms"] = ms
        cases[f"{name}/W"] = W
        if bra is not None:
            cases[f"{name}/bra"] = bra
        cases[f"{name}/out"] = np.asarray(res)
        cases[f"{name}/domain"] = np.array(dom)
    np.savez_compressed(out / "env_cases.npz", **cases)


def gen_krylov(out):
    from renormalizer.lib import expm_krylov
    cases = {}
    k = 0
    for N in (1, 2, 4, 10, 60, 120):
        for imag in (False, True):
            for dt in (1.0, -0.5j, 0.3j):
                np.random.seed(100 + k)
                a = np.random.rand(N, N) / N
                if imag:
                    a = a + np.random.rand(N, N) / N / 1j
                a = a + a.T.conj()
                v = np.random.rand(N) + (np.random.rand(N) * 1j if imag or np.iscomplex(dt) else 0)
                res, j = expm_krylov(lambda x: a.dot(x), dt, v.copy())
                cases[f"k{k}/A"] = a
                cases[f"k{k}/v"] = v
                cases[f"k{k}/dt"] = np.array(dt)
                cases[f"k{k}/res"] = np.asarray(res)
                cases[f"k{k}/n"] = np.array(j)
                k += 1
    cases["count"] = np.array(k)
    np.savez_compressed(out / "krylov_cases.npz", **cases)


def gen_svd(out):
    from renormalizer.mps import svd_qn as S
    from renormalizer.mps.lib import select_basis
    cases = {}
    rng = np.random.default_rng(77)
    # 2-site coefficient (ml, d1, d2, mr) with one U(1) charge
    ml, d1, d2, mr = 6, 2, 3, 5
    qnl = rng.integers(0, 2, size=(ml, 1))
    sig1 = np.array([[0], [1]])
    sig2 = np.zeros((d2, 1), dtype=int)
    qnr = rng.integers(0, 2, size=(mr, 1))
    qntot = np.array([1])
    qnbigl = S.add_outer(qnl, sig1)
    qnbigr = S.add_outer(sig2, qnr)
    qnmat = S.add_outer(qnbigl, qnbigr)
    mask = S.get_qn_mask(qnmat, qntot)
    c = (rng.standard_normal((ml, d1, d2, mr)) + 1j * rng.standard_normal((ml, d1, d2, mr))) * mask
    for fm in (True, False):
        np.random.seed(5)
        u, su, qnl_new, v, sv, qnr_new = S.svd_qn(c, qnbigl, qnbigr, qntot, full_matrices=fm)
        tag = "full" if fm else "econ"
        cases[f"{tag}/su"] = su
        cases[f"{tag}/sv"] = sv
        cases[f"{tag}/qnl"] = np.array(qnl_new)
        cases[f"{tag}/qnr"] = np.array(qnr_new)
        cases[f"{tag}/ucols"] = np.array(u.shape[1])
        cases[f"{tag}/vcols"] = np.array(v.shape[1])
        if fm:
            ms, mdim, mqn, comp = select_basis(u, su, qnl_new, v, 7, percent=0)
            # gauge-invariant: ms @ comp^T reproduces the truncated coefficient
            cases["sel/recon"] = ms @ comp.T
            cases["sel/mdim"] = np.array(mdim)
            cases["sel/mqn"] = mqn
            ms2, mdim2, mqn2, comp2 = select_basis(u, su, qnl_new, v, 7, percent=0.4)
            cases["sel40/recon"] = ms2 @ comp2.T
            cases["sel40/mqn"] = mqn2
    for system in ("L", "R"):
        u, qnl_new, v, qnr_new = S.svd_qn(c, qnbigl, qnbigr, qntot, QR=True, system=system, full_matrices=False)
        cases[f"qr{system}/recon"] = u @ v.T
        cases[f"qr{system}/qnl"] = np.array(qnl_new)
        cases[f"qr{system}/qnr"] = np.array(qnr_new)
    cases["c"] = c
    cases["qnbigl"] = qnbigl
    cases["qnbigr"] = qnbigr
    cases["qntot"] = qntot
    np.savez_compressed(out / "svd_cases.npz", **cases)


def _dense_from_mpo(Ws):
    t = Ws[0]
    for W in Ws[1:]:
        t = np.tensordot(t, W, axes=([-1], [0]))
    t = t[0, ..., 0]
    n = len(Ws)
    perm = [2 * i for i in range(n)] + [2 * i + 1 for i in range(n)]
    t = t.transpose(perm)
    dim = int(np.prod(t.shape[:n]))
    return t.reshape(dim, dim)


def _holstein(nmol, nph_levels, modes, J=1.0):
    from renormalizer.model import Phonon, Mol, HolsteinModel
    from renormalizer.utils import Quantity
    ph_list = [Phonon.simple_phonon(Quantity(w), Quantity(np.sqrt(2.0) * g / np.sqrt(w)), nph_levels)
               for (w, g) in modes]
    return HolsteinModel([Mol(Quantity(0), ph_list)] * nmol, Quantity(J), 3)


def _sbm(nmodes, nlevels, alpha=0.5, omega_c=10.0, delta=1.0, eps=0.0):
    from renormalizer.model import SpinBosonModel, Phonon
    from renormalizer.sbm import SpectralDensityFunction
    from renormalizer.utils import Quantity
    sdf = SpectralDensityFunction(alpha, Quantity(omega_c))
    w, c2 = sdf.Wang1(nmodes)
    c = np.sqrt(c2)
    ph_list = [Phonon.simple_phonon(Quantity(wi), Quantity(ci / wi ** 2), nlevels) for wi, ci in zip(w, c)]
    return SpinBosonModel(Quantity(eps), Quantity(delta), ph_list), w, c


def gen_mpo(out):
    from renormalizer.mps import Mpo
    from renormalizer.utils import Quantity
    cases = {}
    models = {
        "hol3x2": _holstein(3, 2, [(1.0, 1.0 / np.sqrt(2.0))]),
        "hol4x3": _holstein(4, 3, [(1.0, 1.0)]),
        "hol2m2x3": _holstein(2, 3, [(1.0, 1.0), (0.5, 0.7)]),
    }
    sbm, w, c = _sbm(3, 3)
    models["sbm3x3"] = sbm
    cases["sbm3x3/omega"] = w
    cases["sbm3x3/c"] = c
    for name, model in models.items():
        mpo = Mpo(model)
        Ws = [np.asarray(m.array) for m in mpo]
        cases[f"{name}/H"] = _dense_from_mpo(Ws)
        off = Mpo(model, offset=Quantity(0.37))
        cases[f"{name}/H_off"] = _dense_from_mpo([np.asarray(m.array) for m in off])
        cases[f"{name}/pdims"] = np.array(model.pbond_list)
    np.savez_compressed(out / "mpo_cases.npz", **cases)


def _dump_mps(prefix, mps, d):
    d[f"{prefix}/nsites"] = np.array(len(mps))
    for i in range(len(mps)):
        d[f"{prefix}/mt_{i}"] = np.asarray(mps[i].array)
        d[f"{prefix}/sigmaqn_{i}"] = np.asarray(mps.model.basis[i].sigmaqn)
    for i in range(len(mps) + 1):
        d[f"{prefix}/qn_{i}"] = np.asarray(mps.qn[i]).reshape(len(mps.qn[i]), -1)
    d[f"{prefix}/qnidx"] = np.array(mps.qnidx)
    d[f"{prefix}/qntot"] = np.asarray(mps.qntot)
    d[f"{prefix}/to_right"] = np.array(mps.to_right)


def _dump_mpo(prefix, mpo, d):
    for i in range(len(mpo)):
        d[f"{prefix}/W_{i}"] = np.asarray(mpo[i].array)


def gen_tdvp(out):
    from renormalizer.mps import Mps, Mpo
    from renormalizer.utils import EvolveConfig, EvolveMethod, CompressConfig, CompressCriteria, Quantity
    cases = {}

    def run(tag, model, method, dt, nsteps, mmax, init_kind):
        np.random.seed(2024)
        tentative = Mpo(model)
        if init_kind == "exact3":
            init = Mpo.onsite(model, r"a^\dagger", dof_set={0}) @ Mps.ground_state(model, False)
            init = init.expand_bond_dimension(hint_mpo=tentative)
            e = init.expectation(tentative)
            mpo = Mpo(model, offset=Quantity(e))
        else:
            init = Mps.hartree_product_state(model, {0: 1})
            init.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=mmax)
            init = init.expand_bond_dimension(tentative, include_ex=False)
            mpo = tentative
        mps = init.copy()
        mps.evolve_config = EvolveConfig(method)
        if method == EvolveMethod.tdvp_ps2:
            mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=mmax)
        _dump_mps(f"{tag}/init", mps, cases)
        _dump_mpo(f"{tag}/mpo", mpo, cases)
        pops = [np.asarray(mps.e_occupations)]
        energies = [mps.expectation(mpo)]
        for _ in range(nsteps):
            mps = mps.evolve(mpo, dt)
            pops.append(np.asarray(mps.e_occupations))
            energies.append(mps.expectation(mpo))
        cases[f"{tag}/pops"] = np.array(pops)
        cases[f"{tag}/energy"] = np.array(energies)
        cases[f"{tag}/dt"] = np.array(dt)
        cases[f"{tag}/mmax"] = np.array(mmax)
        cases[f"{tag}/bond_dims_final"] = np.array(mps.bond_dims)
        # dense exact propagation (stands in for the qutip oracle of test_evolve.py)
        if len(model.basis) <= 9:
            H = _dense_from_mpo([np.asarray(m.array) for m in mpo])
            psi0 = np.asarray(init.todense()).ravel().astype(complex)
            w, x = np.linalg.eigh(H)
            dims = model.pbond_list
            e_sites = [i for i, b in enumerate(model.basis) if b.is_electron]
            exact = []
            for k in range(nsteps + 1):
                psit = x @ (np.exp(-1j * w * dt * k) * (x.conj().T @ psi0))
                t = psit.reshape(dims)
                row = []
                for s in e_sites:
                    p = np.sum(np.abs(np.take(t, 1, axis=s)) ** 2)
                    row.append(p)
                exact.append(row)
            cases[f"{tag}/exact_pops"] = np.array(exact)

    # the 3-site, 2-level Holstein model of tests/parameter_exact.py:9-17
    # (omega=1, displacement=1, J=1); that module also imports qutip, absent here
    exact_model = _holstein(3, 2, [(1.0, 1.0 / np.sqrt(2.0))])
    run("ps_exact3", exact_model, EvolveMethod.tdvp_ps, 0.4, 12, 0, "exact3")
    run("ps2_exact3", exact_model, EvolveMethod.tdvp_ps2, 0.4, 12, 5, "exact3")
    run("ps_hol4", _holstein(4, 4, [(1.0, 1.0)]), EvolveMethod.tdvp_ps, 0.05, 8, 8, "hartree")
    run("ps2_hol2m2", _holstein(2, 4, [(1.0, 1.0), (0.5, 0.7)]), EvolveMethod.tdvp_ps2, 0.025, 5, 8, "hartree")
    np.savez_compressed(out / "tdvp_cases.npz", **cases)


def _config_run(model, method, dt, nsteps, mmax, d, prefix, dump_init=True):
    """Hartree product (exciton on the first site) expanded with the MPO hint
    (expand_bond_dimension(mpo, include_ex=False), the configs' idiom), then
    nsteps of `method`; populations after every step under prefix."""
    from renormalizer.mps import Mps, Mpo
    from renormalizer.utils import EvolveConfig, CompressConfig, CompressCriteria
    np.random.seed(2024)
    mpo = Mpo(model)
    init = Mps.hartree_product_state(model, {0: 1})
    init.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=mmax)
    init = init.expand_bond_dimension(mpo, include_ex=False)
    mps = init.copy()
    mps.evolve_config = EvolveConfig(method)
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=mmax)
    if dump_init:
        _dump_mps(f"{prefix}/init", mps, d)
        _dump_mpo(f"{prefix}/mpo", mpo, d)
    pops = [np.asarray(mps.e_occupations)]
    for _ in range(nsteps):
        mps = mps.evolve(mpo, dt)
        pops.append(np.asarray(mps.e_occupations))
    d[f"{prefix}/pops"] = np.array(pops)
    d[f"{prefix}/dt"] = np.array(dt)
    d[f"{prefix}/mmax"] = np.array(mmax)
    d[f"{prefix}/bond_dims_final"] = np.array(mps.bond_dims)


def _c1_model():
    # config 1: 10 molecules, one mode (omega = 1, g = 1), 10 levels, J = 1
    return _holstein(10, 10, [(1.0, 1.0)])


def gen_c1_traj(threads, path):
    """one config-1 trajectory in this process (BLAS threads set by the caller)"""
    from renormalizer.utils import EvolveMethod
    d = {}
    _config_run(_c1_model(), EvolveMethod.tdvp_ps, 0.05, 100, 32, d, "c1", dump_init=True)
    np.savez(path, **d)


def gen_configs(out):
    """Config 1 exactly (10-molecule Holstein chain, one mode with omega = 1,
    g = 1 and 10 levels; hint-expanded Hartree start at M = 32; 100 steps of
    one-site TDVP-PS at dt = 0.05), run twice by the reference with 1 and 4
    BLAS threads -- the second run is the reference's own rounding envelope --
    and a reduced config 2 (4 molecules, two modes omega = 1 / 0.5, g = 1 /
    0.7, 16 levels, M = 32, ten steps of two-site TDVP-PS at dt = 0.025)."""
    import subprocess
    import tempfile
    from renormalizer.utils import EvolveMethod
    cases = {}
    with tempfile.TemporaryDirectory() as tmp:
        runs = {}
        for t in (1, 4):
            path = Path(tmp) / f"c1_t{t}.npz"
            env = dict(os.environ, OPENBLAS_NUM_THREADS=str(t), OMP_NUM_THREADS=str(t), MKL_NUM_THREADS=str(t),
                       RENO_NUM_THREADS=str(t))
            subprocess.run([sys.executable, str(Path(__file__).resolve()), "--c1-traj", str(t), str(path)],
                           check=True, env=env)
            runs[t] = dict(np.load(path))
        cases.update({k: v for k, v in runs[1].items()})
        cases["c1/pops_t4"] = runs[4]["c1/pops"]
        cases["c1/threads"] = np.array([1, 4])
    _config_run(_holstein(4, 16, [(1.0, 1.0), (0.5, 0.7)]), EvolveMethod.tdvp_ps2, 0.025, 10, 32, cases, "c2red")
    np.savez_compressed(out / "config_cases.npz", **cases)


def gen_dmrg(out):
    from renormalizer.mps import Mps, Mpo
    from renormalizer.mps.gs import optimize_mps
    from renormalizer.tests.parameter import holstein_model
    cases = {}

    def run(tag, model, procedure, method="2site", nexciton=1, e_atol=1e-8):
        np.random.seed(9012)
        mpo = Mpo(model)
        mps = Mps.random(model, nexciton, procedure[0][0], percent=1.0)
        mps.optimize_config.procedure = procedure
        mps.optimize_config.method = method
        mps.optimize_config.e_atol = e_atol
        _dump_mps(f"{tag}/init", mps, cases)
        _dump_mpo(f"{tag}/mpo", mpo, cases)
        energies, res = optimize_mps(mps.copy(), mpo)
        cases[f"{tag}/energies"] = np.array(energies)
        cases[f"{tag}/expectation"] = np.array(res.expectation(mpo))

    proc = [[10, 0.4], [20, 0.2], [30, 0.1], [40, 0], [40, 0]]
    run("hol_test_gs", holstein_model, proc)
    cases["hol_test_gs/GS_E"] = np.array(0.08401412 + holstein_model.gs_zpe)
    sbm, _, _ = _sbm(6, 4)
    run("sbm6x4", sbm, [[12, 0.4], [12, 0.2], [12, 0.1], [12, 0], [12, 0], [12, 0]], nexciton=0, e_atol=1e-9)
    np.savez_compressed(out / "dmrg_cases.npz", **cases)


def gen_obs(out):
    """calc_1site_rdm, calc_bond_singular_values / calc_bond_entropy and
    expectations (the shared-environment path) of an entangled complex MPS:
    a 3-molecule two-mode Holstein chain after 4 TDVP-PS2 steps."""
    from renormalizer.mps import Mps, Mpo
    from renormalizer.model import Op
    from renormalizer.utils import EvolveConfig, EvolveMethod, CompressConfig, CompressCriteria
    cases = {}
    np.random.seed(77)
    model = _holstein(3, 4, [(1.0, 1.0), (0.5, 0.7)])
    mpo = Mpo(model)
    mps = Mps.hartree_product_state(model, {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=10)
    mps = mps.expand_bond_dimension(mpo, include_ex=False)
    mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps2)
    for _ in range(4):
        mps = mps.evolve(mpo, 0.1)
    _dump_mps("obs/mps", mps, cases)
    rdm = mps.calc_1site_rdm()
    for i in range(len(mps)):
        cases[f"obs/rdm_{i}"] = np.asarray(rdm[i])
    s_array = mps.calc_bond_singular_values()
    cases["obs/bond_sv"] = np.asarray(s_array)
    cases["obs/bond_entropy"] = np.asarray(mps.calc_bond_entropy(s_array))
    # operators sharing prefixes / suffixes: every electronic occupation, the
    # Hamiltonian, and one phonon coordinate
    e_dofs = model.e_dofs
    ops = [Mpo(model, Op(r"a^\dagger a", d)) for d in e_dofs] + [mpo]
    ops.append(Mpo(model, Op("x", model.v_dofs[0])))
    for k, m in enumerate(ops):
        _dump_mpo(f"obs/op{k}", m, cases)
    cases["obs/nops"] = np.array(len(ops))
    cases["obs/expectations"] = np.asarray(mps.expectations(ops))
    cases["obs/expectations_naive"] = np.asarray(mps.expectations(ops, opt=False))
    np.savez_compressed(out / "obs_cases.npz", **cases)


def gen_mpdm(out):
    """Finite temperature (mps/thermalprop.py, mps/mpdm.py): the T = infinity
    one-exciton density operator of a 3-molecule Holstein chain, bonds
    expanded with the Hamiltonian hint (ThermalProp's auto_expand), then
    imaginary-time TDVP-PS / TDVP-PS2 steps towards beta / 2 at 298 K.  Stored:
    the expanded start (4-index sites), and after every step the energy,
    electronic and phonon occupations and bond entropies ThermalProp records."""
    from renormalizer.mps import MpDm, ThermalProp
    from renormalizer.utils import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, Quantity
    cases = {}
    model = _holstein(3, 3, [(1.0, 1.0)])
    beta = Quantity(298, "K").to_beta()
    for tag, method, m in (("ps", EvolveMethod.tdvp_ps, 10), ("ps2", EvolveMethod.tdvp_ps2, 10)):
        np.random.seed(7)
        init = MpDm.max_entangled_ex(model)
        init.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=m)
        tp = ThermalProp(init, evolve_config=EvolveConfig(method))
        _dump_mps(f"{tag}/init", tp.latest_mps, cases)
        nsteps, dbeta = 6, beta / 2j / 2000
        tp.evolve(evolve_dt=dbeta, nsteps=nsteps)
        cases[f"{tag}/dbeta"] = np.array(dbeta)
        cases[f"{tag}/mmax"] = np.array(m)
        cases[f"{tag}/energies"] = np.array(tp.energies)
        cases[f"{tag}/e_occ"] = tp.e_occupations_array
        cases[f"{tag}/ph_occ"] = tp.ph_occupations_array
        cases[f"{tag}/entropy"] = tp.vn_entropy_array
        cases[f"{tag}/bond_dims_final"] = np.array(tp.latest_mps.bond_dims)
    np.savez_compressed(out / "mpdm_cases.npz", **cases)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default=None)
    ap.add_argument("--c1-traj", nargs=2, default=None, metavar=("THREADS", "PATH"),
                    help="internal: run one config-1 trajectory into PATH")
    args = ap.parse_args()
    _import_reference(args.reference)
    if args.c1_traj:
        gen_c1_traj(int(args.c1_traj[0]), args.c1_traj[1])
        return
    gens = dict(heff=gen_heff, env=gen_env, krylov=gen_krylov, svd=gen_svd, mpo=gen_mpo, tdvp=gen_tdvp,
                dmrg=gen_dmrg, obs=gen_obs, configs=gen_configs, mpdm=gen_mpdm)
    for name, fn in gens.items():
        if args.only and name not in args.only.split(","):
            continue
        fn(HERE)
        print("wrote", name)


if __name__ == "__main__":
    main()
