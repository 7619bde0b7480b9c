#!/usr/bin/env python
"""Benchmark: TDVP steps/s of the two-site TDVP-PS sweep on a 32-site Holstein
chain with two modes per site (omega = 1, 0.5; g = 1, 0.7), 16 SHO levels per
mode (96 MPS sites), bond dimension M = 256, dt = 0.025.

One "step" is one full Mps.evolve call (two half-sweeps, every two-site
Krylov exponential, QN-blocked SVD truncation, backward one-site exponential
and environment update), the reference's _evolve_tdvp_ps2
(renormalizer/mps/mps.py:1406-1517).

Arms:
  default            the B200 engine (renormalizer_b200, libreno_b200.so)
  --impl reference   the reference algorithm on the host cores (the numpy
                     oracle port of it: the reference is a Python package
                     that is not installed on the GPU machine), one bounded
                     sample of a step per timed step, extrapolated to a full
                     step from per-operation timings at M = 256.

Prints ONE JSON line (rank 0).  Multi-GPU runs are independent replicas
(the sweep does not shard): value = total steps of all ranks / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# DRAM bytes (read + write) of one phonon-phonon 2-site matvec at M = 256,
# d = 16 x 16, from ncu captures of the four split_gemm_kernel launches (the
# same 4.00 GB in both captures recorded in
# profiles/split_gemm_fused_heff2_ph_ph_M256_bf16x3.md); ncu cannot run
# inside this timed region
TRAFFIC_PH_PH = {"bf16x3": 4.00e9}
METRIC = "TDVP steps/s at M=256 (2-site TDVP-PS, 32-site two-mode Holstein, split-prec vs FP64)"
WORKLOAD = "holstein32x2modes_nlev16_M256_tdvp_ps2_dt0.025"
# average Krylov vectors per local exponential of this workload, measured by
# the engine on B200 (evolve_config.stat); used by the CPU extrapolation
KRY2_DEFAULT = 8.0
KRY1_DEFAULT = 8.0
# the metric's accuracy gate, measured over 200 steps of this workload at 8
# molecules by `bench.py --accuracy 200 --nmol 8 --start hint --accuracy-precs
# bf16x3,tf32x3 --envelope` (52 min of B200 time: too long for this run);
# per-step table in profiles/accuracy_tdvp_ps2_holstein24_M256.md
ACCURACY_200 = {"steps": 200, "nmol": 8, "max_abs_dpop": {"bf16x3": 1.074e-5, "tf32x3": 7.99e-6},
                "fp64_envelope": 1.63e-9, "first_step_above_1e-6": {"bf16x3": 24, "tf32x3": 29},
                "holds_1e-6": False, "record": "profiles/accuracy_tdvp_ps2_holstein24_M256.md",
                "fp64_random_1e-9_per_step_30_steps": 9.3e-9,
                "promoted_accumulation_chunk128_max": {"tf32x3 (25 steps)": 7.95e-8, "bf16x3 (30 steps)": 3.09e-6},
                "cause": "the tensor cores' FP32 accumulation truncates toward zero: a bias linear in K "
                         "(-1.4e-5 BF16x3, -3.0e-5 TF32x3 relative at K = 4096, bench.py --accumulation)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--prec", default=os.environ.get("RENO_BENCH_PREC", "bf16x3"),
                    choices=["fp64", "bf16x3", "tf32x3"])
    ap.add_argument("--nmol", type=int, default=32)
    ap.add_argument("--nlev", type=int, default=16)
    ap.add_argument("--M", type=int, default=256)
    ap.add_argument("--dt", type=float, default=0.025)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--accuracy", type=int, default=0, metavar="STEPS",
                    help="run STEPS steps with --prec and with plain FP64 from the same start and report the "
                         "largest site-population difference after every step (no timing)")
    ap.add_argument("--start", default="random", choices=["random", "hint"],
                    help="bond expansion of the start state: seeded random expander, or the reference's "
                         "expand_bond_dimension(mpo, include_ex=False)")
    ap.add_argument("--accuracy-precs", default="",
                    help="comma-separated precisions compared with FP64 in --accuracy mode (default: --prec)")
    ap.add_argument("--envelope", action="store_true",
                    help="--accuracy mode: also evolve FP64 from the start state perturbed by one ulp per entry "
                         "and report its distance from the unperturbed FP64 run (the FP64 engine's own envelope)")
    ap.add_argument("--acc-chunk", type=int, default=0, metavar="K",
                    help="promote the split GEMMs' tensor-core accumulation every K elements of K "
                         "(reno_set_split_accumulation_chunk; 0 = off)")
    ap.add_argument("--accumulation", action="store_true",
                    help="the split GEMM's FP32 accumulation error on exactly representable operands, K = 64 .. 16384")
    ap.add_argument("--inject", default="",
                    help="--accuracy mode: comma-separated relative sizes delta; each adds an FP64 arm whose site "
                         "tensors get a seeded random relative perturbation of size delta after every step")
    ap.add_argument("--out", default="", help="append the per-step JSON lines of --accuracy mode to this file")
    ap.add_argument("--krylov-tol", default="",
                    help="rtol,atol of the Lanczos convergence test for every arm (default: the reference's "
                         "numpy allclose defaults 1e-5,1e-8)")
    ap.add_argument("--accuracy-lockstep", type=int, default=1,
                    help="--accuracy mode: advance the FP64 reference and every arm together through "
                         "evolve_batch (1, default) or one after another (0)")
    ap.add_argument("--truncation", default="exact", choices=["exact", "subspace"],
                    help="exact (default): every QN block uses the full Gram eigendecomposition; subspace: blocks "
                         "with at least 1024 rows on the smaller side use the opt-in top-k subspace iteration")
    ap.add_argument("--dmrg", action="store_true",
                    help="ground-state DMRG of the spin-boson model (one spin, 64 Ohmic modes with alpha=0.5, "
                         "omega_c=10, 8 levels; M=256) in the chosen split precision and in FP64")
    ap.add_argument("--grad", action="store_true",
                    help="gradient of the site-0 population after a TDVP-PS trajectory with respect to per-molecule "
                         "couplings (16-molecule Holstein, 10 levels, M=64, 50 steps of dt=0.05)")
    ap.add_argument("--heev", type=int, default=0, metavar="N",
                    help="time the device Hermitian eigensolver (leading 320 eigenpairs, or N/2 below 640) against "
                         "cuSOLVER eigh on a seeded N x N complex Gram matrix")
    ap.add_argument("--batch", type=int, default=0, metavar="B",
                    help="config 4: TDVP-PS2 of B static-disorder realisations (--batch-nmol molecules with one "
                         "10-level mode, site energies N(0, 0.5), hoppings 1 + N(0, 0.1), bonds <= --batch-M with "
                         "the 1e-8 threshold) advanced in lockstep, against the same realisations one by one")
    ap.add_argument("--batch-nmol", type=int, default=16)
    ap.add_argument("--batch-M", type=int, default=128)
    ap.add_argument("--batch-serial", type=int, default=4,
                    help="--batch mode: realisations timed one by one for the comparison")
    ap.add_argument("--cpu-worker", default="", help=argparse.SUPPRESS)
    ap.add_argument("--heff-only", action="store_true",
                    help="time only the workload's largest 2-site H_eff matvec (phonon-phonon block, M x 16 x 16 x M)")
    return ap.parse_args()


# ---------------------------------------------------------------- workload
def holstein_2mode(nmol, nlev):
    from renormalizer_b200 import HolsteinModel, Mol, Phonon, Quantity
    modes = [(1.0, 1.0), (0.5, 0.7)]
    ph = [Phonon.simple_phonon(Quantity(w), Quantity(np.sqrt(2.0) * g / np.sqrt(w)), nlev) for w, g in modes]
    return HolsteinModel([Mol(Quantity(0), ph)] * nmol, Quantity(1.0), 3)


def initial_state(model, M, start="random", mpo=None):
    """Hartree product with the exciton on site 0, bond dimension expanded to
    M: "hint" is the reference's idiom expand_bond_dimension(mpo,
    include_ex=False) (coef 1e-10 weighted H^k psi directions); "random" adds
    a seeded random expander instead."""
    from renormalizer_b200 import CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, Mps
    np.random.seed(2024)
    mps = Mps.hartree_product_state(model, {0: 1})
    mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=M)
    if start == "hint":
        mps = mps.expand_bond_dimension(mpo, include_ex=False)
    else:
        mps = mps.expand_bond_dimension()
    mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps2)
    return mps


def heff_flops(nsite, ml, mr, wl, wm, wr, d1, d2, cplx=True):
    """algorithmic flops of one H_eff matvec (complex x complex = 8, complex x real = 4)"""
    c1, c2 = (8, 4) if cplx else (2, 2)
    if nsite == 2:
        return c1 * (ml * wl * ml * d1 * d2 * mr + ml * d1 * d2 * wr * mr * mr) + \
            c2 * (ml * d1 * wm * wl * d1 * d2 * mr + ml * d1 * d2 * wr * wm * d2 * mr)
    if nsite == 1:
        return c1 * (ml * wl * ml * d1 * mr + ml * d1 * wr * mr * mr) + c2 * ml * d1 * wr * wl * d1 * mr
    return c1 * (ml * wl * ml * mr + ml * wl * mr * mr)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU (oracle) sample
def cpu_step_sample(M, nlev, kry2, kry1, n_pairs_pp, n_pairs_ep):
    """Time the reference algorithm's per-operation costs at M on the host
    cores with the numpy restatement (oracle), then assemble one TDVP-PS2
    step: per half-sweep every two-site pair runs kry2 two-site matvecs, one
    QN-blocked SVD, one environment update and (all but the last pair) a
    backward one-site exponential of kry1 matvecs plus a QN QR."""
    from oracle import reno_oracle as O
    rng = np.random.default_rng(0)
    w = 5
    cx = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    L, R = cx(M, w, M), cx(M, w, M)
    Wp, We = rng.standard_normal((w, nlev, nlev, w)), rng.standard_normal((w, 2, 2, w))
    t = {}

    def timed(name, fn):
        s = time.perf_counter()
        fn()
        t[name] = time.perf_counter() - s

    psi_pp = cx(M, nlev, nlev, M)
    psi_ep = cx(M, 2, nlev, M)
    timed("mv2_pp", lambda: O.hop(L, [Wp, Wp], R, psi_pp))
    timed("mv2_ep", lambda: O.hop(L, [We, Wp], R, psi_ep))
    psi_p, psi_e = cx(M, nlev, M), cx(M, 2, M)
    timed("mv1_p", lambda: O.hop(L, [Wp], R, psi_p))
    timed("mv1_e", lambda: O.hop(L, [We], R, psi_e))
    timed("env_p", lambda: O.contract_one_site(L, psi_p, Wp, "L"))
    timed("env_e", lambda: O.contract_one_site(L, psi_e, We, "L"))
    # QN blocks of the one-exciton sector: left bond labels {0,1} half/half
    qnl = np.array([[0]] * (M // 2) + [[1]] * (M // 2))
    sig_e, sig_p = np.array([[0], [1]]), np.zeros((nlev, 1), dtype=int)
    qnbigl = O.add_outer(qnl, sig_p)
    qnbigr = O.add_outer(sig_p, qnl)
    mask = O.get_qn_mask(O.add_outer(qnbigl, qnbigr), np.array([1]))
    timed("svd_pp", lambda: O.svd_qn(psi_pp * mask, qnbigl, qnbigr, np.array([1])))
    qnbigl_e = O.add_outer(qnl, sig_e)
    mask_e = O.get_qn_mask(O.add_outer(qnbigl_e, qnbigr), np.array([1]))
    timed("svd_ep", lambda: O.svd_qn(psi_ep * mask_e, qnbigl_e, qnbigr, np.array([1])))
    qn1 = O.add_outer(qnl, sig_p)
    timed("qr_p", lambda: O.svd_qn(psi_p * O.get_qn_mask(O.add_outer(qn1, qnl), np.array([1])), qn1, qnl,
                                   np.array([1]), QR=True, system="L", full_matrices=False))
    sample_s = sum(t.values())
    per_pair_pp = kry2 * t["mv2_pp"] + t["svd_pp"] + t["env_p"] + kry1 * t["mv1_p"] + t["qr_p"]
    per_pair_ep = kry2 * t["mv2_ep"] + t["svd_ep"] + 0.5 * (t["env_p"] + t["env_e"]) + \
        kry1 * 0.5 * (t["mv1_p"] + t["mv1_e"]) + t["qr_p"]
    step_s = 2 * (n_pairs_pp * per_pair_pp + n_pairs_ep * per_pair_ep)
    return step_s, sample_s, t


def config1_anchor(nsteps):
    """Config 1 (10-molecule Holstein chain, one 10-level mode, the
    reference's hint-expanded start at M = 32) on the host: nsteps of the
    numpy restatement's one-site TDVP-PS at dt = 0.05, timed directly.
    Returns steps/s."""
    from oracle import reno_oracle as O
    d = np.load(ROOT / "tests" / "golden" / "config_cases.npz")
    n = int(d["c1/init/nsites"])
    init = O.OMps([d[f"c1/init/mt_{i}"] for i in range(n)], [d[f"c1/init/qn_{i}"] for i in range(n + 1)],
                  int(d["c1/init/qnidx"]), d["c1/init/qntot"], bool(d["c1/init/to_right"]),
                  [d[f"c1/init/sigmaqn_{i}"] for i in range(n)], compress=O.Compress("fixed", max_bonddim=32))
    mpo = [d[f"c1/mpo/W_{i}"] for i in range(n)]
    mps = init
    t0 = time.perf_counter()
    for _ in range(nsteps):
        mps = O.evolve_tdvp_ps(mps, mpo, 0.05)
    return nsteps / (time.perf_counter() - t0)


def cpu_worker(spec):
    """Internal (--cpu-worker): run the CPU samples in this process, whose
    BLAS thread count the parent set, and print them as one JSON line."""
    M, nlev, kry2, kry1, npp, nep, c1_steps = json.loads(spec)
    st, ss, _ = cpu_step_sample(M, nlev, kry2, kry1, npp, nep)
    out = {"threads": threads(), "m256_step_s": st, "m256_sample_s": ss}
    if c1_steps:
        out["config1_steps_per_s"] = config1_anchor(c1_steps)
    print(json.dumps(out), flush=True)


def cpu_baselines(M, nlev, kry2, kry1, npp, nep, thread_counts=(1, 4, 8), c1_steps=10):
    """The host baseline at several BLAS thread counts (one subprocess each:
    the thread count is fixed when numpy loads its BLAS).  Per count: the
    modelled M-site step (per-operation timings assembled into one step) and
    a directly timed config-1 anchor."""
    out = {}
    ncpu = os.cpu_count() or 1
    for t in thread_counts:
        if t > ncpu:
            continue
        env = dict(os.environ, OPENBLAS_NUM_THREADS=str(t), OMP_NUM_THREADS=str(t), MKL_NUM_THREADS=str(t),
                   RENO_NUM_THREADS=str(t))
        spec = json.dumps([M, nlev, kry2, kry1, npp, nep, c1_steps])
        r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--cpu-worker", spec], env=env,
                           capture_output=True, text=True, timeout=900)
        lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
        if r.returncode == 0 and lines:
            out[t] = json.loads(lines[-1])
    return out


def threads():
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 1) for i in threadpool_info() if i.get("user_api") == "blas"]
        return max(n) if n else os.cpu_count()
    except Exception:
        return os.cpu_count()


def n_pairs(nmol):
    # pairs (e,p1), (p1,p2), (p2,e') along the 3*nmol-site chain
    npp = nmol
    nep = 3 * nmol - 1 - npp
    return npp, nep


# ---------------------------------------------------------------- arms
def run_reference(args, rank, world):
    if rank != 0:
        return
    npp, nep = n_pairs(args.nmol)
    for _ in range(args.warmup):
        from oracle import reno_oracle as O
        O.hop(np.ones((8, 2, 8)), [np.ones((2, 3, 3, 2))], np.ones((8, 2, 8)), np.ones((8, 3, 8)))
    steps, samples = [], []
    for _ in range(args.steps):
        st, ss, _ = cpu_step_sample(args.M, args.nlev, KRY2_DEFAULT, KRY1_DEFAULT, npp, nep)
        steps.append(st)
        samples.append(ss)
    step_s = float(np.mean(steps))
    value = 1.0 / step_s
    cores = threads()
    c1 = config1_anchor(10)
    sample = (f"per-operation timings at M={args.M} (2-site matvecs, QN SVDs, 1-site matvecs, env updates, QR) "
              f"with the numpy oracle, {np.mean(samples):.1f} s of CPU work per step, assembled into one step "
              f"with {KRY2_DEFAULT}/{KRY1_DEFAULT} Krylov vectors per 2-/1-site exponential (modelled: a full "
              f"CPU step takes about half an hour); beside it, config 1 timed directly")
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "nsites": 3 * args.nmol, "M": args.M, "nlev": args.nlev,
                       "dt": args.dt, "parallelism": "replicas" if world > 1 else "single"},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample,
                             "modelled": True, "host_cpus": os.cpu_count(),
                             "RENO_NUM_THREADS": os.environ.get("RENO_NUM_THREADS", "unset"),
                             "config1_anchor": {"steps_per_s": c1, "steps": 10, "measured": True,
                                                "workload": "holstein10_nlev10_M32_tdvp_ps_dt0.05"}},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


class HeffTimer:
    """Records CUDA events around every 2-site H_eff matvec on its stream."""

    def __init__(self):
        self.events = []

    def install(self):
        import importlib
        import torch
        H = importlib.import_module("renormalizer_b200.hop_expr")
        orig = H.HeffOperator.apply
        timer = self

        def apply(op, psi, out=None):
            if op.nsite != 2:
                return orig(op, psi, out)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            r = orig(op, psi, out)
            e.record()
            d = op.desc
            timer.events.append((s, e, heff_flops(2, d.ml, d.mr, d.wl, d.wm, d.wr, d.d1, d.d2),
                                 (d.ml, d.mr, d.d1, d.d2)))
            return r

        H.HeffOperator.apply = apply
        self._orig = orig
        return self

    def uninstall(self):
        import importlib
        importlib.import_module("renormalizer_b200.hop_expr").HeffOperator.apply = self._orig

    def result(self, shape=None):
        """(flops, ms, count) over all 2-site matvecs, or over those of one
        block shape (ml, mr, d1, d2)"""
        ev = [x for x in self.events if shape is None or x[3] == shape]
        tot_ms = sum(s.elapsed_time(e) for s, e, _, _ in ev)
        fl = sum(f for _, _, f, _ in ev)
        return fl, tot_ms, len(ev)


class PhaseTimer:
    """CUDA-event device time per phase of the sweep (host-visible breakdown)."""

    def __init__(self):
        self.events = {}
        self._saved = []

    def wrap(self, module, name, label):
        import torch
        orig = getattr(module, name)
        events = self.events.setdefault(label, [])

        def wrapped(*a, **k):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            r = orig(*a, **k)
            e.record()
            events.append((s, e))
            return r

        setattr(module, name, wrapped)
        self._saved.append((module, name, orig))

    def install(self):
        import importlib
        mps_mod = importlib.import_module("renormalizer_b200.mps")
        lib_mod = importlib.import_module("renormalizer_b200.lib")
        self.wrap(mps_mod, "svd_truncate", "svd_truncate")
        self.wrap(mps_mod, "qr_split", "qr_split")
        self.wrap(mps_mod, "expm_krylov", "krylov_total")
        self.wrap(lib_mod, "contract_one_site", "env_update")
        return self

    def uninstall(self):
        for m, n, o in self._saved:
            setattr(m, n, o)

    def result(self):
        return {k: round(sum(s.elapsed_time(e) for s, e in v), 1) for k, v in self.events.items()}


def fp64_peak_tflops(dev):
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ a
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a
    return best


def tf32_peak_tflops(dev):
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float32, device=dev)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ a
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a
    return best


def reduce_max_ms(t_ms: float, dist, device) -> float:
    """The multi-GPU timing rule: every rank's device time, max over ranks
    (one all-reduce; identity without a process group)."""
    if dist is None:
        return float(t_ms)
    import torch
    tt = torch.tensor([float(t_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def run_engine(args, rank, world, dist):
    import torch
    from renormalizer_b200 import Mpo, backend
    from renormalizer_b200._native import launch_count
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    backend.prec = args.prec
    model = holstein_2mode(args.nmol, args.nlev)
    mpo = Mpo(model)
    mps0 = initial_state(model, args.M, args.start, mpo)
    mps = mps0
    pops_first = None
    for i in range(args.warmup):
        mps = mps.evolve(mpo, args.dt)
        if i == 0:
            pops_first = mps.e_occupations
    kry = mps.evolve_config.stat

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    timer = HeffTimer().install()
    phases = PhaseTimer().install()
    barrier()
    l0 = launch_count()
    import importlib
    svdmod = importlib.import_module("renormalizer_b200.svd_qn")
    sub0 = (svdmod.subspace.calls, svdmod.subspace.fallbacks, svdmod.subspace.retries, svdmod.refine.calls,
            svdmod.refine.blocks)
    svdmod.flop_log = []
    with ClockSampler(local) as clocks:
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_ev.record()
        for _ in range(args.steps):
            mps = mps.evolve(mpo, args.dt)
        e_ev.record()
        barrier()
    launches = launch_count() - l0
    trunc_fl = float(sum(svdmod.flop_log))
    svdmod.flop_log = None
    heev_mod = importlib.import_module("renormalizer_b200.heev")
    trunc = {"device_eigensolver_fallbacks": heev_mod.heev_opts.fallbacks,
             "small_sigma_refinements": {"truncations": svdmod.refine.calls - sub0[3],
                                         "blocks": svdmod.refine.blocks - sub0[4], "tau": svdmod.refine.tau},
             "subspace_blocks": svdmod.subspace.calls - sub0[0], "retries": svdmod.subspace.retries - sub0[2],
             "fallbacks": svdmod.subspace.fallbacks - sub0[1],
             "options": {"min_dim": svdmod.subspace.min_dim, "iters": svdmod.subspace.iters,
                         "oversample": svdmod.subspace.oversample, "rtol": svdmod.subspace.rtol}}
    timer.uninstall()
    phases.uninstall()
    t_ms = reduce_max_ms(s_ev.elapsed_time(e_ev), dist, dev)
    value = world * args.steps / (t_ms * 1e-3)
    fl, heff_ms, nheff = timer.result()
    kry_timed = {k: v for k, v in (mps.evolve_config.stat or {}).items() if k != "counts"} or None

    # e2e: host-resident MPS (pinned), copied in, evolved, populations copied out
    e2e = None
    if not args.no_e2e:
        host_sites = [t.cpu().pin_memory() for t in mps]
        h2d = sum(t.numel() * t.element_size() for t in host_sites)
        barrier()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.record()
        ne2e = min(args.steps, 3)
        for _ in range(ne2e):
            m = mps.metacopy()
            m._mp = [t.to(dev, non_blocking=True) for t in host_sites]
            m = m.evolve(mpo, args.dt)
            pops = m.e_occupations
        e2.record()
        barrier()
        te = reduce_max_ms(s2.elapsed_time(e2), dist, dev)
        e2e = {"value": world * ne2e / (te * 1e-3), "unit": "steps/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(pops.size * 8)}

    # plain FP64 engine from the same start state: population difference after
    # the first step, and its steps/s over several steps
    fp64 = None
    if args.prec != "fp64":
        backend.prec = "fp64"
        nfp = max(1, min(args.steps, 4))
        barrier()
        s3, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s3.record()
        ref = mps0.evolve(mpo, args.dt)
        pops_ref = ref.e_occupations
        for _ in range(nfp - 1):
            ref = ref.evolve(mpo, args.dt)
        e3.record()
        barrier()
        t_fp = reduce_max_ms(s3.elapsed_time(e3), dist, dev)
        fp64 = {"steps_per_s": world * nfp / (t_fp * 1e-3), "steps_timed": nfp,
                "max_abs_dpop_after_1_step": float(np.abs(pops_ref - pops_first).max())}
        backend.prec = args.prec

    peaks = None
    if rank == 0:
        peaks = {"fp64_dgemm_tflops": fp64_peak_tflops(dev), "tf32_tflops": tf32_peak_tflops(dev),
                 "source": "cuBLAS 8192^3 GEMMs measured in this run (best of 4)"}
        try:
            mp = json.load(open(ROOT / "MEASURED_PEAKS.json"))
            peaks["bf16_tflops_sustained"] = mp.get("bf16_tflops_sustained")
            peaks["hbm_gbs"] = mp.get("hbm_gbs")
        except Exception:
            pass

    if args.prec == "fp64":
        peak, peak_src = peaks["fp64_dgemm_tflops"] if peaks else fp64_peak_tflops(dev), \
            "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)"
    else:
        peak, peak_src = None, "MEASURED_PEAKS.json bf16_tflops_sustained"
        try:
            peak = json.load(open(ROOT / "MEASURED_PEAKS.json"))["bf16_tflops_sustained"]
        except Exception:
            peak, peak_src = 1400.0, "fallback 1.4 PFLOP/s sustained (MEASURED_PEAKS.json absent)"
    achieved_all = fl / (heff_ms * 1e-3) / 1e12 if heff_ms > 0 else 0.0
    # the dominant kernel: the phonon-phonon 2-site matvec (M x 16 x 16 x M),
    # timed in situ; its DRAM traffic per matvec is from one ncu capture of
    # the same block (bench.py --heff-only --steps 1 --warmup 3, the four
    # split_gemm_kernel launches of one matvec: dram__bytes_read.sum +
    # dram__bytes_write.sum)
    blk = (args.M, args.M, args.nlev, args.nlev)
    fl_b, ms_b, n_b = timer.result(blk)
    achieved = fl_b / (ms_b * 1e-3) / 1e12 if ms_b > 0 else achieved_all
    traffic = TRAFFIC_PH_PH.get(args.prec) if (args.M, args.nlev) == (256, 16) else None
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None, "traffic": traffic,
                "kernel": f"reno_heff_apply nsite=2, phonon-phonon block {blk} (fused split chain: 4 persistent "
                          f"split_gemm_kernel launches), algorithmic complex flops",
                "launches_timed": n_b, "ms_per_launch": ms_b / n_b if n_b else None,
                "traffic_unit": "bytes per matvec (DRAM read + write)",
                "all_2site_matvecs": {"achieved": achieved_all, "launches_timed": nheff},
                "peak_source": peak_src}

    # truncation: algorithmic FP64 flops of its block factorisations against
    # the measured DGEMM rate
    trunc_ms = phases.result().get("svd_truncate", 0.0)
    trunc_roof = None
    if trunc_fl and trunc_ms > 0 and peaks:
        ach = trunc_fl / (trunc_ms * 1e-3) / 1e12
        trunc_roof = {"bound": "fp64 (latency-bound reduction)", "achieved": ach, "unit": "TFLOP/s",
                      "peak": peaks["fp64_dgemm_tflops"], "frac": ach / peaks["fp64_dgemm_tflops"],
                      "ms_per_step": trunc_ms / args.steps, "gflop_per_step": trunc_fl / args.steps / 1e9,
                      "counted": "per QN block: Gram 8 s^2 l, tridiagonal reduction 16/3 s^3, back-transformation "
                                 "8 s^2 k, projection 8 s l k (complex; real blocks a quarter), s / l the block's "
                                 "smaller / larger side, k the eigenvectors used"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        npp, nep = n_pairs(args.nmol)
        k2 = kry_timed["mean"] if kry_timed else KRY2_DEFAULT
        by_t = cpu_baselines(args.M, args.nlev, k2, k2, npp, nep)
        if by_t:
            tmax = max(by_t)
            cpu = {"value": 1.0 / by_t[tmax]["m256_step_s"], "unit": "steps/s", "cores": by_t[tmax]["threads"],
                   "kind": "port", "modelled": True, "host_cpus": os.cpu_count(),
                   "RENO_NUM_THREADS": {str(t): t for t in by_t},
                   "sample": f"numpy oracle per-operation timings at M={args.M} "
                             f"({by_t[tmax]['m256_sample_s']:.1f} s of CPU work at {tmax} BLAS threads), assembled "
                             f"into one TDVP-PS2 step with the engine's measured {k2:.2f} Krylov vectors per "
                             f"exponential (a full CPU step takes about half an hour)",
                   "by_threads": {str(t): {"modelled_steps_per_s": 1.0 / v["m256_step_s"],
                                           "config1_steps_per_s": v.get("config1_steps_per_s")}
                                  for t, v in by_t.items()},
                   "config1_anchor": "holstein10_nlev10_M32_tdvp_ps_dt0.05, 10 steps of the numpy restatement "
                                     "timed directly per thread count"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128" if args.prec == "fp64" else args.prec,
                "data": f"synthetic (Hartree product + {'the hint-MPO' if args.start == 'hint' else 'a seeded random'} bond expansion to M)",
                "config": {"workload": WORKLOAD, "nsites": 3 * args.nmol, "M": args.M, "nlev": args.nlev,
                           "dt": args.dt, "prec": args.prec, "parallelism": "replicas" if world > 1 else "single",
                           "l2": "inputs larger than L2 (MPS ~1.5 GB, environments ~1 GB resident in HBM)"},
                "tflops_heff2": achieved_all, "heff2_ms": round(heff_ms, 1), "phase_ms": phases.result(),
                "krylov": kry_timed, "bond_dims_max": max(mps.bond_dims), "truncation": trunc,
                "roofline": roofline, "truncation_roofline": trunc_roof, "peaks": peaks, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks.summary(), "fp64_engine": fp64, "accuracy": ACCURACY_200}
        print(json.dumps(line), flush=True)


def run_heff_only(args):
    """--steps matvecs of the phonon-phonon block (ml = mr = M, d1 = d2 = nlev)
    with the workload's own MPO tensors and seeded random complex L, R, psi.
    Inputs (~1.6 GB incl. intermediates) exceed L2; each timed matvec reads
    and writes them all."""
    import torch
    from renormalizer_b200 import Mpo, backend
    from renormalizer_b200._native import launch_count
    from renormalizer_b200.hop_expr import HeffOperator
    torch.cuda.set_device(0)
    backend.prec = args.prec
    model = holstein_2mode(args.nmol, args.nlev)
    mpo = Mpo(model)
    i = next(k for k in range(1, len(mpo) - 1) if mpo[k].shape[1] == args.nlev and mpo[k + 1].shape[1] == args.nlev)
    W1, W2 = mpo[i], mpo[i + 1]
    wl, wm, wr = W1.shape[0], W1.shape[3], W2.shape[3]
    M, d = args.M, args.nlev
    g = torch.Generator(device="cuda").manual_seed(7)
    cx = lambda *s: torch.complex(torch.randn(s, dtype=torch.float64, device="cuda", generator=g),
                                  torch.randn(s, dtype=torch.float64, device="cuda", generator=g))
    L, R, psi = cx(M, wl, M), cx(M, wr, M), cx(M, d, d, M)
    op = HeffOperator(L, R, [W1, W2], psi.shape, prec=args.prec)
    y = torch.empty_like(psi)
    for _ in range(args.warmup):
        op.apply(psi, y)
    torch.cuda.synchronize()
    l0 = launch_count()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s_ev, e_ev in evs:
        s_ev.record()
        op.apply(psi, y)
        e_ev.record()
    torch.cuda.synchronize()
    ms = [s_ev.elapsed_time(e_ev) for s_ev, e_ev in evs]
    fl = heff_flops(2, M, M, wl, wm, wr, d, d)
    t = statistics.median(ms)
    print(json.dumps({"metric": "2-site H_eff matvec (phonon-phonon block)", "value": fl / (t * 1e-3) / 1e12,
                      "unit": "TFLOP/s", "ms_per_matvec": t, "ms_all": ms, "gflop": fl / 1e9, "prec": args.prec,
                      "shape": {"M": M, "d1": d, "d2": d, "wl": wl, "wm": wm, "wr": wr},
                      "gpu_launches_per_matvec": (launch_count() - l0) / args.steps}))


def perturb_ulp(mps, seed=11):
    """A copy of mps with every site-tensor entry moved by one unit in the last
    place (random direction per entry and per real/imaginary part)."""
    import torch
    new = mps.copy()
    g = torch.Generator(device=new[0].device).manual_seed(seed)
    for i, t in enumerate(new._mp):
        r = torch.view_as_real(t) if t.is_complex() else t
        sign = torch.randint(0, 2, r.shape, device=r.device, generator=g).to(torch.float64) * 2 - 1
        r2 = torch.nextafter(r, sign * float("inf")).contiguous()
        new._mp[i] = torch.view_as_complex(r2) if t.is_complex() else r2
    return new


def perturb_rel(mps, delta, seed):
    """A copy of mps with every site-tensor entry x replaced by x (1 + delta r),
    r uniform in (-1, 1) per entry and per real/imaginary part: a step's worth
    of relative error delta injected into an FP64 trajectory."""
    import torch
    new = mps.copy()
    g = torch.Generator(device=new[0].device).manual_seed(seed)
    for i, t in enumerate(new._mp):
        r = torch.view_as_real(t) if t.is_complex() else t
        u = torch.rand(r.shape, dtype=torch.float64, device=r.device, generator=g) * 2 - 1
        r2 = (r * (1 + delta * u)).contiguous()
        new._mp[i] = torch.view_as_complex(r2) if t.is_complex() else r2
    return new


def run_accumulation(args):
    """Accumulation error of the split GEMM alone: operands exactly
    representable in the split's piece format (BF16 / TF32), so every
    product is exact and only the accumulation rounds.  One JSON line per
    (chunk, sign, precision, K): normwise relative error against FP64, the
    mean signed error over mean |C| (bias) and the fraction of positive
    errors, for random-sign and all-positive operands; chunk 0 is the
    tensor cores' accumulation over all of K, chunk 128 the promoted form
    (reno_set_split_accumulation_chunk)."""
    import torch
    from renormalizer_b200._native import Engine
    torch.cuda.set_device(0)
    eng = Engine.get(0)
    g = torch.Generator(device="cuda").manual_seed(0)

    def exact(x, prec):
        if prec == "bf16x3":
            return x.to(torch.bfloat16).to(torch.float64)
        f = x.to(torch.float32)                     # TF32: 10 explicit mantissa bits
        return (f.view(torch.int32) & ~((1 << 13) - 1)).view(torch.float32).to(torch.float64)

    from renormalizer_b200._native import load_library
    lib = load_library()
    for chunk, sign, prec in [(c, s, p) for c in (0, 128) for s in ("random", "positive") for p in ("bf16x3", "tf32x3")]:
        assert lib.reno_set_split_accumulation_chunk(chunk) == 0
        for K in (64, 256, 1024, 4096, 16384):
            A = torch.randn(256, K, dtype=torch.float64, device="cuda", generator=g)
            B = torch.randn(K, 256, dtype=torch.float64, device="cuda", generator=g)
            if sign == "positive":
                A, B = A.abs(), B.abs()
            A, B = exact(A, prec).contiguous(), exact(B, prec).contiguous()
            C = eng.matmul(A, B, prec=prec)
            ref = eng.matmul(A, B, prec="fp64")
            err = C - ref
            print(json.dumps({"chunk": chunk, "sign": sign, "prec": prec, "K": K,
                              "rel": float(err.norm() / ref.norm()),
                              "bias": float(err.mean() / ref.abs().mean()),
                              "frac_positive_errors": float((err > 0).double().mean())}), flush=True)
    lib.reno_set_split_accumulation_chunk(0)


def run_accuracy(args):
    """max |population(prec) - population(FP64)| after every step, for each
    precision in --accuracy-precs, from the same start state; with
    --envelope also FP64 from the 1-ulp perturbed start against FP64 (the
    size of the FP64 engine's own trajectory spread).  Every step prints one
    JSON line (and appends it to --out)."""
    import torch
    from renormalizer_b200 import Mpo, backend, evolve_batch
    torch.cuda.set_device(0)
    model = holstein_2mode(args.nmol, args.nlev)
    mpo = Mpo(model)
    t0 = time.time()
    mps0 = initial_state(model, args.M, args.start, mpo)
    t_start = time.time() - t0
    precs = [p for p in (args.accuracy_precs or args.prec).split(",") if p and p != "fp64"]
    arms = {p: mps0 for p in precs}
    if args.envelope:
        arms["fp64_ulp"] = perturb_ulp(mps0)
    inject = {f"fp64_inject_{d}": float(d) for d in args.inject.split(",") if d}
    for k in inject:
        arms[k] = mps0
    ref = mps0
    out = open(args.out, "a") if args.out else None
    worst = {k: 0.0 for k in arms}
    step_s = {k: 0.0 for k in list(arms) + ["fp64"]}

    def emit(obj):
        line = json.dumps(obj)
        print(line, flush=True)
        if out:
            out.write(line + "\n")
            out.flush()

    emit({"start": args.start, "start_s": t_start, "bond_dims": mps0.bond_dims, "nmol": args.nmol, "M": args.M,
          "dt": args.dt, "arms": list(arms), "lockstep": bool(args.accuracy_lockstep), "acc_chunk": args.acc_chunk,
          "krylov_tol": args.krylov_tol or "1e-5,1e-8"})
    names = list(arms)
    for step in range(args.accuracy):
        row = {"step": step + 1}
        if args.accuracy_lockstep:
            # every arm and the FP64 reference advance together (evolve_batch):
            # their truncations share the batched eigensolver launches
            t1 = time.time()
            res = evolve_batch([ref] + [arms[k] for k in names], mpo, args.dt,
                               precs=["fp64"] + ["fp64" if k.startswith("fp64_") else k for k in names])
            ref = res[0]
            arms = dict(zip(names, res[1:]))
            for k, d in inject.items():
                arms[k] = perturb_rel(arms[k], d, seed=1000 * (step + 1) + names.index(k))
            step_s["lockstep"] = step_s.get("lockstep", 0.0) + time.time() - t1
            pref = ref.e_occupations
            kref = (ref.evolve_config.stat or {}).get("counts", [])
            for k in names:
                row[k] = float(np.abs(arms[k].e_occupations - pref).max())
                worst[k] = max(worst[k], row[k])
                # local exponentials of this step whose Lanczos stopped at another
                # length than the FP64 reference's
                ka = (arms[k].evolve_config.stat or {}).get("counts", [])
                row[k + "_krylov_mismatch"] = sum(a != b for a, b in zip(ka, kref)) + abs(len(ka) - len(kref))
            emit(row)
            continue
        backend.prec = "fp64"
        t1 = time.time()
        ref = ref.evolve(mpo, args.dt)
        pref = ref.e_occupations
        step_s["fp64"] += time.time() - t1
        for k in arms:
            backend.prec = "fp64" if k.startswith("fp64_") else k
            t1 = time.time()
            arms[k] = arms[k].evolve(mpo, args.dt)
            if k in inject:
                arms[k] = perturb_rel(arms[k], inject[k], seed=1000 * (step + 1) + names.index(k))
            d = float(np.abs(arms[k].e_occupations - pref).max())
            step_s[k] += time.time() - t1
            worst[k] = max(worst[k], d)
            row[k] = d
        emit(row)
    backend.prec = args.prec
    emit({"metric": "max |population(arm) - population(fp64)| over the trajectory", "workload": WORKLOAD,
          "nmol": args.nmol, "M": args.M, "dt": args.dt, "start": args.start, "steps": args.accuracy,
          "max": worst, "s_per_step": {k: v / max(args.accuracy, 1) for k, v in step_s.items() if v}})
    if out:
        out.close()


def run_dmrg(args):
    """Davidson DMRG (gs.optimize_mps, 2-site, one root) of eps = 0, Delta = 1
    and 64 modes from the Ohmic spectral density alpha = 0.5, omega_c = 10
    (Wang1 discretisation), 8 SHO levels (65 sites, real float64), M = 256,
    procedure [[256, .4], [256, .2], [256, .1]] + [[256, 0]] * 8 until the two
    lowest sweep energies agree to 1e-9; the same seeded random start in
    --prec (split matvecs) and in FP64."""
    import torch
    from renormalizer_b200 import Mpo, Mps, Phonon, Quantity, SpectralDensityFunction, SpinBosonModel, backend
    from renormalizer_b200.gs import optimize_mps
    torch.cuda.set_device(0)
    nmodes, nlev, M = 64, 8, 256
    w, c2 = SpectralDensityFunction(0.5, Quantity(10.0)).Wang1(nmodes)
    ph = [Phonon.simple_phonon(Quantity(wi), Quantity(np.sqrt(ci) / wi ** 2), nlev) for wi, ci in zip(w, c2)]
    model = SpinBosonModel(Quantity(0.0), Quantity(1.0), ph)
    mpo = Mpo(model)
    proc = [[M, 0.4], [M, 0.2], [M, 0.1]] + [[M, 0]] * 8
    out = {}
    for prec in (args.prec, "fp64"):
        backend.prec = prec
        np.random.seed(9012)
        mps = Mps.random(model, 0, M)
        mps.optimize_config.procedure = proc
        mps.optimize_config.method = "2site"
        mps.optimize_config.e_atol = 1e-9
        torch.cuda.synchronize()
        t0 = time.time()
        energies, _ = optimize_mps(mps, mpo)
        torch.cuda.synchronize()
        out[prec] = {"energies": [float(e) for e in energies], "seconds": time.time() - t0,
                     "sweeps": len(energies)}
    a, b = out[args.prec], out["fp64"]
    print(json.dumps({"metric": "spin-boson DMRG (65 sites, M=256): lowest energy, split precision vs FP64",
                      "value": a["seconds"] / a["sweeps"], "unit": f"s per sweep ({args.prec})",
                      "fp64_s_per_sweep": b["seconds"] / b["sweeps"], "e_min": {args.prec: min(a["energies"]),
                                                                              "fp64": min(b["energies"])},
                      "e_min_abs_diff": abs(min(a["energies"]) - min(b["energies"])), "runs": out}), flush=True)


def run_heev(args):
    """heev.heev_top against torch.linalg.eigh (cuSOLVER) on G = X X^H / N,
    X seeded complex Gaussian; three timed calls each after one warm-up."""
    import torch
    from renormalizer_b200._native import Engine
    from renormalizer_b200.heev import accepted, heev_top
    torch.cuda.set_device(0)
    eng = Engine.get(0)
    n = args.heev
    kt = 320 if n >= 640 else max(1, n // 2)
    g = torch.Generator(device="cuda").manual_seed(1)
    X = torch.complex(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g),
                      torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    G = X @ X.mH / n

    def timed(f, reps=3):
        f()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            out = f()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps * 1e3, out

    t_ref, (w_ref, _) = timed(lambda: torch.linalg.eigh(G))
    t_dev, (w, K, chk) = timed(lambda: heev_top(eng, G, kt))
    top = torch.flip(w_ref, dims=[0])[:kt]
    # the two QN blocks of a bond in one batched call
    from renormalizer_b200.heev import heev_top_batched
    X2 = torch.complex(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g),
                       torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    G2 = X2 @ X2.mH / n
    t_pair, res2 = timed(lambda: heev_top_batched(eng, [G, G2], [kt, kt]))
    print(json.dumps({"metric": f"Hermitian eigensolver, leading {kt} of {n}x{n} complex128", "unit": "ms",
                      "value": t_dev, "cusolver_eigh_ms": t_ref, "accepted": bool(accepted(chk.cpu().numpy())),
                      "max_eigenvalue_diff_rel": float((w - top).abs().max() / top.abs().max()),
                      "two_blocks_batched_ms": t_pair,
                      "two_blocks_accepted": all(bool(accepted(c.cpu().numpy())) for _, _, c in res2)}), flush=True)


def c4_cases(B, nmol, M, nlev=10, seed=4):
    """Config 4: B static-disorder realisations of an nmol-molecule Holstein
    chain (omega = 1, g = 1, nlev levels); site energies eps_i ~ N(0, 0.5)
    and nearest-neighbour hoppings J (1 + N(0, 0.1)), J = 1, all drawn from
    one seeded generator; bonds capped at M with the 1e-8 singular-value
    threshold (CompressCriteria.both), so they truncate unevenly; start:
    the exciton on molecule 0, bonds expanded with a seeded random expander."""
    from renormalizer_b200 import (CompressConfig, CompressCriteria, EvolveConfig, EvolveMethod, HolsteinModel, Mol,
                                   Mpo, Mps, Phonon, Quantity)
    rng = np.random.default_rng(seed)
    cases = []
    for b in range(B):
        eps = rng.normal(0.0, 0.5, nmol)
        hop = 1.0 * (1.0 + rng.normal(0.0, 0.1, nmol - 1))
        J = np.zeros((nmol, nmol))
        for i in range(nmol - 1):
            J[i, i + 1] = J[i + 1, i] = hop[i]
        ph = [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0)), nlev)]
        model = HolsteinModel([Mol(Quantity(float(e)), ph) for e in eps], J, 3)
        np.random.seed(1000 + b)
        mps = Mps.hartree_product_state(model, {0: 1})
        mps.compress_config = CompressConfig(CompressCriteria.both, threshold=1e-8, max_bonddim=M)
        mps = mps.expand_bond_dimension()
        mps.evolve_config = EvolveConfig(EvolveMethod.tdvp_ps2)
        cases.append((mps, Mpo(model)))
    return cases


def run_batch(args):
    """Config 4 (c4_cases, TDVP-PS2, dt = 0.05): the realisations advanced in
    lockstep by evolve_batch -- grouped FP64 matvecs, lockstep Lanczos, and
    every round's truncations in one batched eigensolver pass -- against the
    same realisations evolved one by one with Mps.evolve.  One warm-up step
    each, then --steps timed lockstep steps of all realisations and --steps
    timed steps of the first --batch-serial realisations one by one;
    realisation-steps per second of both and their populations compared."""
    import torch
    from renormalizer_b200 import backend, evolve_batch
    from renormalizer_b200._native import launch_count
    torch.cuda.set_device(0)
    backend.prec = "fp64"
    B, nmol, M, dt = args.batch, args.batch_nmol, args.batch_M, 0.05
    cases = c4_cases(B, nmol, M)
    mpos = [mpo for _, mpo in cases]
    bat = evolve_batch([m for m, _ in cases], mpos, dt)
    nser = min(args.batch_serial, B)
    seq = [m.evolve(o, dt) for (m, _), o in zip(cases[:nser], mpos[:nser])]
    torch.cuda.synchronize()
    l0 = launch_count()
    t0 = time.time()
    for _ in range(args.steps):
        bat = evolve_batch(bat, mpos, dt)
    torch.cuda.synchronize()
    t_bat = time.time() - t0
    launches = launch_count() - l0
    t0 = time.time()
    for _ in range(args.steps):
        seq = [m.evolve(o, dt) for m, o in zip(seq, mpos[:nser])]
    torch.cuda.synchronize()
    t_seq = time.time() - t0
    dpop = max(float(np.abs(a.e_occupations - b.e_occupations).max()) for a, b in zip(bat[:nser], seq))
    v_bat, v_seq = B * args.steps / t_bat, nser * args.steps / t_seq
    print(json.dumps({"metric": f"TDVP-PS2 realisation-steps/s, {B} static-disorder realisations (config 4)",
                      "value": v_bat, "unit": "realisation-steps/s", "one_by_one_value": v_seq,
                      "speedup_vs_one_by_one": v_bat / v_seq,
                      "config": {"realisations": B, "nmol": nmol, "nlev": 10, "M_cap": M, "threshold": 1e-8,
                                 "dt": dt, "prec": "fp64", "timed_steps": args.steps,
                                 "one_by_one_sample": nser},
                      "bond_dims_max_mean": [int(max(max(m.bond_dims) for m in bat)),
                                             float(np.mean([np.mean(m.bond_dims) for m in bat]))],
                      "max_abs_dpop_lockstep_vs_one_by_one": dpop, "engine_launches_lockstep": launches}),
          flush=True)


def run_grad(args):
    """16 molecules x (e, one mode omega = 1, 10 levels), J = 1, g_i ~ U(0.5, 1.5)
    (seed 5), exciton on molecule 0, bonds expanded to M = 64, 1-site TDVP-PS,
    50 steps of dt = 0.05 (t = 2.5), checkpoints every 10 steps.  Times the
    engine gradient of the site-0 population with respect to all 16 g_i and
    checks every component against torch autograd through FP64 tensordot on
    the same device and against central differences (h = 1e-5 and 1e-4,
    all 32 perturbed trajectories of each h in one batched FP64 run).

    The start is expand_bond_dimension(coef=1e-2) (the seeded random
    expander at weight 1e-2): every bond direction then carries weight far
    above rounding.  With the default coef = 1e-10 the padding directions'
    orientation is set by rounding, the fixed-M trajectory amplifies that to
    ~1e-9 in the population, and QR's backward applies R^-1 across those
    directions; that start is reported beside it (population and the
    engine-vs-autograd spread only)."""
    import torch
    from renormalizer_b200 import CompressConfig, CompressCriteria, HolsteinModel, Mol, Mpo, Mps, Phonon, Quantity, \
        backend
    from renormalizer_b200.tdvp_grad import coupling_gradient, trajectory_values
    torch.cuda.set_device(0)
    backend.prec = "fp64"
    nmol, nlev, M, dt, nsteps = 16, 10, 64, 0.05, 50
    g0 = np.random.default_rng(5).uniform(0.5, 1.5, nmol)

    def model(g):
        mols = [Mol(Quantity(0), [Phonon.simple_phonon(Quantity(1.0), Quantity(np.sqrt(2.0) * gi), nlev)]) for gi in g]
        return HolsteinModel(mols, Quantity(1.0), 3)

    build = lambda g: [Mpo(model(g)).numpy(i) for i in range(2 * nmol)]
    op = np.diag([0.0, 1.0])

    def start(coef):
        np.random.seed(2024)
        mps = Mps.hartree_product_state(model(g0), {0: 1})
        mps.compress_config = CompressConfig(CompressCriteria.fixed, max_bonddim=M)
        mps = mps.expand_bond_dimension(coef=coef)
        mps.ensure_right_canonical()
        return [mps[i] for i in range(len(mps))]

    out = {}
    for coef in (1e-2, 1e-10):
        sites0 = start(coef)
        torch.cuda.synchronize()
        t0 = time.time()
        val, grad = coupling_gradient(build, g0, sites0, dt, nsteps, 0, op, krylov=8, checkpoint_every=10)
        torch.cuda.synchronize()
        t_grad = time.time() - t0
        t0 = time.time()
        val_e, grad_e = coupling_gradient(build, g0, sites0, dt, nsteps, 0, op, krylov=8, checkpoint_every=0,
                                          contract="einsum")
        torch.cuda.synchronize()
        t_einsum = time.time() - t0
        res = {"population": val, "gradient": grad.tolist(), "grad_s": t_grad, "einsum_reference_s": t_einsum,
               "max_abs_diff_vs_einsum_autograd": float(np.abs(grad - grad_e).max()),
               "max_rel_diff_vs_einsum_autograd": float(np.abs(grad - grad_e).max() / np.abs(grad_e).max()),
               "population_vs_einsum": abs(val - val_e)}
        if coef == 1e-2:
            fd = {}
            for h in (1e-5, 1e-4):
                sets = []
                for j in range(nmol):
                    e = np.zeros(nmol)
                    e[j] = h
                    sets += [build(g0 + e), build(g0 - e)]
                t0 = time.time()
                vals = trajectory_values(sets, sites0, dt, nsteps, 0, op, krylov=8)
                fdg = (vals[0::2] - vals[1::2]) / (2 * h)
                fd[f"h{h:g}"] = {"fd": fdg.tolist(), "max_abs_diff": float(np.abs(fdg - grad).max()),
                                 "max_rel_diff": float(np.abs(fdg - grad).max() / np.abs(grad).max()),
                                 "seconds": time.time() - t0}
            res["finite_differences"] = fd
        out[f"coef{coef:g}"] = res
    main = out["coef0.01"]
    print(json.dumps({"metric": "d <n_0>(t=2.5) / d g_i through TDVP-PS (16-molecule Holstein, M=64, 50 steps)",
                      "value": main["grad_s"], "unit": "s per gradient (16 couplings)",
                      "start": "expand_bond_dimension(coef=1e-2), seeded random expander",
                      "runs": out, "checkpoint_every": 10, "krylov_vectors": 8}), flush=True)


def main():
    args = parse()
    if args.cpu_worker:
        cpu_worker(args.cpu_worker)
        return
    if args.dmrg:
        run_dmrg(args)
        return
    if args.grad:
        run_grad(args)
        return
    if args.batch:
        run_batch(args)
        return
    if args.heev:
        run_heev(args)
        return
    import importlib
    importlib.import_module("renormalizer_b200.svd_qn").subspace.min_dim = 1024 if args.truncation == "subspace" else 0
    if args.krylov_tol:
        tol = importlib.import_module("renormalizer_b200.krylov").tolerance
        tol.rtol, tol.atol = (float(x) for x in args.krylov_tol.split(","))
    if args.acc_chunk:
        from renormalizer_b200._native import load_library
        assert load_library().reno_set_split_accumulation_chunk(args.acc_chunk) == 0
    if args.accumulation:
        run_accumulation(args)
        return
    if args.accuracy:
        run_accuracy(args)
        return
    if args.heff_only:
        run_heff_only(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import torch
        import torch.distributed as D
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        D.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = D
    try:
        run_engine(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
