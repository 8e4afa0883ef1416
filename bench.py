"""Benchmark of the TD-SCHA Lanczos hot path on B200: apply_full_L throughput (apply_L/s).

Workload (default): rock-salt 4x4x4 supercell (128 atoms, n = 381 modes), N = 10000 configurations
at T = 300 K, 3072 symmetry operations (O_h x 64), seeded synthetic ensemble; `--chains` bi-conjugate
Lanczos chains advanced in lockstep, so one step = one batched apply of 2*chains vectors (L q and
L^T p of every chain) + one batched FP64 recurrence launch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision bf16x3] [--chains 8]
  python bench.py --impl reference       # the reference's own C kernel on the host cores
Under torchrun every rank runs its own chains on its own GPU (weak scaling, no collective on the
data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "python-sscha_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

# DRAM bytes (read + write) of one [a|b] contraction launch, keyed by (L, N, chains, precision).
# Captured by ncu on a reduced launch of the same kernel (N = 2500 configurations, symmetry chunk
# of 768, 16 vectors: M = 12288, N = 5000, K = 72832; 4.92e10 B read + written against 5.29e9 B of
# algorithmic operand and output bytes, 9.3x) and scaled to the full launch by its algorithmic bytes
# (2.406e10 B x 9.3).
# On the character-class path: the grouped [a|b] launch of the same system with N = 2500 moved
# 3.05e9 B against 2.92e9 B of algorithmic bytes (1.04x); scaled by the algorithmic bytes of the
# N = 10000 launch (1.033e10 B).
MEASURED_TRAFFIC = {(4, 10000, 8, "bf16x3"): 2.24e11, (4, 10000, 8, "bf16x3", "classes"): 1.08e10}
METRIC = "apply_L/s at 128 atoms N=1e4: mixed+batched vs FP64 GPU at G(w) rel err <=1e-5"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--chains", type=int, default=8)
    ap.add_argument("--L", type=int, default=4)
    ap.add_argument("--N", type=int, default=10000)
    ap.add_argument("--T", type=float, default=300.0)
    ap.add_argument("--k3", type=float, default=-3.0, help="cubic bond coupling, eV/A^3")
    ap.add_argument("--k4", type=float, default=6.0, help="quartic bond coupling, eV/A^4")
    ap.add_argument("--sym-on-gpu", action="store_true",
                    help="project the symmetry operations onto the modes on the GPU (large supercells)")
    ap.add_argument("--accuracy-steps", type=int, default=200)
    ap.add_argument("--perturbed-fp64", action="store_true",
                    help="when no stored FP64 chain matches: run the live FP64 reference chain together with a "
                         "copy whose applies are perturbed by 3e-10 (the sensitivity of G(w) at each step count)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--batch-systems", action="store_true",
                    help="16 chains (3 IR, 6 Raman, 7 random) on each of three uneven rock-salt systems "
                         "(2x2x2 N=2000, 3x3x3 N=5000, 4x4x4 N=10000) in one graph-captured multi-system run")
    ap.add_argument("--batch-steps", type=int, default=150)
    ap.add_argument("--grad", action="store_true",
                    help="gradient of sum_w Im G(w) (64 points 50-350 cm^-1) of one chain w.r.t. the forces, the "
                         "weights and (k3, k4), with finite-difference checks (use with --L 3 --N 5000)")
    ap.add_argument("--grad-steps", type=int, default=50)
    ap.add_argument("--shard-configs", action="store_true",
                    help="strong scaling of one batch of chains: every rank holds a contiguous slice of the "
                         "configurations and each apply all-reduces (f_av, d2v_av) over NCCL")
    ap.add_argument("--fp64-repeats", type=int, default=5,
                    help="timed repeats of the FP64 comparison arm (same batched apply, FP64 contractions)")
    ap.add_argument("--precision-study", action="store_true",
                    help="only the 200-step G(w) / a_n / b_n errors of every mixed precision against FP64")
    return ap.parse_args()


def workload_name(a):
    nat = 2 * a.L ** 3
    return (f"rock-salt {a.L}x{a.L}x{a.L} ({nat} atoms, n={3 * nat - 3}), N={a.N}, T={a.T:g} K, "
            f"k3={a.k3:g} eV/A^3, k4={a.k4:g} eV/A^4, "
            f"O_h x {a.L ** 3} = {48 * a.L ** 3} symmetries, {a.chains} bi-conjugate chains "
            f"(2 x {a.chains} applies per step)")


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's GetPerturbAverageSym (oracle/_ref, compiled from its sources)
# ------------------------------------------------------------------------------------------------
_REF_DATA = {}


def _ref_worker(i):
    d = _REF_DATA
    from oracle import lanczos_oracle as LO
    t0 = time.perf_counter()
    LO.perturb_average_sym(d["X"][i:i + 1], d["Y"][i:i + 1], d["w"], d["rho"][i:i + 1], d["R1"], d["Y1"], d["T"], 1,
                           d["syms"], d["n_deg"], d["degs"], d["bid"], backend=d["backend"], n_threads=1)
    return time.perf_counter() - t0


def cpu_backend():
    """The reference's own kernel (oracle/_ref) when it was compiled here, else the C port."""
    from oracle import lanczos_oracle as LO
    try:
        LO.reference_module()
        return "reference"
    except Exception:
        return "port"


def cpu_reference_timing(system, X, Y, rho, seconds_target=20.0, max_procs=None, backend=None):
    """Time the reference kernel on P host processes, one configuration each (the reference's MPI
    partition: contiguous config slices, LanczosFunctions.c:2123-2136).  Returns (apply/s for the
    full ensemble, cores, sample description).  The per-(configuration, symmetry) cost is O(n^2)
    and the same for every pair, so the full apply time is the sample time x (N N_sym) / pairs.
    Must run before any CUDA context exists in this process (the pool forks)."""
    import multiprocessing as mp
    n = system.n_modes
    rng = np.random.default_rng(7)
    R1 = rng.standard_normal(n) * 1e-3
    Y1 = rng.standard_normal((n, n)) * 1e-3
    Y1 = Y1 + Y1.T
    procs = min(max_procs or min(os.cpu_count() or 1, 64), X.shape[0])
    backend = backend or cpu_backend()
    # bounded sample: a slice of the symmetry group keeps one task near seconds_target on big cells
    per_pair = 6.4e-3 * (n / 381.0) ** 2
    n_sym_sample = int(min(system.n_syms, max(48, seconds_target / per_pair)))
    _REF_DATA.update(X=X, Y=Y, w=system.w, rho=rho, R1=R1, Y1=Y1, T=system.T,
                     syms=[s[:n_sym_sample] for s in system.symmetries],
                     n_deg=np.array([len(d) for d in system.deg_space], dtype=np.intc), degs=system.deg_space,
                     bid=system.blocks_ids, backend=backend)
    ctx = mp.get_context("fork")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        per_task = pool.map(_ref_worker, range(procs))
    wall = time.perf_counter() - t0
    pairs_sample = procs * n_sym_sample
    pairs_full = X.shape[0] * system.n_syms
    t_apply = max(per_task) * pairs_full / pairs_sample
    what = ("reference GetPerturbAverageSym (oracle/_ref, gcc -O2)" if backend == "reference"
            else "C port of GetPerturbAverageSym (oracle/tdscha_oracle.c; the reference kernel is not built here)")
    sample = (f"{what} on {procs} processes x 1 configuration x "
              f"{n_sym_sample} symmetries ({pairs_sample} pairs, {wall:.1f} s wall); one apply = "
              f"{pairs_full} pairs, extrapolated linearly in pairs")
    return 1.0 / t_apply, procs, sample, ("reference" if backend == "reference" else "port")


# ------------------------------------------------------------------------------------------------
def dgemm_peak(torch, n=8192, reps=10):
    """FP64 tensor-core peak measured here the way the bf16 peak is: a torch float64 n^3 matmul
    (cuBLAS DGEMM), CUDA events, best of `reps` after warm-up."""
    a_ = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b_ = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c_ = torch.empty_like(a_)
    for _ in range(2):
        torch.matmul(a_, b_, out=c_)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(reps):
        e0.record()
        torch.matmul(a_, b_, out=c_)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a_, b_, c_
    torch.cuda.empty_cache()
    return {"tflops": 2.0 * n ** 3 / (best / 1e3) / 1e12, "ms": best,
            "basis": f"measured in this run: torch float64 {n}^3 matmul (cuBLAS DGEMM), best of {reps}"}


# ------------------------------------------------------------------------------------------------
def clocks_sampler_start(path):
    try:
        f = open(path, "w")
        p = subprocess.Popen(["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                              "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=f, stderr=subprocess.DEVNULL)
        return p, f
    except Exception:
        return None, None


def clocks_sampler_stop(p, f, path, device_index):
    if p is None:
        return None
    p.terminate()
    try:
        p.wait(timeout=5)
    except Exception:
        p.kill()
    f.close()
    sm, smax, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9 or parts[0] != str(device_index):
            continue
        try:
            sm.append(float(parts[1]))
            smax = float(parts[2])
        except ValueError:
            continue
        for nm, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------------
def run_reference_arm(a, rank):
    if rank != 0:
        return None
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(a.L, T=a.T, k3=a.k3, k4=a.k4)   # host cores only: the pool forks
    X, Y, rho = RS.sample_ensemble(s, a.N, seed=0)
    vals = []
    for _ in range(max(1, a.warmup // 3)):      # untimed warm-up (import + page-in)
        cpu_reference_timing(s, X, Y, rho, seconds_target=2.0, max_procs=min(2, os.cpu_count() or 1))
    cores = 1
    sample = ""
    t0 = time.perf_counter()
    for _ in range(a.steps):
        v, cores, sample, kind = cpu_reference_timing(s, X, Y, rho, seconds_target=8.0)
        vals.append(v)
    wall = time.perf_counter() - t0
    v = float(np.mean(vals))
    applies = 2 * a.chains   # one step of the repo arm: one batched apply of L q and L^T p per chain
    line = {"metric": METRIC, "value": v, "unit": "apply_L/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * applies / v, "higher_is_better": True, "scaling": "weak",
            "applies_per_step": applies, "ms_per_apply": 1e3 / v,
            "ms_note": "ms_per_step and ms_per_apply extrapolated from the bounded sample at the measured rate; "
                       "wall_s is the wall time of this run",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded rock-salt ensemble)",
            "config": {"workload": workload_name(a), "N": a.N, "n_modes": s.n_modes, "N_sym": s.n_syms},
            "impl": "reference",
            # "reference": the reference's own C kernel (oracle/_ref, compiled from its sources);
            # "port": the oracle's C restatement, used only where oracle/_ref was not built
            "reference_kind": kind,
            "cpu_baseline": {"value": v, "unit": "apply_L/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "apply_L/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    return line


# ------------------------------------------------------------------------------------------------
FP64_CHAIN = os.path.join(REPO, "tests", "golden", "c2_fp64_chain.npz")
FP64_PERTURBED = os.path.join(REPO, "tests", "golden", "c2_fp64_perturbed_chains.npz")


def fp64_device_chains(ens, psi0, steps, apply_noise, seed=5):
    """Bi-conjugate FP64 chains (run_FT semantics, DynamicalLanczos.py:6059-6153) from the rows of
    psi0, advanced together; the apply outputs of chain c are moved by a seeded Gaussian vector of
    relative 2-norm apply_noise[c].  Returns (steps, chains, 4): a, b, c, s_norm."""
    import torch
    from tdscha_b200 import _native
    dev = "cuda"
    nc, ln = psi0.shape
    q = torch.as_tensor(psi0, device=dev)
    q = q / q.norm(dim=1, keepdim=True)
    p = q.clone()
    qp, pp = torch.zeros_like(q), torch.zeros_like(q)
    sc = torch.tensor([[0.0, 0.0, 1.0, 0.0, 1.0, 0.0]] * nc, dtype=torch.float64, device=dev)
    opts = _native.ApplyOpts(0, 0, 0, 0, 0, 0.0)
    tr = [0] * nc + [1] * nc
    vec = torch.empty((2 * nc, ln), dtype=torch.float64, device=dev)
    out = torch.empty_like(vec)
    qn, pn = torch.empty_like(q), torch.empty_like(q)
    sc_out = torch.empty((nc, 4), dtype=torch.float64, device=dev)
    eps = torch.as_tensor(np.concatenate([apply_noise, apply_noise]), device=dev)[:, None]
    gen = torch.Generator(device=dev).manual_seed(seed)
    coef = []
    for k in range(steps):
        vec[:nc].copy_(q)
        vec[nc:].copy_(p)
        ens.apply_full_L(vec, out, tr, opts, "fp64")
        g = torch.randn(out.shape, generator=gen, dtype=torch.float64, device=dev)
        out += eps * out.norm(dim=1, keepdim=True) * g / g.norm(dim=1, keepdim=True)
        _native.lanczos_step(out[:nc], out[nc:], q, p, qp, pp, sc, None, qn, pn, sc_out)
        new = torch.empty_like(sc)
        new[:, 0] = sc_out[:, 2]
        new[:, 1] = sc_out[:, 1]
        new[:, 2] = sc_out[:, 3]
        new[:, 3] = sc[:, 2]
        new[:, 4] = sc[:, 0] if k >= 1 else 1.0
        new[:, 5] = k + 1
        qp, pp, q, p, sc = q, p, qn.clone(), pn.clone(), new
        coef.append(sc_out.cpu().numpy().copy())
    return np.array(coef)


def precision_check(a, s, X, Y, rho, ens, precision=None):
    """G(w) of the seeded chain after `accuracy_steps` steps in `precision` (default the benchmark's)
    against the same chain in FP64: the stored FP64 chain when it was made from these inputs, else
    a live run."""
    from tdscha_b200 import rocksalt as RS
    precision = precision or a.precision
    steps = a.accuracy_steps
    ref = None
    if os.path.exists(FP64_CHAIN):
        d = np.load(FP64_CHAIN)
        same = (int(d["L"]) == a.L and int(d["N"]) == a.N and float(d["T"]) == a.T and int(d["steps"]) >= steps
                and np.allclose(d["checksum"], RS.ensemble_checksum(X, Y, rho), rtol=1e-12, atol=0))
        if same:
            ref = {"a": d["a"][:steps], "b": d["b"][:steps], "c": d["c"][:steps], "source": "stored FP64 chain "
                   f"(tests/golden/c2_fp64_chain.npz, {int(d['steps'])} steps, same ensemble checksum)"}
    t0 = time.perf_counter()
    mixed = RS.seeded_chain(s, X, Y, rho, ens, precision, steps)
    t_mixed = time.perf_counter() - t0
    live_perturbed = None
    if ref is None:
        if a.perturbed_fp64:
            # the FP64 chain and, beside it, the same chain with every apply moved by a seeded 3e-10
            # (relative 2-norm), advanced together
            n = s.n_modes
            psi0 = np.zeros(n + n * (n + 1))
            psi0[:n] = np.random.default_rng(RS.CHAIN_SEED).standard_normal(n)
            coef = fp64_device_chains(ens, np.tile(psi0, (2, 1)), steps, np.array([0.0, 3e-10]))
            ref = {"a": coef[:, 0, 0], "b": coef[:, 0, 1], "c": coef[:, 0, 2], "source": "live FP64 chain"}
            live_perturbed = {"apply_3e-10": (coef[:, 1, 0], coef[:, 1, 1], coef[:, 1, 2])}
        else:
            c64 = RS.seeded_chain(s, X, Y, rho, ens, "fp64", steps)
            ref = {"a": np.array(c64.a_coeffs), "b": np.array(c64.b_coeffs), "c": np.array(c64.c_coeffs),
                   "source": "live FP64 chain"}
    w, eta = RS.gf_grid()
    k = min(len(ref["a"]), len(mixed.a_coeffs))
    amx, bmx, cmx = (np.array(x) for x in (mixed.a_coeffs, mixed.b_coeffs, mixed.c_coeffs))

    def gf(av, bv, cv, ns):   # ns steps: a_0..a_{ns-1}, b/c_0..b/c_{ns-2}
        mixed.a_coeffs, mixed.b_coeffs, mixed.c_coeffs = list(av[:ns]), list(bv[:ns - 1]), list(cv[:ns - 1])
        return mixed.get_green_function_continued_fraction(w, use_terminator=False, smearing=eta)

    gmx = gf(amx, bmx, cmx, k)
    g64 = gf(ref["a"], ref["b"], ref["c"], k)
    kk = min(20, k - 1)
    kb = min(k - 1, len(bmx), len(ref["b"]))
    big = np.abs(g64) >= 1e-3 * np.abs(g64).max()      # pointwise errors where |G| is not negligible
    out = {"precision": precision, "steps": k, "omega": "500 points 0-400 cm^-1, smearing 5 cm^-1, no terminator",
           "reference": ref["source"], "mixed_chain_s": round(t_mixed, 1),
           "g_rel_err_max": float(np.abs(gmx - g64).max() / np.abs(g64).max()),
           "g_rel_err_pointwise_median": float(np.median(np.abs(gmx - g64) / np.abs(g64))),
           "g_rel_err_pointwise_max": float(np.max(np.abs(gmx - g64)[big] / np.abs(g64)[big])),
           "g_pointwise_floor": "|G| >= 1e-3 max|G|",
           "a_rel_err_first20_max": float(np.max(np.abs(amx[:kk] - ref["a"][:kk]) / np.abs(ref["a"][:kk]))),
           "b_rel_err_first20_max": float(np.max(np.abs(bmx[:kk] - ref["b"][:kk]) / np.abs(ref["b"][:kk]))),
           "a_rel_err_chain_max": float(np.max(np.abs(amx[:k] - ref["a"][:k]) / np.abs(ref["a"][:k]))),
           "b_rel_err_chain_max": float(np.max(np.abs(bmx[:kb] - ref["b"][:kb]) / np.abs(ref["b"][:kb]))),
           "bound": 1e-5}
    # G(w) error of the truncated chains (the chains resolve new poles at different steps)
    counts = [ns for ns in (25, 50, 100, 150, 200) if ns <= k]

    def by_steps_of(av, bv, cv):
        res = {}
        for ns in counts:
            g_ref = gf(ref["a"], ref["b"], ref["c"], ns)
            res[ns] = float(np.abs(gf(av, bv, cv, ns) - g_ref).max() / np.abs(g_ref).max())
        return res

    def first_divergence(av):   # first step whose a_n differs from the reference chain's by > 1e-6 relative
        kk_ = min(len(av), len(ref["a"]))
        e = np.abs(np.asarray(av[:kk_]) - ref["a"][:kk_]) / np.abs(ref["a"][:kk_])
        idx = np.nonzero(e > 1e-6)[0]
        return int(idx[0]) if len(idx) else None

    out["g_rel_err_max_by_steps"] = by_steps_of(amx, bmx, cmx)
    out["a_first_step_rel_err_above_1e-6"] = first_divergence(amx)
    # the same for FP64 chains with tiny seeded perturbations (start vector 1e-12; every apply
    # 3e-9 / 3e-10 relative): how much any error of that size moves G(w) of the unconverged chain
    if live_perturbed is not None:
        out["fp64_perturbed_g_rel_err_max_by_steps"] = {nm: by_steps_of(*v) for nm, v in live_perturbed.items()}
        out["fp64_perturbed_a_first_step_rel_err_above_1e-6"] = {nm: first_divergence(v[0])
                                                                  for nm, v in live_perturbed.items()}
    if ref["source"].startswith("stored") and os.path.exists(FP64_PERTURBED):
        dp = np.load(FP64_PERTURBED)
        if np.allclose(dp["checksum"], RS.ensemble_checksum(X, Y, rho), rtol=1e-12, atol=0) and int(dp["steps"]) >= k:
            out["fp64_perturbed_g_rel_err_max_by_steps"] = {
                str(nm): by_steps_of(dp[f"{nm}_a"], dp[f"{nm}_b"], dp[f"{nm}_c"]) for nm in dp["names"]}
            out["fp64_perturbed_a_first_step_rel_err_above_1e-6"] = {
                str(nm): first_divergence(dp[f"{nm}_a"]) for nm in dp["names"]}
    return out


# ------------------------------------------------------------------------------------------------
BATCH_SYSTEMS = ((2, 2000, 31), (3, 5000, 32), (4, 10000, 33))   # (L, N, seed), T = 300 K


def batch_chains(base):
    """The 16 chains of one system: IR along x, y, z (seeded Born charges), Raman for the six
    (in, out) polarisation pairs xx yy zz xy yz xz (seeded Raman tensors), 7 seeded random unit
    vectors on R^(1)."""
    e = np.eye(3)
    chains = []
    for pol in e:
        L = base.new_chain()
        L.prepare_ir(pol_vec=pol)
        chains.append(L)
    for i, j in ((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)):
        L = base.new_chain()
        L.prepare_raman(pol_vec_in=e[i], pol_vec_out=e[j])
        chains.append(L)
    for sd in range(7):
        L = base.new_chain()
        L.prepare_random(seed=100 + sd, sector="R")
        chains.append(L)
    return chains


def run_batch_systems(a):
    """Throughput of 48 chains (16 per system) over three uneven systems advanced together by
    tdscha_lanczos_run_device (two eager steps, then one CUDA graph holding all remaining steps), against the
    host-driven per-system loop; G(w) error of the mixed chains against FP64 on the two small
    systems."""
    import torch
    from tdscha_b200 import DynamicalLanczos as DL
    from tdscha_b200 import rocksalt as RS
    bases, names = [], []
    for L_, N_, seed in BATCH_SYSTEMS:
        ens = RS.make_ensemble(L_, N_, T=300.0, seed=seed)
        b = DL.Lanczos(ens)
        b.init()
        bases.append(b)
        names.append(f"{L_}x{L_}x{L_} (n={b.n_modes}) N={N_} N_sym={b.n_syms}")
    steps = a.batch_steps
    prec = a.precision
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # warm-up (untimed): tunes the contraction tiles, allocates the workspaces
    DL.run_FT_multi([batch_chains(b) for b in bases], max(a.warmup, 3), precision=prec, use_graph=True)
    groups = [batch_chains(b) for b in bases]
    smi_path = os.path.join(REPO, ".bench_clocks_batch.csv")
    sp, sf = clocks_sampler_start(smi_path)
    torch.cuda.synchronize()
    e0.record(stream)
    DL.run_FT_multi(groups, steps, precision=prec, use_graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clocks_sampler_stop(sp, sf, smi_path, 0)
    try:
        os.remove(smi_path)
    except OSError:
        pass
    ms = e0.elapsed_time(e1)
    n_chains = sum(len(g) for g in groups)
    applies = 2 * n_chains * steps
    lengths = {names[i]: [len(L.a_coeffs) for L in g] for i, g in enumerate(groups)}
    # comparisons on a short run: the same run without the graph, and the host-driven loop
    cmp_steps = 20
    cmp = {}
    for label, fn in (("multi_no_graph", lambda gs: DL.run_FT_multi(gs, cmp_steps, precision=prec, use_graph=False)),
                      ("multi_graph", lambda gs: DL.run_FT_multi(gs, cmp_steps, precision=prec, use_graph=True)),
                      ("host_loop_per_system", lambda gs: [DL.run_FT_batched(g, cmp_steps, precision=prec) for g in gs])):
        gs = [batch_chains(b) for b in bases]
        torch.cuda.synchronize()
        e0.record(stream)
        fn(gs)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        cmp[label] = {"ms": round(t, 1), "apply_L_per_s": 2 * n_chains * cmp_steps / (t / 1e3)}
    # accuracy of the mixed chains (first `steps` steps) against FP64 chains, small systems
    w, eta = RS.gf_grid()
    acc = {}
    for i in range(2):
        ref = batch_chains(bases[i])
        DL.run_FT_multi([ref], steps, precision="fp64", use_graph=True)
        errs = []
        for Lm, Lr in zip(groups[i], ref):
            k = min(len(Lm.a_coeffs), len(Lr.a_coeffs))
            gm = _gf_truncated(Lm, k, w, eta)
            gr = _gf_truncated(Lr, k, w, eta)
            errs.append(float(np.abs(gm - gr).max() / np.abs(gr).max()))
        acc[names[i]] = {"g_rel_err_max_over_chains": max(errs), "g_rel_err_median_over_chains": float(np.median(errs))}
    acc[names[2]] = ("not compared here (16 FP64 chains of 150 steps); at 150 steps the 4x4x4 chains are not "
                     "converged: see the default run's accuracy_vs_fp64, whose FP64 chain perturbed by 3e-10 per apply "
                     "is off by as much as bf16x3 at 150 steps")
    line = {"metric": "apply_L/s, 48 chains over three uneven systems, one graph-captured run", "value": applies / (ms / 1e3),
            "unit": "apply_L/s", "n_gpus": 1, "steps": steps, "warmup": max(a.warmup, 3), "ms_total": ms,
            "higher_is_better": True, "dtype": f"{prec} contractions (f32 accumulate) + f64 recurrence",
            "data": "synthetic (seeded rock-salt ensembles, T = 300 K)",
            "config": {"workload": "16 chains (3 IR, 6 Raman, 7 random R1) on each of " + "; ".join(names),
                       "graph": "2 eager steps, then one CUDA graph launch holding every remaining step of all systems",
                       "streams": "one per system, forked from and joined into the run's stream"},
            "chain_lengths": lengths, "comparison_20_steps": cmp, "accuracy_vs_fp64": acc, "clocks": clocks}
    print(json.dumps(line))


def run_grad(a):
    """dG/d(Y, rho, k3, k4) of one seeded chain (checkpoint every 10 steps) through the hand-written
    adjoint: time per gradient with FP64 contractions and with the benchmark's mixed precision in
    the applies and in the averages' vector-Jacobian product (recurrence, continued fraction and the
    VJP's own algebra FP64 in both), and the mixed gradient against the FP64 one.  Finite-difference
    checks of the FP64 value (Richardson-extrapolated central differences along random directions
    of Y and rho and along k3, k4) run on a 12-step chain; on the configured 50-step chain central
    differences at h and h/2 along Y are reported side by side: there the chain has started to
    resolve its spectrum and G(w) at a fixed step count is too sensitive to its inputs for finite
    differences to converge."""
    import torch
    from tdscha_b200 import adjoint
    from tdscha_b200 import DynamicalLanczos as DL
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(a.L, T=a.T, k3=a.k3, k4=a.k4)
    X, Y3, Y4, rho = RS.sample_force_components(s, a.N, seed=0)
    k3, k4 = s.k3, s.k4
    Y = k3 * Y3 + k4 * Y4
    w = np.linspace(50.0, 350.0, 64) / RS.RY_TO_CM
    eta = 5.0 / RS.RY_TO_CM

    def lanczos(Yv, rv):
        ens = RS.SyntheticEnsemble(T=s.T, nat=s.nat, m=s.masses, w=s.w, pols=s.pols, N=len(rv), rho=rv, X=X, Y=Yv,
                                   symmetries=s.symmetries, deg_space=s.deg_space, blocks_ids=s.blocks_ids,
                                   supercell=(a.L,) * 3)
        L = DL.Lanczos(ens)
        L.init()
        L.prepare_random(seed=RS.CHAIN_SEED, sector="R")
        return L

    base = lanczos(Y, rho)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def gradient(prec, steps):
        Yt = torch.tensor(Y, device="cuda", requires_grad=True)
        rt = torch.tensor(rho, device="cuda", requires_grad=True)
        torch.cuda.synchronize()
        e0.record()
        G = adjoint.green_function(base, w, eta, steps, Yt, rt, checkpoint_every=10, precision=prec)
        gY, gr = torch.autograd.grad(G.imag.sum(), (Yt, rt))
        e1.record()
        torch.cuda.synchronize()
        return {"G": G.detach().cpu().numpy(), "gY": gY.cpu().numpy(), "gr": gr.cpu().numpy(), "ms": e0.elapsed_time(e1)}

    def rel(x, y):
        return float(np.abs(x - y).max() / np.abs(y).max())

    res, cmp = {}, {}
    for steps in (a.grad_steps, 12):
        r = {}
        for prec in ("fp64", a.precision):
            if steps == a.grad_steps:
                gradient(prec, steps)                    # warm-up: tiles, workspaces
            r[prec] = gradient(prec, steps)
        res[steps] = r
        cmp[steps] = {"G_rel_err_max": rel(r[a.precision]["G"], r["fp64"]["G"]),
                      "dY_rel_err_max": rel(r[a.precision]["gY"], r["fp64"]["gY"]),
                      "drho_rel_err_max": rel(r[a.precision]["gr"], r["fp64"]["gr"])}

    def value(Yv, rv, steps):
        L = lanczos(Yv, rv)
        with torch.no_grad():
            v = adjoint.green_function(L, w, eta, steps, torch.as_tensor(Yv, device="cuda"),
                                       torch.as_tensor(rv, device="cuda")).imag.sum()
        out = float(v)
        L.device_ensemble.close()
        return out

    def central(f, h):
        return (f(h) - f(-h)) / (2 * h)

    def richardson(f, h):
        return (4 * central(f, h / 2) - central(f, h)) / 3

    rng = np.random.default_rng(17)
    dY = rng.standard_normal(Y.shape)
    dr = rng.standard_normal(rho.shape) * 0.1
    hY = 1e-4 * np.abs(Y).max()
    g12 = res[12]["fp64"]
    checks = {
        "Y_direction": (float((g12["gY"] * dY).sum()), richardson(lambda t: value(Y + t * dY, rho, 12), hY)),
        "rho_direction": (float((g12["gr"] * dr).sum()), richardson(lambda t: value(Y, rho + t * dr, 12), 1e-3)),
        "k3": (adjoint.force_gradient_to_k(g12["gY"], Y3, Y4)[0],
               richardson(lambda t: value((k3 + t) * Y3 + k4 * Y4, rho, 12), 1e-3 * abs(k3))),
        "k4": (adjoint.force_gradient_to_k(g12["gY"], Y3, Y4)[1],
               richardson(lambda t: value(k3 * Y3 + (k4 + t) * Y4, rho, 12), 1e-3 * abs(k4))),
    }
    fd = {k: {"adjoint": v[0], "finite_difference": v[1], "rel_err": abs(v[0] - v[1]) / abs(v[1])}
          for k, v in checks.items()}
    gL = res[a.grad_steps]["fp64"]
    fY = lambda t: value(Y + t * dY, rho, a.grad_steps)   # noqa: E731
    long_chain = {"adjoint": float((gL["gY"] * dY).sum()), "central_h": central(fY, hY),
                  "central_h_over_2": central(fY, hY / 2), "h": hY}
    gm = res[a.grad_steps][a.precision]
    line = {"metric": "gradient of sum_w Im G(w) w.r.t. forces, weights and (k3, k4): ms per gradient",
            "value": gm["ms"], "unit": "ms", "higher_is_better": False, "n_gpus": 1,
            "dtype": f"{a.precision} contractions in the applies and the VJP; f64 recurrence, continued fraction",
            "data": "synthetic (seeded rock-salt ensemble)",
            "config": {"workload": f"rock-salt {a.L}x{a.L}x{a.L} (n={s.n_modes}), N={a.N}, T={a.T:g} K, "
                                   f"{s.n_syms} symmetries, {a.grad_steps} Lanczos steps, checkpoint every 10, "
                                   "64 frequencies 50-350 cm^-1, smearing 5 cm^-1",
                       "objective": "sum over the 64 frequencies of Im G(w)"},
            "ms_per_gradient": {p: round(r["ms"], 1) for p, r in res[a.grad_steps].items()},
            "ms_per_gradient_12_steps": {p: round(r["ms"], 1) for p, r in res[12].items()},
            "mixed_vs_fp64": {f"{k}_steps": v for k, v in cmp.items()},
            "finite_differences_fp64_12_steps": fd,
            f"finite_differences_fp64_{a.grad_steps}_steps_Y_direction": long_chain,
            "dk": {"dG_dk3": checks["k3"][0], "dG_dk4": checks["k4"][0], "units": "per internal Ry/Bohr^n coupling"}}
    print(json.dumps(line))


def run_sharded(a, rank, world, local_rank):
    """Configuration-sharded apply_full_L (tdscha_b200.parallel.ShardedEnsemble): the `chains` chains'
    2 x chains vectors are replicated on every rank, each rank averages over its slice of the N
    configurations (the reference's MPI partition, LanczosFunctions.c:2123-2136) and one NCCL
    all-reduce of (f_av, d2v_av) per batched apply sums the slices (its MPI_Allreduce, :2237).  The
    total work is fixed: strong scaling."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from tdscha_b200 import _native
    from tdscha_b200 import rocksalt as RS
    from tdscha_b200.parallel import ShardedEnsemble
    s = RS.build_system(a.L, T=a.T, k3=a.k3, k4=a.k4, symmetries_on_gpu=a.sym_on_gpu)
    X, Y, rho = RS.sample_ensemble(s, a.N, seed=0)
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    sh = ShardedEnsemble(X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids) if world > 1 else None
    ens = sh.local if sh is not None else _native.DeviceEnsemble(X, Y, s.w, rho, s.T, s.symmetries, s.deg_space,
                                                                 s.blocks_ids)
    n = s.n_modes
    ln = n + n * (n + 1)
    nb = 2 * a.chains
    gen = torch.Generator(device="cpu").manual_seed(1000)
    vec = torch.randn(nb, ln, generator=gen, dtype=torch.float64).to(f"cuda:{local_rank}")
    out = torch.empty_like(vec)
    tr = [0] * a.chains + [1] * a.chains
    opts = _native.ApplyOpts(0, 0, 0, 0, 0, 0.0)

    def apply():
        if sh is not None:
            sh.apply_full_L(vec, out, tr, opts, a.precision)
        else:
            ens.apply_full_L(vec, out, tr, opts, a.precision)

    for _ in range(a.warmup):
        apply()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        apply()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if rank == 0:
        value = nb * a.steps / (ms / 1e3)
        print(json.dumps({"metric": "apply_L/s, one batch of chains over configuration shards", "value": value,
                          "unit": "apply_L/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                          "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": f"{a.precision} contractions + f64 all-reduce",
                          "data": "synthetic (seeded rock-salt ensemble)",
                          "config": {"workload": workload_name(a), "parallelism": f"configuration shards x{world}, "
                                     "NCCL all-reduce of n + n^2 FP64 per vector per apply",
                                     "configs_per_rank": a.N // world}}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _gf_truncated(L, k, w, eta):
    a, b, c = list(L.a_coeffs), list(L.b_coeffs), list(L.c_coeffs)
    L.a_coeffs, L.b_coeffs, L.c_coeffs = a[:k], b[:k - 1], c[:k - 1]
    g = L.get_green_function_continued_fraction(w, use_terminator=False, smearing=eta)
    L.a_coeffs, L.b_coeffs, L.c_coeffs = a, b, c
    return g


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        line = run_reference_arm(a, rank)
        if line is not None:
            print(json.dumps(line))
        return

    if a.shard_configs:
        run_sharded(a, rank, world, local_rank)
        return

    if a.grad:
        import torch
        torch.cuda.set_device(local_rank)
        if rank == 0:
            run_grad(a)
        return

    if a.batch_systems:
        import torch
        torch.cuda.set_device(local_rank)
        if rank == 0:
            run_batch_systems(a)
        return

    from tdscha_b200 import rocksalt as RS

    # CPU baseline first (spawned processes, before any CUDA context): rank 0 at N = 1 only
    s = RS.build_system(a.L, T=a.T, k3=a.k3, k4=a.k4, symmetries_on_gpu=a.sym_on_gpu)
    X, Y, rho = RS.sample_ensemble(s, a.N, seed=0)
    cpu_base = None
    if a.sym_on_gpu and not a.no_cpu_baseline:
        # the baseline's process pool forks, which is unsafe once the symmetry build opened a CUDA context
        cpu_base = {"value": None, "unit": "apply_L/s", "cores": 0, "kind": "reference",
                    "sample": "skipped: --sym-on-gpu opens a CUDA context before the forking process pool"}
    elif rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            v, cores, sample, kind = cpu_reference_timing(s, X, Y, rho)
            cpu_base = {"value": v, "unit": "apply_L/s", "cores": cores, "kind": kind, "sample": sample}
        except Exception as ex:   # reference kernel not built on this machine
            cpu_base = {"value": None, "unit": "apply_L/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {ex}"}

    import torch
    import torch.distributed as dist
    from tdscha_b200 import _native

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    ens = _native.DeviceEnsemble(X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids)
    if a.precision_study:
        if rank == 0:
            res = [precision_check(a, s, X, Y, rho, ens, p) for p in ("bf16x3", "tf32x3", "tf32", "bf16")]
            print(json.dumps({"precision_study": workload_name(a), "results": res}))
        return
    n = s.n_modes
    ln = n + n * (n + 1)
    nc = a.chains
    nb = 2 * nc
    opts = _native.ApplyOpts(0, 0, 0, 0, 0, 0.0)
    gen = torch.Generator(device="cpu").manual_seed(1000 + rank)
    q0 = torch.randn(nc, ln, generator=gen, dtype=torch.float64)
    q0 /= q0.norm(dim=1, keepdim=True)
    dev = f"cuda:{local_rank}"
    stream = torch.cuda.current_stream()

    state = {}

    def reset_chains():
        state["q"] = q0.to(dev).contiguous()
        state["p"] = state["q"].clone()
        state["qp"] = torch.zeros_like(state["q"])
        state["pp"] = torch.zeros_like(state["q"])
        state["sc"] = torch.tensor([[0.0, 0.0, 1.0, 0.0, 1.0, 0.0]] * nc, dtype=torch.float64, device=dev)
        state["k"] = 0

    vec = torch.empty((nb, ln), dtype=torch.float64, device=dev)
    out = torch.empty_like(vec)
    qn = torch.empty((nc, ln), dtype=torch.float64, device=dev)
    pn = torch.empty_like(qn)
    sc_out = torch.empty((nc, 4), dtype=torch.float64, device=dev)
    tr = [0] * nc + [1] * nc

    def step(prec):
        """One bi-conjugate step of every chain: batched apply of [q; p] + batched recurrence."""
        vec[:nc].copy_(state["q"])
        vec[nc:].copy_(state["p"])
        ens.apply_full_L(vec, out, tr, opts, prec)
        _native.lanczos_step(out[:nc], out[nc:], state["q"], state["p"], state["qp"], state["pp"], state["sc"], None,
                             qn, pn, sc_out)
        # history for the next step (device-side scalar bookkeeping, no host sync)
        k = state["k"]
        sc_prev = state["sc"]
        new = torch.empty_like(sc_prev)
        new[:, 0] = sc_out[:, 2]                      # c_k
        new[:, 1] = sc_out[:, 1]                      # b_k
        new[:, 2] = sc_out[:, 3]                      # s_norm_{k+1}
        new[:, 3] = sc_prev[:, 2]                     # s_norm_k
        new[:, 4] = sc_prev[:, 0] if k >= 1 else 1.0  # c_{k-1}
        new[:, 5] = k + 1
        state["qp"], state["pp"] = state["q"], state["p"]
        state["q"], state["p"] = qn.clone(), pn.clone()
        state["sc"] = new
        state["k"] = k + 1

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------- device-resident throughput ----------------
    reset_chains()
    for _ in range(a.warmup):
        step(a.precision)
    ens.read_profile()
    ens.set_profiling(True)
    smi_path = os.path.join(REPO, f".bench_clocks_{rank}.csv")
    sp, sf = clocks_sampler_start(smi_path)
    # the bounded-wait error word is read once after the timed steps instead of after every apply
    # (no host synchronisation inside the step loop)
    _native.set_error_check(False)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step(a.precision)
    e1.record(stream)
    barrier()
    _native.check_errors(ens.handle)
    clocks = clocks_sampler_stop(sp, sf, smi_path, local_rank)
    try:
        os.remove(smi_path)
    except OSError:
        pass
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    prof = ens.read_profile()
    ens.set_profiling(False)
    applies = nb * a.steps * world
    value = applies / (ms_total / 1e3)
    launches = sum(c for _, c in prof.values()) + 3 * a.steps          # + 3 recurrence kernels per step

    # roofline of the dominant contraction ([a | b] projection, K = n(n+1)/2).  On the character-class
    # path its executed work is flops_ratio x that of the contraction over every symmetry row.
    P = n * (n + 1) // 2
    ab_ms, ab_launches = prof["gemm_ab"]
    cls = ens.classes()
    ratio = cls["flops_ratio"] if cls["n_class"] else 1.0
    flops_ab_per_apply = 2.0 * s.n_syms * (2 * a.N) * P * ratio        # = 2 N N_sym n(n+1) ~ 2 M n^2 (x ratio)
    flops_per_launch = flops_ab_per_apply * nb * a.steps / max(ab_launches, 1)
    t_launch = ab_ms / 1e3 / max(ab_launches, 1)
    peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(REPO, "MEASURED_PEAKS.json")) else {}
    # the contraction runs back to back inside a seconds-long step: the sustained (power-capped) peak
    bf16_peak = peaks.get("bf16_tflops_sustained", 1400.0)
    peak_src = "of measured" if "bf16_tflops_sustained" in peaks else "of fallback"
    nprod = 3 if a.precision.endswith("x3") else 1
    rate_div = {"bf16": 1.0, "tf32": 2.0}[a.precision[:4]] * nprod
    achieved = flops_per_launch / t_launch / 1e12
    if cls["n_class"]:
        kernel = (f"tc_gemm_kernel, grouped: [a|b] over {cls['n_class']} character classes of the translation subgroup "
                  f"(executed work {ratio:.4f} x the contraction over all {s.n_syms} symmetry rows)")
        traffic = MEASURED_TRAFFIC.get((a.L, a.N, a.chains, a.precision, "classes"))
        tnote = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the grouped [a|b] launch at N = 2500 (1.04x its "
                 "algorithmic bytes), scaled by the algorithmic bytes of this launch")
    else:
        kernel = "tc_gemm_kernel ([a|b] = Y~ . V^T projection)"
        traffic = MEASURED_TRAFFIC.get((a.L, a.N, a.chains, a.precision))
        tnote = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of a reduced [a|b] launch (M 12288, N 5000, K 72832: "
                 "9.3x its algorithmic bytes), scaled to this launch by algorithmic bytes "
                 f"{(nb * s.n_syms + 2 * a.N) * P * 4 + nb * s.n_syms * 2 * a.N * 4:.3e}")
    roofline = {"kernel": kernel, "bound": "tensor",
                "achieved": achieved, "peak": bf16_peak / rate_div, "unit": "TFLOP/s",
                "frac": achieved / (bf16_peak / rate_div),
                "traffic": traffic, "traffic_note": tnote,
                "peak_basis": f"{peak_src} bf16 dense sustained {bf16_peak} TFLOP/s / {rate_div:g} "
                              f"({nprod} product(s){', tf32 at half the bf16 rate' if a.precision.startswith('tf32') else ''})",
                "algorithmic_flops_per_launch": flops_per_launch, "avg_launch_ms": t_launch * 1e3}
    total_prof = sum(v for v, _ in prof.values()) or 1.0
    stage_share = {k: round(v / total_prof, 4) for k, (v, _) in prof.items()}

    # ---------------- end to end through the host-buffer API ----------------
    host_in = torch.empty((nb, ln), dtype=torch.float64).pin_memory()
    host_out = torch.empty((nb, ln), dtype=torch.float64).pin_memory()
    host_in.copy_(vec.cpu())
    barrier()
    for _ in range(2):
        vec.copy_(host_in, non_blocking=True)
        ens.apply_full_L(vec, out, tr, opts, a.precision)
        host_out.copy_(out, non_blocking=True)
    barrier()
    e0.record(stream)
    for _ in range(a.steps):
        vec.copy_(host_in, non_blocking=True)
        ens.apply_full_L(vec, out, tr, opts, a.precision)
        host_out.copy_(out, non_blocking=True)
    e1.record(stream)
    barrier()
    _native.check_errors(ens.handle)
    _native.set_error_check(True)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e = {"value": applies / (e2e_ms / 1e3), "unit": "apply_L/s", "h2d_bytes_per_step": nb * ln * 8,
           "d2h_bytes_per_step": nb * ln * 8}

    # ---------------- FP64 GPU path (the comparison arm of the metric) ----------------
    # the same batched apply of the same 2 x chains vectors with FP64 contractions, repeated
    fp64 = None
    fp64_value = None
    if rank == 0 and a.fp64_repeats > 0:
        dgemm = dgemm_peak(torch)
        ens.apply_full_L(vec, out, tr, opts, "fp64")                 # warm-up (workspace, operands)
        ens.read_profile()
        ens.set_profiling(True)
        smi64 = os.path.join(REPO, f".bench_clocks_fp64_{rank}.csv")
        sp64, sf64 = clocks_sampler_start(smi64)
        torch.cuda.synchronize()
        times = []
        for _ in range(a.fp64_repeats):
            e0.record(stream)
            ens.apply_full_L(vec, out, tr, opts, "fp64")
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        clocks64 = clocks_sampler_stop(sp64, sf64, smi64, local_rank)
        try:
            os.remove(smi64)
        except OSError:
            pass
        prof64 = ens.read_profile()
        ens.set_profiling(False)
        ms_med = float(np.median(times))
        fp64_value = nb / (ms_med / 1e3)
        # the two big contractions ([a|b] and Z, cuBLAS DGEMM in this mode) per apply
        flops_big = 2 * 2.0 * s.n_syms * (2 * a.N) * P * ratio
        big_ms = (prof64["gemm_ab"][0] + prof64["gemm_z"][0]) / a.fp64_repeats
        fp64 = {"value": fp64_value, "unit": "apply_L/s", "applies_per_repeat": nb, "repeats": a.fp64_repeats,
                "ms_per_repeat": [round(t, 2) for t in times], "ms_median": ms_med, "clocks": clocks64,
                "stage_share": {k: round(v / (sum(x for x, _ in prof64.values()) or 1.0), 4) for k, (v, _) in prof64.items()},
                "roofline": {"kernel": "[a|b] + Z contractions (cuBLAS DGEMM)", "bound": "tensor (FP64 DMMA)",
                             "achieved": flops_big * nb / (big_ms / 1e3) / 1e12, "peak": dgemm["tflops"],
                             "unit": "TFLOP/s", "frac": flops_big * nb / (big_ms / 1e3) / 1e12 / dgemm["tflops"],
                             "peak_basis": dgemm["basis"]},
                "whole_apply_tflops": flops_big * nb / (ms_med / 1e3) / 1e12}

    # ---------------- G(w) accuracy of the mixed chain vs the FP64 chain ----------------
    accuracy = None
    if rank == 0 and not a.no_accuracy and a.accuracy_steps > 0:
        accuracy = precision_check(a, s, X, Y, rho, ens)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "apply_L/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_total / a.steps, "higher_is_better": True, "scaling": "weak",
                "applies_per_step": nb, "ms_per_apply": ms_total / a.steps / nb,   # per GPU
                "vs_baseline": None, "dtype": f"{a.precision} contractions (f32 accumulate) + f64 recurrence",
                "data": "synthetic (seeded rock-salt ensemble)",
                "config": {"workload": workload_name(a), "N": a.N, "n_modes": n, "N_sym": s.n_syms, "chains": nc,
                           "applies_per_step_per_gpu": nb, "precision": a.precision,
                           "symmetry_path": (f"{cls['n_class']} character classes of the translation subgroup x coset "
                                             "representatives" if cls["n_class"] else "every symmetry row"),
                           "l2": "inputs larger than L2 (ensemble operands several GB per precision)",
                           "parallelism": f"replicas x{world} (independent chains per GPU)"},
                "roofline": roofline, "cpu_baseline": cpu_base, "e2e": e2e, "gpu_launches": launches,
                "error_check": "bounded-wait error word read after each timed loop (tdscha_check_errors: ok)",
                "clocks": clocks, "fp64_gpu_value": fp64_value, "fp64_gpu": fp64,
                "ratio_vs_fp64_gpu": (value / world) / fp64_value if fp64_value else None,
                "accuracy_vs_fp64": accuracy, "stage_share": stage_share,
                "stage_ms": {k: round(v, 3) for k, (v, _) in prof.items()}}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
