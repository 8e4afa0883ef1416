"""Generate c2_fp64_perturbed_chains.npz: the FP64 chain of the benchmark's precision check run again
with tiny seeded perturbations, to measure how sensitive G(w) of the unconverged chain is to errors
of the size the mixed-precision contractions make.

Same workload and start as tests/golden/c2_fp64_chain.npz (rock-salt 4x4x4, n = 381, N = 10000
configurations from seed 0, T = 300 K, 3072 symmetries, seeded random unit R^(1) start, 200 steps),
with every contraction in FP64.  Chains, advanced together (one batched apply of their L q and
L^T p per step, then the batched FP64 recurrence):
  start_1e-12   the start vector perturbed by a seeded relative 2-norm error of 1e-12, exact applies;
  apply_3e-9    exact start, every apply output perturbed by a seeded Gaussian vector of relative
                2-norm 3e-9 (the per-apply error of bf16x3 on Krylov vectors of this chain);
  apply_3e-10   the same with 3e-10.
Needs a GPU (about 10 minutes on one B200):

    python tests/golden/make_c2_perturbed_chains.py
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "python-sscha_b200"))

CHAINS = (("start_1e-12", 1e-12, 0.0), ("apply_3e-9", 0.0, 3e-9), ("apply_3e-10", 0.0, 3e-10))


def device_chains(ens, psi0, steps, precision, apply_noise, seed=5):
    """Bi-conjugate chains (run_FT semantics, DynamicalLanczos.py:6059-6153) from the rows of psi0,
    with the apply outputs of chain c perturbed by a relative 2-norm error apply_noise[c]."""
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
        ens.apply_full_L(vec, out, tr, opts, precision)
        if float(eps.abs().max()) > 0:
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
    return np.array(coef)     # (steps, nc, 4): a, b, c, s_norm


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--out", default=os.path.join(HERE, "c2_fp64_perturbed_chains.npz"))
    a = ap.parse_args()
    from tdscha_b200 import rocksalt as RS, _native
    s = RS.build_system(4, T=300.0)
    X, Y, rho = RS.sample_ensemble(s, 10000, seed=0)
    ens = _native.DeviceEnsemble(X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids)
    n = s.n_modes
    ln = n + n * (n + 1)
    rng = np.random.default_rng(RS.CHAIN_SEED)       # the start of Lanczos.prepare_random(seed, "R")
    v = np.zeros(ln)
    v[:n] = rng.standard_normal(n)
    v /= np.linalg.norm(v)
    psi0 = np.tile(v, (len(CHAINS), 1))
    prng = np.random.default_rng(123)
    for i, (_, start_eps, _) in enumerate(CHAINS):
        if start_eps > 0:
            g = prng.standard_normal(ln)
            psi0[i] += start_eps * g / np.linalg.norm(g)
    t0 = time.time()
    coef = device_chains(ens, psi0, a.steps, "fp64", np.array([c[2] for c in CHAINS]))
    dt = time.time() - t0
    out = dict(L=4, N=10000, T=300.0, steps=a.steps, chain_seed=RS.CHAIN_SEED, seconds=dt,
               checksum=RS.ensemble_checksum(X, Y, rho), names=np.array([c[0] for c in CHAINS]),
               start_eps=np.array([c[1] for c in CHAINS]), apply_eps=np.array([c[2] for c in CHAINS]))
    for i, (name, _, _) in enumerate(CHAINS):
        out[f"{name}_a"] = coef[:, i, 0]
        out[f"{name}_b"] = coef[:, i, 1]
        out[f"{name}_c"] = coef[:, i, 2]
    np.savez(a.out, **out)
    print(f"{len(CHAINS)} perturbed FP64 chains x {a.steps} steps in {dt:.0f} s -> {a.out}")


if __name__ == "__main__":
    main()
