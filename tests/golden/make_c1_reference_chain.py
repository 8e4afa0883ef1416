"""Generate c1_reference_chain.npz: the FP64 Lanczos chain of the 2x2x2 rock-salt workload computed
with the reference's own averaging kernel (run where the reference sources are available).

    make -C oracle ref && python tests/golden/make_c1_reference_chain.py [--procs 8]

Workload: rock-salt 2x2x2 supercell (16 atoms, n = 45 modes), T = 300 K, N = 2000 seeded Gaussian
configurations (seed 0), 384 symmetries (O_h x 8); one bi-conjugate chain of 100 steps from the
seeded random unit perturbation on R^(1) (seed 11, the start of the benchmark's precision check).
The averages are the reference's compiled GetPerturbAverageSym (oracle/_ref, built from
CModules/odd_corr_module.c + LanczosFunctions.c by oracle/Makefile) on `procs` processes, each on a
contiguous configuration slice with the partial sums recombined as the reference's MPI_Allreduce
does (LanczosFunctions.c:2123-2136, 2236-2248); everything around them is the numpy restatement of
apply_full_L / run_FT in oracle/lanczos_oracle.py (DynamicalLanczos.py:3467-3570, 5843-6374).

Stored: the ensemble inputs (X, Y, rho, w, symmetry blocks; eigenvectors inside degenerate blocks
are not unique, so the inputs are kept rather than regenerated), the coefficients a, b, c and
s_norm of every step, and at steps 0, 10, ... the Krylov vectors q_k, p_k with the reference
applies L q_k and L^T p_k (per-step parity of the GPU apply).
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "python-sscha_b200"))

from oracle import lanczos_oracle as LO  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=2)
    ap.add_argument("--N", type=int, default=2000)
    ap.add_argument("--T", type=float, default=300.0)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--backend", default="reference", choices=["reference", "port"])
    ap.add_argument("--out", default=os.path.join(HERE, "c1_reference_chain.npz"))
    a = ap.parse_args()

    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(a.L, T=a.T)
    X, Y, rho = RS.sample_ensemble(s, a.N, seed=0)
    n = s.n_modes
    n_deg = np.array([len(d) for d in s.deg_space], dtype=np.intc)

    # the seeded start of the benchmark's precision check (Lanczos.prepare_random(seed, "R"))
    rng = np.random.default_rng(RS.CHAIN_SEED)
    psi0 = np.zeros(n + n * (n + 1))
    psi0[:n] = rng.standard_normal(n)
    psi0 /= np.linalg.norm(psi0)

    O = LO.OracleLanczos(X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids)
    recorded = {}
    t0 = time.time()
    with LO.SlicedAverages(X, Y, s.w, rho, s.T, s.symmetries, n_deg, s.deg_space, s.blocks_ids,
                           backend=a.backend, procs=a.procs) as avg:
        O.averages = avg
        plain_apply = O.apply_full_L

        def apply_recording(target=None, transpose=False):
            k = len(O.a_coeffs)
            out = plain_apply(target, transpose)
            if k % a.every == 0:
                recorded[(k, bool(transpose))] = (np.array(target, copy=True), out.copy())
            if transpose:
                print(f"step {k:4d} done, {time.time() - t0:8.1f} s", flush=True)
            return out

        O.apply_full_L = apply_recording
        O.psi = psi0.copy()
        O.run_FT(a.steps)
    dt = time.time() - t0
    ks = sorted({k for k, _ in recorded})
    out = dict(L=a.L, N=a.N, T=s.T, steps=a.steps, chain_seed=RS.CHAIN_SEED, backend=a.backend, procs=a.procs,
               seconds=dt, X=X, Y=Y, rho=rho, w=s.w, blocks_ids=s.blocks_ids, n_blocks=len(s.symmetries),
               a=np.array(O.a_coeffs), b=np.array(O.b_coeffs), c=np.array(O.c_coeffs), s_norm=np.array(O.s_norm),
               psi0=psi0, probe_steps=np.array(ks),
               probe_q=np.array([recorded[(k, False)][0] for k in ks]),
               probe_Lq=np.array([recorded[(k, False)][1] for k in ks]),
               probe_p=np.array([recorded[(k, True)][0] for k in ks]),
               probe_pL=np.array([recorded[(k, True)][1] for k in ks]),
               checksum=RS.ensemble_checksum(X, Y, rho))
    for i, (sy, b) in enumerate(zip(s.symmetries, s.deg_space)):
        out[f"sym{i}"] = sy
        out[f"block{i}"] = b
    np.savez_compressed(a.out, **out)
    print(f"{len(O.a_coeffs)} steps in {dt:.0f} s -> {a.out} ({os.path.getsize(a.out)} bytes)")


if __name__ == "__main__":
    main()
