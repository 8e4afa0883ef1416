"""Generate c2_fp64_chain.npz: the FP64 reference chain of the benchmark's precision check.

The benchmark workload (rock-salt 4x4x4, n = 381, N = 10000 configurations from seed 0, T = 300 K,
3072 symmetries) runs one bi-conjugate chain from the seeded random R^(1) start for 200 steps in
FP64 on the GPU (every FP64 apply matches the reference kernel to ~1e-12 relative in the parity
tests).  The file stores its a/b/c coefficients and a checksum of the sampled ensemble, so that a
mixed-precision chain can be compared against it without re-running the 200 FP64 steps (about
3.5 minutes on one B200).  Needs a GPU:

    python tests/golden/make_c2_fp64_chain.py --out tests/golden/c2_fp64_chain.npz
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "python-sscha_b200"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=4)
    ap.add_argument("--N", type=int, default=10000)
    ap.add_argument("--T", type=float, default=300.0)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--out", default=os.path.join(HERE, "c2_fp64_chain.npz"))
    a = ap.parse_args()
    from tdscha_b200 import rocksalt as RS, _native
    s = RS.build_system(a.L, T=a.T)
    X, Y, rho = RS.sample_ensemble(s, a.N, seed=0)
    ens = _native.DeviceEnsemble(X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids)
    t0 = time.time()
    lanc = RS.seeded_chain(s, X, Y, rho, ens, "fp64", a.steps)
    dt = time.time() - t0
    np.savez(a.out, L=a.L, N=a.N, T=a.T, steps=a.steps, chain_seed=RS.CHAIN_SEED,
             checksum=RS.ensemble_checksum(X, Y, rho), a=np.array(lanc.a_coeffs), b=np.array(lanc.b_coeffs),
             c=np.array(lanc.c_coeffs), seconds=dt)
    print(f"{len(lanc.a_coeffs)} FP64 steps in {dt:.1f} s -> {a.out}")


if __name__ == "__main__":
    main()
