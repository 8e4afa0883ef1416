"""Generate the golden fixtures in tests/golden/ (run here, where the reference is mounted).

    python tests/golden/make_golden.py     # needs the reference sources ($TDSCHA_REFERENCE) and `make -C oracle ref`

mode10.npz
    The reference's own test system (tests/test_lanczos_fast/test_c_code_lanczos/mode10.*: the exact
    inputs of its C driver) with the coefficients of its Lanczos run
    (tests/test_lanczos_fast/normal/LANCZOS_STEP10.npz: a, b, c, s_norm and the first Krylov vector),
    plus outputs of the reference's compiled GetPerturbAverageSym (CModules/odd_corr_module.c:491-634)
    for seeded perturbations.
rocksalt_L2.npz
    A seeded 2x2x2 rock-salt ensemble (N = 6, 384 symmetries) from tdscha_b200.rocksalt, stored
    with its inputs (eigenvectors inside degenerate blocks are not unique, so the inputs are kept
    rather than regenerated), plus reference-kernel outputs for seeded perturbations.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "python-sscha_b200"))

from oracle import lanczos_oracle as LO  # noqa: E402

REF = os.path.join(os.environ.get("TDSCHA_REFERENCE", "/root/reference"), "tests", "test_lanczos_fast")


def load_mode10():
    D = os.path.join(REF, "test_c_code_lanczos")
    ndegs = np.loadtxt(os.path.join(D, "mode10.ndegs"), dtype=np.intc)
    blocks = [np.atleast_1d(np.loadtxt(os.path.join(D, f"mode10.block{i}"), dtype=np.intc)) for i in range(len(ndegs))]
    syms = [np.loadtxt(os.path.join(D, f"mode10.symsb{i}")).reshape(-1, d, d) for i, d in enumerate(ndegs)]
    return dict(X=np.loadtxt(os.path.join(D, "mode10.X.dat")), Y=np.loadtxt(os.path.join(D, "mode10.Y.dat")),
                w=np.loadtxt(os.path.join(D, "mode10.freqs")), rho=np.loadtxt(os.path.join(D, "mode10.rho")),
                blocks_ids=np.loadtxt(os.path.join(D, "mode10.blockid"), dtype=np.intc), syms=syms, blocks=blocks,
                T=250.0)


def averages_cases(d, seed):
    n = d["X"].shape[1]
    rng = np.random.default_rng(seed)
    out = {}
    for ci, (sym, d4) in enumerate([(True, 1), (False, 1), (True, 0)]):
        R1 = rng.standard_normal(n)
        Y1 = rng.standard_normal((n, n))
        if sym:
            Y1 = Y1 + Y1.T
        f, dv = LO.perturb_average_sym(d["X"], d["Y"], d["w"], d["rho"], R1, Y1, d["T"], d4, d["syms"],
                                       [len(b) for b in d["blocks"]], d["blocks"], d["blocks_ids"], backend="reference")
        out.update({f"case{ci}_R1": R1, f"case{ci}_Y1": Y1, f"case{ci}_d4": d4, f"case{ci}_f": f, f"case{ci}_d2v": dv})
    return out


def pack(d):
    out = dict(X=d["X"], Y=d["Y"], w=d["w"], rho=d["rho"], blocks_ids=d["blocks_ids"], T=d["T"],
               n_blocks=len(d["syms"]))
    for i, (s, b) in enumerate(zip(d["syms"], d["blocks"])):
        out[f"sym{i}"] = s
        out[f"block{i}"] = b
    return out


def main():
    m10 = load_mode10()
    npz = np.load(os.path.join(REF, "normal", "LANCZOS_STEP10.npz"))
    assert np.array_equal(npz["X"], m10["X"]) and np.array_equal(npz["w"], m10["w"])
    out = pack(m10)
    out.update(a_coeffs=npz["a_coeffs"], b_coeffs=npz["b_coeffs"], c_coeffs=npz["c_coeffs"], s_norm=npz["s_norm"],
               q0=npz["basis_Q"][0], c4_test_constant=6.59744344e-07)
    out.update(averages_cases(m10, seed=10))
    np.savez_compressed(os.path.join(HERE, "mode10.npz"), **out)

    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(2, T=300.0)
    X, Y, rho = RS.sample_ensemble(s, 6, seed=2)
    rs = dict(X=X, Y=Y, w=s.w, rho=rho, blocks_ids=s.blocks_ids, syms=s.symmetries, blocks=s.deg_space, T=s.T)
    out = pack(rs)
    out.update(averages_cases(rs, seed=20))
    np.savez_compressed(os.path.join(HERE, "rocksalt_L2.npz"), **out)
    for f in ("mode10.npz", "rocksalt_L2.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
