"""The CPU oracle, pinned against the reference's own golden data (no GPU)."""
import glob
import os

import numpy as np
import pytest

from conftest import REPO
from oracle import lanczos_oracle as LO


def _avg(d, case, backend="port"):
    return LO.perturb_average_sym(d["X"], d["Y"], d["w"], d["rho"], d[f"{case}_R1"], d[f"{case}_Y1"], d["T"],
                                  int(d[f"{case}_d4"]), d["syms"], d["n_deg"], d["blocks"], d["blocks_ids"],
                                  backend=backend)


@pytest.mark.parametrize("fixture", ["mode10", "rocksalt_l2"])
@pytest.mark.parametrize("case", ["case0", "case1", "case2"])
def test_port_matches_reference_kernel_outputs(request, fixture, case):
    """oracle/tdscha_oracle.c reproduces the reference GetPerturbAverageSym outputs stored in the
    golden files (symmetric / non-symmetric Y1, apply_d4 = 1 / 0)."""
    d = request.getfixturevalue(fixture)
    f, dv = _avg(d, case)
    gf, gd = d[f"{case}_f"], d[f"{case}_d2v"]
    assert np.abs(f - gf).max() <= 1e-13 * np.abs(gf).max()
    assert np.abs(dv - gd).max() <= 1e-13 * np.abs(gd).max()


def test_port_thread_count_and_slices_are_consistent(mode10):
    """Config-sliced partial sums (the reference's MPI partition, LanczosFunctions.c:2123-2136)
    add up to the full average."""
    d = mode10
    f_full, d_full = _avg(d, "case0")
    parts = [LO.perturb_average_sym(d["X"], d["Y"], d["w"], d["rho"], d["case0_R1"], d["case0_Y1"], d["T"], 1,
                                    d["syms"], d["n_deg"], d["blocks"], d["blocks_ids"], i_range=r, n_threads=1)
             for r in [(0, 4), (4, 7), (7, 10)]]
    f_sum = sum(p[0] for p in parts)
    d_sum = sum(p[1] for p in parts)
    assert np.allclose(f_sum, f_full, rtol=1e-12, atol=1e-14 * np.abs(f_full).max())
    assert np.allclose(d_sum, d_full, rtol=1e-12, atol=1e-14 * np.abs(d_full).max())


def test_oracle_chain_replays_reference_coefficients(mode10):
    """Bi-conjugate Lanczos replay of the reference run (tests/test_lanczos_fast/normal/LANCZOS_STEP10.npz):
    steps 0-6 agree to 1e-12 relative; c_4 equals the reference test constant 6.59744344e-07 (rel 1e-6)."""
    d = mode10
    L = LO.OracleLanczos(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    L.psi = d["q0"].copy()
    L.run_FT(10)
    a, b, c = (np.array(x) for x in (L.a_coeffs, L.b_coeffs, L.c_coeffs))
    for got, ref in ((a, d["a_coeffs"]), (b, d["b_coeffs"]), (c, d["c_coeffs"])):
        rel = np.abs(got[:7] - ref[:7]) / np.abs(ref[:7])
        assert rel.max() < 1e-12, rel
    assert abs(c[4] - d["c4_test_constant"]) / d["c4_test_constant"] < 1e-6


def test_reference_kernel_agrees_with_port_when_built(mode10):
    """When oracle/_ref holds the reference kernel compiled from its sources, it agrees with the port."""
    if not glob.glob(os.path.join(REPO, "oracle", "_ref", "sscha_HP_odd*.so")):
        pytest.skip("reference kernel not built (make -C oracle ref)")
    d = mode10
    f1, d1 = _avg(d, "case1", backend="reference")
    f2, d2 = _avg(d, "case1", backend="port")
    assert np.abs(f1 - f2).max() <= 1e-13 * np.abs(f1).max()
    assert np.abs(d1 - d2).max() <= 1e-13 * np.abs(d1).max()


def test_transpose_identity_on_dense_operator(rocksalt_l2):
    """apply_full_L(transpose=True) is the transpose of apply_full_L (the reference's heavy
    test_1D_model.py:181-225 check), on a reduced rock-salt problem."""
    d = rocksalt_l2
    L = LO.OracleLanczos(d["X"][:2], d["Y"][:2], d["w"], d["rho"][:2], d["T"])  # no symmetries, 2 configs
    n = L.n_modes
    ln = n + n * (n + 1)
    rng = np.random.default_rng(0)
    cols = rng.choice(ln, 12, replace=False)
    rows = rng.choice(ln, 12, replace=False)
    Lmat = np.zeros((len(rows), len(cols)))
    LTmat = np.zeros((len(cols), len(rows)))
    for ci, c in enumerate(cols):
        e = np.zeros(ln); e[c] = 1
        Lmat[:, ci] = L.apply_full_L(e, transpose=False)[rows]
    for ri, r in enumerate(rows):
        e = np.zeros(ln); e[r] = 1
        LTmat[:, ri] = L.apply_full_L(e, transpose=True)[cols]
    assert np.allclose(Lmat, LTmat.T, rtol=1e-8, atol=1e-10 * np.abs(Lmat).max())


@pytest.mark.parametrize("use_wigner", [False, True])
def test_explicit_operator_equals_applied_operator_on_the_oracle(rocksalt_l2, use_wigner):
    """For the trivial symmetry group, the reference's analytic operator from explicit d3 / d4
    tensors (einsum restatement) equals the operator its apply_full_L applies (C averages), column
    by column: the two routes of the reference agree, which pins the explicit restatement."""
    import types
    d = rocksalt_l2
    O = LO.OracleLanczos(d["X"], d["Y"], d["w"], d["rho"], d["T"])          # no symmetries
    O.use_wigner = use_wigner
    n = O.n_modes
    ln = n + n * (n + 1)
    La = np.zeros((ln, ln))
    for i in range(ln):
        e = np.zeros(ln)
        e[i] = 1.0
        La[:, i] = O.apply_full_L(e)
    o = types.SimpleNamespace(X=O.X, Y=O.Y, rho=O.rho, w=O.w, T=O.T, n_modes=n, use_wigner=use_wigner,
                              ignore_harmonic=False, ignore_v3=False, ignore_v4=False)
    Lx = LO.explicit_L_operator_FT(o)
    assert np.abs(Lx - La).max() <= 1e-10 * np.abs(La).max()


def test_static_limit_on_the_oracle(rocksalt_l2):
    """The oracle's static operator (apply_L1_static + apply_anharmonic_static) and its dynamical
    operator (apply_full_L) are restated from different reference functions; the R-R block of
    their inverses must agree (the static limit of the dynamical response)."""
    d = rocksalt_l2
    # with the symmetry group: without it, 6 configurations leave the dynamical operator singular
    O = LO.OracleLanczos(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    n = O.n_modes
    ln, ls = n + n * (n + 1), n + n * (n + 1) // 2
    Ld = np.zeros((ln, ln))
    for i in range(ln):
        e = np.zeros(ln)
        e[i] = 1.0
        Ld[:, i] = O.apply_full_L(e)
    Ls = np.zeros((ls, ls))
    for i in range(ls):
        e = np.zeros(ls)
        e[i] = 1.0
        Ls[:, i] = O.apply_static_L(e)
    Gd = np.linalg.inv(Ld)[:n, :n]
    Gs = np.linalg.inv(Ls)[:n, :n]
    assert np.abs(Gd - Gs).max() <= 1e-8 * np.abs(Gs).max()
