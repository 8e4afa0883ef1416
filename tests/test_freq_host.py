"""Character classes of the factorised path (tdscha_symmetry_classes), no device needed.

On the factorised path the symmetries are S_p D_t with D_t in an abelian subgroup (the lattice
translations), and the averages of CModules/LanczosFunctions.c:2082-2754 (GetPerturbAverageSym: the
loop over configurations and symmetries) run their two big contractions class by class over the
characters of that subgroup.  This test takes the library's host-built tables and evaluates the
averages with them in numpy, step for step as the device does (left operands from the coset
representatives, per-class contractions, weights in the character basis, reconstruction, fold over
the representatives), and checks the result against the oracle's averages."""
import numpy as np
import pytest

from oracle import lanczos_oracle as LO
from tdscha_b200 import _native, rocksalt as RS


def _emulate(ens, R1, Y1, d4):
    syms, blocks = ens.symmetries, ens.deg_space
    X, Y, w, rho, T = ens.X, ens.Y, ens.w, ens.rho, ens.T
    N, n = X.shape
    N_sym = syms[0].shape[0]
    cos = _native.symmetry_cosets(syms)
    cl = _native.symmetry_classes(syms)
    assert cos is not None and cl is not None
    starts = np.cumsum([0] + [len(b) for b in blocks])
    Rf = np.zeros((n, n))
    for b, Rb in enumerate(cos["R"]):
        Rf[starts[b]:starts[b + 1], starts[b]:starts[b + 1]] = Rb

    def full(j):
        S = np.zeros((n, n))
        for b, t in enumerate(syms):
            S[starts[b]:starts[b + 1], starts[b]:starts[b + 1]] = t[j]
        return S

    nbose = 1.0 / np.expm1(w * 157887.32400374097 / T)
    ups, psi = 2 * w / (1 + 2 * nbose), (1 + 2 * nbose) / (2 * w)
    Xr, Yr = X @ Rf, Y @ Rf
    Gr, Xtr = Yr * psi, Xr * ups
    Ysr = Rf.T @ (0.5 * (Y1 + Y1.T)) @ Rf
    R1r = R1 @ Rf
    sub, ncos, order = cos["coset_size"], cos["n_cosets"], cos["order"]
    Srep = [Rf.T @ full(order[p * sub]) @ Rf for p in range(ncos)]
    mu, nu = np.triu_indices(n)
    pi, pd = cl["pcol_i"], cl["pcol_d"]
    mi, md = cl["mcol_i"], cl["mcol_d"]

    def own_pairs(Ms):          # Ms: (k, n, n) symmetric -> (k, Kq) own values
        return pd[:, 0] * Ms[:, pi[:, 0], pi[:, 1]] + pd[:, 1] * Ms[:, pi[:, 2], pi[:, 3]]

    def partner_of(v, partner):  # v: (k, cols) -> values at the partner column (0 without one)
        out = np.zeros_like(v)
        has = partner >= 0
        out[:, has] = v[:, partner[has]]
        return out

    # left operands (rows: real parts, then imaginary parts)
    U = np.stack([S.T @ Ysr @ S for S in Srep])
    own_u = own_pairs(U)
    Lab = np.vstack([pd[:, 2] * own_u, pd[:, 3] * partner_of(own_u, pi[:, 4])])
    r1p = np.stack([ups * (S.T @ R1r) for S in Srep])
    own_r = md[:, 0] * r1p[:, mi[:, 0]]
    Lcd = np.vstack([md[:, 1] * own_r, md[:, 2] * partner_of(own_r, mi[:, 1])])
    # ensemble operands in the character basis
    MA = np.einsum("ia,ib->iab", Xr, Xr)
    MB = 0.5 * (np.einsum("ia,ib->iab", Xr, Gr) + np.einsum("ia,ib->iab", Gr, Xr))
    Vq = np.vstack([own_pairs(MA), own_pairs(MB)])                     # (2N, Kq)
    XGq = md[:, 0] * np.vstack([Xr[:, mi[:, 0]], Gr[:, mi[:, 0]]])      # (2N, Kmq)
    YXq = md[:, 0] * np.vstack([Yr[:, mi[:, 0]], Xtr[:, mi[:, 0]]])     # (2N, Kmq)
    O = np.zeros((2 * ncos, cl["Kq"]))
    OF = np.zeros((2 * ncos, cl["Kmq"]))
    for real, po, pc, mo, mc in cl["cls"]:
        P_ = slice(po, po + pc)
        M_ = slice(mo, mo + mc)
        H = Lab[:, P_] @ Vq[:, P_].T
        C = Lcd[:, M_] @ XGq[:, M_].T if mc else np.zeros_like(H)
        a, b, c, d = H[:, :N], H[:, N:], C[:, :N], C[:, N:]
        gam = rho * (-c / 3 + d4 * a / 8)
        dlt = rho * (-d / 3 + d4 * b / 4)
        Cw = np.hstack([0.5 * dlt, gam])
        AB = np.hstack([-rho * a / 6, -rho * b / 3])
        if real:
            Cw[ncos:] = 0
            AB[ncos:] = 0
        O[:, P_] = Cw @ Vq[:, P_]
        if mc:
            OF[:, M_] = AB @ YXq[:, M_]
    own_o = O[:ncos] + pd[:, 4] * partner_of(O[ncos:], pi[:, 4])
    Nt = cl["pp_d"][:, 0] * own_o[:, cl["pp_i"][:, 0]] + cl["pp_d"][:, 1] * own_o[:, cl["pp_i"][:, 1]]
    own_f = OF[:ncos] + md[:, 3] * partner_of(OF[ncos:], mi[:, 1])
    mc_ = cl["mode_col"]
    Fs = np.where(mc_ >= 0, md[np.maximum(mc_, 0), 0] * own_f[:, np.maximum(mc_, 0)], 0.0)
    Dr, fr = np.zeros((n, n)), np.zeros(n)
    for p, S in enumerate(Srep):
        Nm = np.zeros((n, n))
        Nm[mu, nu] = Nt[p]
        Nm[nu, mu] = Nt[p]
        Dr += S @ (2 * np.outer(ups, ups) * Nm) @ S.T
        fr += S @ Fs[p]
    norm = 1.0 / (rho.sum() * N_sym)
    return Rf @ (fr * norm), Rf @ (Dr * norm) @ Rf.T, cl


@pytest.mark.parametrize("L,N,n_class", [(2, 6, 8), (3, 3, 14), (4, 2, 36)])   # 4x4x4: the benchmark's group
def test_class_tables_reproduce_the_averages(L, N, n_class):
    ens = RS.make_ensemble(L, N, seed=5)
    n = ens.X.shape[1]
    rng = np.random.default_rng(L)
    R1, Y1 = rng.standard_normal(n), rng.standard_normal((n, n))
    n_deg = np.array([len(b) for b in ens.deg_space], dtype=np.intc)
    for d4 in (0, 1):
        f_ref, d_ref = LO.perturb_average_sym(ens.X, ens.Y, ens.w, ens.rho, R1, Y1, ens.T, d4, ens.symmetries, n_deg,
                                              ens.deg_space, ens.blocks_ids)
        f, d, cl = _emulate(ens, R1, Y1, d4)
        assert np.abs(f - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
        assert np.abs(d - d_ref).max() <= 1e-12 * np.abs(d_ref).max()
    assert cl["n_class"] == n_class
    sub = len(ens.symmetries[0]) // 48
    # the class contractions do about 2 / |K| of the work over every symmetry (plus class padding)
    assert cl["flops_ratio"] < 2.0 / sub * 1.3


def test_class_tables_reproduce_the_averages_at_5x5x5():
    """The largest group of the benchmark configurations: O_h x 125 = 6000 operations, 63 classes."""
    ens = RS.make_ensemble(5, 2, seed=5)
    n = ens.X.shape[1]
    rng = np.random.default_rng(5)
    R1, Y1 = rng.standard_normal(n), rng.standard_normal((n, n))
    n_deg = np.array([len(b) for b in ens.deg_space], dtype=np.intc)
    f_ref, d_ref = LO.perturb_average_sym(ens.X, ens.Y, ens.w, ens.rho, R1, Y1, ens.T, 1, ens.symmetries, n_deg,
                                          ens.deg_space, ens.blocks_ids)
    f, d, cl = _emulate(ens, R1, Y1, 1)
    assert np.abs(f - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
    assert np.abs(d - d_ref).max() <= 1e-12 * np.abs(d_ref).max()
    assert cl["n_class"] == 63
    assert cl["flops_ratio"] < 2.0 / 125 * 1.3


def test_classes_of_the_benchmark_system():
    system = RS.build_system(4)
    cl = _native.symmetry_classes(system.symmetries)
    n = sum(t.shape[1] for t in system.symmetries)
    assert cl is not None and cl["n_class"] == 36                  # 8 real + 28 complex characters of Z4^3
    assert int(cl["cls"][:, 0].sum()) == 8
    assert cl["Kq"] % 64 == 0 and cl["Kq"] >= n * (n + 1) // 2
    assert cl["flops_ratio"] < 0.035                               # vs 1 over all 3072 symmetry rows


def test_no_classes_without_the_structure():
    tables = [np.stack([np.eye(3), -np.eye(3)]), np.stack([np.eye(2), -np.eye(2)])]
    assert _native.symmetry_classes(tables) is None
