"""Host-side pieces of the apply_full_L consumers: the harmonic-inverse preconditioner
(DynamicalLanczos.py:2391-2502) against the oracle's harmonic operator, and the Lanczos matrix
built from the coefficients (:4571-4613).  No GPU needed."""
import types

import numpy as np

from oracle import lanczos_oracle as LO


def _lanczos(d):
    from tdscha_b200 import DynamicalLanczos as DL
    n = d["X"].shape[1]
    ens = types.SimpleNamespace(T=d["T"], nat=16, m=np.ones(48), w=d["w"], pols=np.eye(48, n), N=len(d["rho"]),
                                rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"], deg_space=d["blocks"],
                                blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)
    return DL.Lanczos(ens)


def _oracle(d):
    return LO.OracleLanczos(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])


def test_l1_inverse_inverts_the_harmonic_operator(rocksalt_l2):
    """M (L1 x) = x on R and on every pair whose 2 x 2 free propagator the reference inverts exactly
    (den above its epsilon; the regularised pairs get the reference's diagonal substitutes)."""
    d = rocksalt_l2
    L, O = _lanczos(d), _oracle(d)
    n = L.n_modes
    m = n * (n + 1) // 2
    r, c = np.triu_indices(n)
    w_a, w_b = L.w[c], L.w[r]
    na, nb = LO.bose(w_a, L.T), LO.bose(w_b, L.T)
    Xab = -w_a ** 2 - w_b ** 2 - (2 * w_a * w_b) / ((2 * na + 1) * (2 * nb + 1))
    Yab = -(8 * w_a * w_b) / ((2 * na + 1) * (2 * nb + 1))
    X1 = -(2 * na * nb + na + nb) * (2 * na * nb + na + nb + 1) * (2 * w_a * w_b) / ((2 * na + 1) * (2 * nb + 1))
    Y1 = -w_a ** 2 - w_b ** 2 + (2 * w_a * w_b) / ((2 * na + 1) * (2 * nb + 1))
    regular = (Xab * Y1 - X1 * Yab >= 1e-12) & ~((w_a == w_b) & (na > 1e-12))
    assert regular.sum() > 0.5 * m
    x = np.random.default_rng(3).standard_normal(n + 2 * m)
    for transpose in (False, True):
        O.psi = x.copy()
        got = L.apply_L1_inverse_FT(O.apply_L1_FT(transpose=transpose), transpose=transpose)
        keep = np.concatenate([np.ones(n, bool), regular, regular])
        assert np.abs(got - x)[keep].max() < 1e-10 * np.abs(x).max()


def test_l1_inverse_transpose_identity(rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal((2, len(L.psi)))
    lhs = y @ L.apply_L1_inverse_FT(x)
    rhs = L.apply_L1_inverse_FT(y, transpose=True) @ x
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_l1_inverse_ignore_harmonic_is_zero(rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    L.ignore_harmonic = True
    assert not np.any(L.apply_L1_inverse_FT(np.ones(len(L.psi))))


def test_lanczos_matrix_from_coeffs(rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    L.a_coeffs, L.b_coeffs, L.c_coeffs = [1.0, 2.0, 3.0], [0.5, 0.25], [0.7, 0.9]
    M = L.build_lanczos_matrix_from_coeffs()
    ref = np.array([[1.0, 0.7, 0.0], [0.5, 2.0, 0.9], [0.0, 0.25, 3.0]])
    assert np.array_equal(M, ref)
    L.reverse_L, L.shift_value = True, 0.1
    assert np.allclose(L.build_lanczos_matrix_from_coeffs(), -ref + 0.1 * np.eye(3))
    L.reverse_L, L.shift_value, L.c_coeffs = False, 0, []
    M = L.build_lanczos_matrix_from_coeffs()          # symmetric Lanczos: b on both sides
    assert M[0, 1] == M[1, 0] == 0.5
