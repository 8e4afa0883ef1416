"""Host-side logic of the static Hessian: the packed state <-> row-vector maps of StaticHessian
and the oracle's minimum-residual restatement (no GPU)."""
import numpy as np

from oracle import lanczos_oracle as LO


def test_state_layout_matches_reference_loops():
    from tdscha_b200 import StaticHessian as SH
    n = 6
    rng = np.random.default_rng(0)
    n_g, n_w = n * (n + 1) // 2, n * (n + 1) * (n + 2) // 6
    vec = rng.standard_normal(n_g + n_w)
    h = SH.StaticHessian()
    h.lanczos.n_modes = n
    G, W = h.get_G_W(vec)
    Go, Wo = LO.static_hessian_get_G_W(vec, n)
    assert np.array_equal(G, Go) and np.array_equal(W, Wo)
    assert np.array_equal(h.get_vector(G, W), LO.static_hessian_get_vector(Go, Wo))
    # the row maps reproduce apply_L's row vectors and get_vector's extraction
    gather, srow, selem = SH.row_maps(n)
    rows = vec[gather]
    for i in range(n):
        assert np.array_equal(rows[i, :n], Go[i])
        assert np.array_equal(rows[i, n:], LO.pack_upper(Wo[i]))
    out_rows = rng.standard_normal(rows.shape)
    Gr = np.array([r[:n] for r in out_rows])
    Wr = np.array([LO.unpack_sym(r[n:], n) for r in out_rows])
    assert np.array_equal(out_rows[srow, selem], LO.static_hessian_get_vector(Gr, Wr))


def test_minimum_residual_restatement_solves_spd_system():
    rng = np.random.default_rng(1)
    Q = rng.standard_normal((30, 30))
    A = Q @ Q.T + 30 * np.eye(30)
    b = rng.standard_normal(30)
    x = LO.minimum_residual_algorithm(lambda v: A @ v, b, b.copy(), max_iters=200, conv_thr=1e-12)
    assert np.abs(A @ x - b).max() < 1e-9 * np.abs(b).max()
    d = np.sqrt(np.diag(A))
    x2 = LO.minimum_residual_algorithm_precond(lambda v: A @ v, b, lambda v: v / d, max_iters=200, conv_thr=1e-12)
    assert np.abs(A @ x2 - b).max() < 1e-9 * np.abs(b).max()
