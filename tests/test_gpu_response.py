"""Consumers of apply_full_L on the GPU (DynamicalLanczos.py:3761-3972, 5273-5307, 5454-5789):
the dense operator built from batched applies, the static response by BiCGSTAB (the batched
device solver and scipy's sequential one) against a dense solve, and the static frequency of a
converged chain against the dense inverse."""
import types

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lanczos(d, **kw):
    from tdscha_b200 import DynamicalLanczos as DL
    n = d["X"].shape[1]
    ens = types.SimpleNamespace(T=d["T"], nat=16, m=np.ones(48), w=d["w"], pols=np.eye(48, n), N=len(d["rho"]),
                                rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"], deg_space=d["blocks"],
                                blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)
    L = DL.Lanczos(ens, **kw)
    L.init()
    return L


@pytest.fixture(scope="module")
def dense(cuda, rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    return L, L.get_full_L_operator_FT(overwrite_L_operator=False)


def test_full_operator_is_apply_full_L(dense):
    L, Lmat = dense
    rng = np.random.default_rng(8)
    for transpose in (False, True):
        v = rng.standard_normal(len(L.psi)) * 1e-2
        got = (Lmat.T if transpose else Lmat) @ v
        ref = L._apply_host(v, transpose, L._opts())
        assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


def test_static_response_batched_bicgstab_matches_dense_solve(dense):
    L, Lmat = dense
    n = L.n_modes
    G_exact = np.linalg.solve(Lmat, np.eye(len(L.psi))[:, :n])[:n, :].T
    H_exact = np.linalg.inv(0.5 * (G_exact + G_exact.T))
    H = L.run_biconjugate_gradient(verbose=False, tol=1e-10, maxiter=2000, batched=True, batch=16)
    assert np.abs(H - H_exact).max() <= 1e-6 * np.abs(H_exact).max()
    assert np.allclose(H, H.T)


def test_static_response_scipy_path_matches_batched(dense):
    L, _ = dense
    Hb = L.run_biconjugate_gradient(verbose=False, tol=1e-10, maxiter=2000, batched=True)
    Hs = L.run_biconjugate_gradient(verbose=False, tol=1e-10, maxiter=2000, batched=False)
    assert np.abs(Hs - Hb).max() <= 1e-6 * np.abs(Hb).max()


def test_static_frequency_of_converged_chain(dense):
    """For a perturbation on mode i, G(0) of the chain is (L^-1)_ii: the static frequency is
    sqrt(1 / (L^-1)_ii)."""
    L, Lmat = dense
    i = 5
    e = np.zeros(len(L.psi))
    e[i] = 1.0
    x = np.linalg.solve(Lmat, e)
    w_ref = np.sqrt(abs(1 / x[i])) * np.sign(1 / x[i])
    L.prepare_mode(i)
    L.run_FT(300, verbose=False)
    assert abs(L.get_static_frequency() - w_ref) <= 1e-6 * abs(w_ref)
