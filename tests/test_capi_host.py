"""No-GPU checks: the C ABI library loads and exports every symbol include/*.h declares; the
synthetic generator's invariants; host-side API logic (perturbation set-up, checkpoint schema)."""
import glob
import os
import re
import types

import numpy as np
import pytest

from conftest import REPO


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(?:int|const char \*)\s*(tdscha_\w+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from tdscha_b200 import _native
    lib = _native.load()
    names = declared_symbols()
    assert len(names) >= 15
    for nm in sorted(names):
        assert hasattr(lib, nm), f"{nm} declared in include/ but not exported"
    assert lib.tdscha_version().startswith(b"tdscha_b200")


def test_errors_are_returned_not_exit():
    """Without a usable device the C ABI returns an error code and a message (the reference's
    binding calls exit(); this one never does)."""
    from tdscha_b200 import _native
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(_native.TdschaError):
        _native.DeviceEnsemble(np.ones((2, 3)), np.ones((2, 3)), np.ones(3), np.ones(2), 300.0,
                               [np.ones((1, 1, 1))] * 3, [np.array([i]) for i in range(3)], np.arange(3))


@pytest.mark.parametrize("L,n_expected", [(2, 45)])
def test_generator_invariants(L, n_expected):
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(L, T=300.0)
    assert s.n_modes == n_expected == 3 * s.nat - 3
    assert s.n_syms == 48 * L ** 3
    # frequencies equal inside each block; blocks contiguous and ordered
    start = 0
    for b, blk in enumerate(s.deg_space):
        assert blk[0] == start and np.all(np.diff(blk) == 1)
        assert np.ptp(s.w[blk]) == 0.0
        assert np.all(s.blocks_ids[blk] == b)
        start += len(blk)
    # every symmetry block is orthogonal
    for S in s.symmetries:
        I = np.einsum("jab,jcb->jac", S, S)
        assert np.abs(I - np.eye(S.shape[1])).max() < 1e-12
    # harmonic frequencies commute with the symmetries: the eigenvectors span invariant subspaces
    X, Y, rho = RS.sample_ensemble(s, 4, seed=0)
    assert X.shape == (4, n_expected) and np.all(np.isfinite(Y))


def test_unwrapped_ensemble_equals_symmetrised_blocks():
    """The reference's heavy snse test (tests/_heavy_tests/test_fast_lanczos_snse): averages over an
    ensemble unwrapped by every symmetry (N * N_sym configurations, no symmetries) equal the
    on-the-fly symmetrised averages."""
    from oracle import lanczos_oracle as LO
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(2, T=300.0)
    X, Y, rho = RS.sample_ensemble(s, 2, seed=1)
    n = s.n_modes
    rng = np.random.default_rng(3)
    R1 = rng.standard_normal(n)
    Y1 = rng.standard_normal((n, n))
    f1, d1 = LO.perturb_average_sym(X, Y, s.w, rho, R1, Y1, s.T, 1, s.symmetries, [len(b) for b in s.deg_space],
                                    s.deg_space, s.blocks_ids)
    E = s.pols
    Xu, Yu = [], []
    for i in range(len(X)):
        ut = (E @ X[i]).reshape(s.nat, 3)
        ft = (E @ Y[i]).reshape(s.nat, 3)
        for j in range(s.n_syms):
            u2 = np.zeros_like(ut)
            f2 = np.zeros_like(ft)
            u2[s.perm[j]] = ut @ s.rot[j].T
            f2[s.perm[j]] = ft @ s.rot[j].T
            Xu.append(E.T @ u2.ravel())
            Yu.append(E.T @ f2.ravel())
    Xu, Yu = np.array(Xu), np.array(Yu)
    f2_, d2_ = LO.perturb_average_sym(Xu, Yu, s.w, np.ones(len(Xu)), R1, Y1, s.T, 1, [np.ones((1, 1, 1))] * n,
                                      np.ones(n, dtype=np.intc), [np.array([k]) for k in range(n)], np.arange(n))
    assert np.abs(f1 - f2_).max() <= 1e-12 * np.abs(f1).max()
    assert np.abs(d1 - d2_).max() <= 1e-12 * np.abs(d1).max()


def _lanczos():
    from tdscha_b200 import DynamicalLanczos as DL, rocksalt as RS
    ens = RS.make_ensemble(2, 4, seed=0)
    return DL.Lanczos(ens), ens


def test_attribute_whitelist():
    L, _ = _lanczos()
    L.shift_value = 1e-3
    with pytest.raises(AttributeError, match="similar"):
        L.shift_valeu = 1.0


def test_prepare_perturbations_follow_reference_formulas():
    """prepare_perturbation (DynamicalLanczos.py:1963-2013), prepare_ir (:1647-1689) and
    prepare_raman (:1003-1124) on the host."""
    L, ens = _lanczos()
    n = L.n_modes
    v = np.random.default_rng(0).standard_normal(3 * ens.nat)
    L.prepare_perturbation(v, masses_exp=-1)
    ref = np.einsum("a,a,ab->b", np.sqrt(ens.m) ** -1, v, ens.pols)
    assert np.allclose(L.psi[:n], ref) and np.all(L.psi[n:] == 0)
    assert np.isclose(L.perturbation_modulus, ref @ ref)
    L.prepare_ir(pol_vec=np.array([0, 1.0, 0]))
    z = np.einsum("abc,b", ens.effective_charges, np.array([0, 1.0, 0]))
    ref = np.einsum("a,a,ab->b", np.sqrt(ens.m) ** -1, np.tile(z.ravel(), 8), ens.pols)
    assert np.allclose(L.psi[:n], ref)
    L.prepare_raman(pol_vec_in=np.array([1.0, 0, 0]), pol_vec_out=np.array([0, 0, 1.0]))
    from tdscha_b200.rocksalt import raman_vector
    rv = np.tile(raman_vector(ens.raman_tensor, np.array([1.0, 0, 0]), np.array([0, 0, 1.0])), 8)
    ref = np.einsum("a,a,ab->b", np.sqrt(ens.m) ** -1, rv, ens.pols)
    assert np.allclose(L.psi[:n], ref)
    L.prepare_mode(5)
    assert L.psi[5] == 1 and L.psi.sum() == 1 and L.perturbation_modulus == 1


REFERENCE_NPZ_KEYS = {"T", "nat", "m", "w", "pols", "n_modes", "ignore_v3", "ignore_v4", "N", "rho", "X", "Y", "psi",
                      "a_coeffs", "b_coeffs", "c_coeffs", "basis_Q", "basis_P", "s_norm", "krilov_basis",
                      "arnoldi_matrix", "reverse", "shift", "perturbation_modulus", "use_wigner", "ignore_small_w",
                      "sym_julia", "deg_julia", "n_syms"}   # DynamicalLanczos.py:3617-3646


def test_checkpoint_schema_round_trip(tmp_path):
    L, _ = _lanczos()
    L.a_coeffs, L.b_coeffs, L.c_coeffs = [1.0, 2.0], [0.5], [0.25]
    L.basis_Q = [np.ones(len(L.psi)), np.zeros(len(L.psi))]
    L.basis_P = list(L.basis_Q)
    L.s_norm = [1, 0.3]
    L.reverse_L, L.shift_value, L.perturbation_modulus = True, 2e-4, 3.5
    f = str(tmp_path / "STEP2")
    L.save_status(f)
    keys = set(np.load(f + ".npz", allow_pickle=True).files)
    assert keys == REFERENCE_NPZ_KEYS
    L2, _ = _lanczos()
    L2.load_status(f)
    assert L2.a_coeffs == [1.0, 2.0] and L2.c_coeffs == [0.25] and L2.reverse_L and L2.shift_value == 2e-4
    assert L2.perturbation_modulus == 3.5 and np.array_equal(np.asarray(L2.basis_Q), np.asarray(L.basis_Q))


def test_argument_errors_of_run_and_static_entry_points():
    """Argument checks of the multi-system run and the static operator come back as error codes
    with a message before any device call (no GPU needed)."""
    import ctypes
    from tdscha_b200 import _native
    lib = _native.load()
    EINVAL = [k for k, v in _native.ERRORS.items() if v == "EINVAL"][0]
    rc = lib.tdscha_lanczos_run_device(0, None, 5, 1, None)
    assert rc != 0 and b"systems per run" in lib.tdscha_last_error()
    rc = lib.tdscha_lanczos_run_device(1, None, 5, 1, None)
    assert rc != 0 and b"bad run arguments" in lib.tdscha_last_error()
    sysarr = (_native.RunSystem * 1)()           # NULL ensemble and buffers
    rc = lib.tdscha_lanczos_run_device(1, sysarr, 5, 1, None)
    assert rc != 0 and b"NULL argument" in lib.tdscha_last_error()
    rc = lib.tdscha_apply_static_L_device(None, 1, None, 0, 1, 0, None, None)
    assert rc != 0 and b"NULL ensemble" in lib.tdscha_last_error()
    rc = lib.tdscha_apply_L1_static_device(None, 1, None, ctypes.c_double(1.0), None, None)
    assert rc == EINVAL and b"NULL ensemble" in lib.tdscha_last_error()
