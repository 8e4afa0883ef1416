"""The Lanczos inputs built on the GPU (tdscha_project_ensemble, tdscha_symmetries_on_modes)
against the numpy construction of the rock-salt generator and plain numpy projections."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    from tdscha_b200 import rocksalt as RS
    return RS.build_system(2)


def test_symmetries_on_modes_match_numpy(cuda, system):
    from tdscha_b200 import modes
    s = system
    syms, blocks, bids = modes.symmetries_on_modes(s.pols, s.w, s.perm, s.rot)
    assert [list(b) for b in blocks] == [list(b) for b in s.deg_space] and np.array_equal(bids, s.blocks_ids)
    for got, ref in zip(syms, s.symmetries):
        assert got.shape == ref.shape
        assert np.abs(got - ref).max() <= 1e-12
    # orthogonality of every block of every operation
    for S in syms:
        eye = np.einsum("jab,jcb->jac", S, S)
        assert np.abs(eye - np.eye(S.shape[1])).max() <= 1e-10


def test_generator_gpu_symmetries_match_numpy(cuda):
    """build_system(symmetries_on_gpu=True), the path of the large-supercell benchmark, on 3x3x3."""
    from tdscha_b200 import rocksalt as RS
    ref = RS.build_system(3)
    got = RS.build_system(3, symmetries_on_gpu=True)
    assert np.array_equal(ref.perm, got.perm)
    for a, b in zip(got.symmetries, ref.symmetries):
        assert np.abs(a - b).max() <= 1e-12


def test_ensemble_projection_matches_numpy(cuda, system):
    from tdscha_b200 import modes
    s = system
    rng = np.random.default_rng(2)
    N, nat3 = 300, 3 * s.nat
    u = rng.standard_normal((N, nat3)) * 0.05
    f = rng.standard_normal((N, nat3)) * 1e-3
    fs = rng.standard_normal((N, nat3)) * 1e-4
    fm = rng.standard_normal((2, 3)) * 1e-5
    X, Y = modes.ensemble_to_modes(u, f, fs, s.masses, s.pols, f_mean_uc=fm, n_cell=s.nat // 2)
    ub = u / modes.BOHR_TO_ANG
    fb = (f - fs) * modes.BOHR_TO_ANG - np.tile(fm, (s.nat // 2, 1)).ravel() * modes.BOHR_TO_ANG
    Xr = (ub * np.sqrt(s.masses)) @ s.pols
    Yr = (fb / np.sqrt(s.masses)) @ s.pols
    assert np.abs(X - Xr).max() <= 1e-12 * np.abs(Xr).max()
    assert np.abs(Y - Yr).max() <= 1e-12 * np.abs(Yr).max()
