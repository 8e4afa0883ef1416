"""The reference's analytic L operator from explicit d3 / d4 tensors (get_full_L_operator_FT with
symmetrize=False or debug_d3) against the oracle's einsum restatement, and against the operator
that apply_full_L applies when the symmetry group is trivial."""
import types

import numpy as np
import pytest

from oracle import lanczos_oracle as LO

pytestmark = pytest.mark.gpu


def _ens(d, nat=16):
    n = d["X"].shape[1]
    return types.SimpleNamespace(T=d["T"], nat=nat, m=np.ones(3 * nat), w=d["w"], pols=np.eye(3 * nat, n),
                                 N=len(d["rho"]), rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"],
                                 deg_space=d["blocks"], blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)


def _lanczos(d, use_symmetries=True, **kw):
    from tdscha_b200 import DynamicalLanczos as DL
    L = DL.Lanczos(_ens(d), **kw)
    L.init(use_symmetries=use_symmetries)
    return L


def _oracle_obj(L):
    return types.SimpleNamespace(X=np.asarray(L.X), Y=np.asarray(L.Y), rho=np.asarray(L.rho), w=np.asarray(L.w),
                                 T=float(L.T), n_modes=L.n_modes, use_wigner=L.use_wigner,
                                 ignore_harmonic=L.ignore_harmonic, ignore_v3=L.ignore_v3, ignore_v4=L.ignore_v4)


FLAGS = [dict(), dict(use_wigner=True), dict(ignore_v4=True), dict(ignore_v3=True), dict(ignore_harmonic=True),
         dict(use_wigner=True, ignore_v4=True)]


@pytest.mark.parametrize("flags", FLAGS, ids=lambda f: "-".join(f) or "default")
def test_explicit_operator_matches_oracle(cuda, rocksalt_l2, flags):
    flags = dict(flags)
    L = _lanczos(rocksalt_l2, use_wigner=flags.pop("use_wigner", False))
    for k, v in flags.items():
        setattr(L, k, v)
    got = L.get_full_L_operator_FT(symmetrize=False, overwrite_L_operator=False)
    ref = LO.explicit_L_operator_FT(_oracle_obj(L))
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


def test_debug_d3_and_symmetrize_semantics(cuda, rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    n = L.n_modes
    rng = np.random.default_rng(8)
    A = rng.standard_normal((n, n, n))
    d3 = sum(np.transpose(A, p) for p in [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]) / 6
    L.ignore_v4 = True
    got = L.get_full_L_operator_FT(debug_d3=d3, overwrite_L_operator=False)
    ref = LO.explicit_L_operator_FT(_oracle_obj(L), debug_d3=d3)
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
    # the reference cannot symmetrise d4: symmetrize=True with v4 on and a debug d3 raises
    L.ignore_v4 = False
    with pytest.raises(NotImplementedError):
        L.explicit_L_operator_FT(debug_d3=d3, symmetrize=True)


@pytest.mark.parametrize("use_wigner", [False, True])
def test_explicit_operator_equals_applied_operator_without_symmetries(cuda, rocksalt_l2, use_wigner):
    """With the trivial symmetry group the averages of apply_full_L and the explicit tensors
    describe the same operator (the two routes of the reference agree)."""
    L = _lanczos(rocksalt_l2, use_symmetries=False, use_wigner=use_wigner)
    Lx = L.get_full_L_operator_FT(symmetrize=False, overwrite_L_operator=False)
    La = L.get_full_L_operator_FT(symmetrize=True, overwrite_L_operator=False)
    print("max |explicit - applied| / max:", np.abs(Lx - La).max() / np.abs(La).max())
    assert np.abs(Lx - La).max() <= 1e-9 * np.abs(La).max()
