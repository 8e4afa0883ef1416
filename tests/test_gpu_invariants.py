"""Invariants of the operator (the reference's heavy tests, restated on the synthetic systems):
  * on-the-fly symmetrisation equals the explicitly unwrapped ensemble (N N_sym configurations
    S_j x_i, S_j y_i and no symmetry), for the device averages in every precision;
  * the static limit: the R-R block of the inverse dynamical operator at w = 0 equals the R-R block
    of the inverse static operator (both dense, built from device applies)."""
import types

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _full_S(d, n):
    N_sym = d["syms"][0].shape[0]
    S = np.zeros((N_sym, n, n))
    for tab, blk in zip(d["syms"], d["blocks"]):
        blk = np.asarray(blk)
        S[:, blk[:, None], blk[None, :]] = tab
    return S


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("bf16x3", 2e-4), ("tf32x3", 2e-5)])
def test_symmetrised_equals_unwrapped_ensemble(cuda, rocksalt_l2, precision, tol):
    from tdscha_b200 import _native
    d = rocksalt_l2
    X, Y, rho = d["X"], d["Y"], d["rho"]
    N, n = X.shape
    S = _full_S(d, n)
    Xu = np.einsum("jab,ib->jia", S, X).reshape(-1, n)      # configuration (j, i): S_j x_i
    Yu = np.einsum("jab,ib->jia", S, Y).reshape(-1, n)
    rho_u = np.tile(rho, S.shape[0])
    one = [np.ones((1, 1, 1))] * n
    blocks1 = [np.array([m], dtype=np.intc) for m in range(n)]
    ids1 = np.arange(n, dtype=np.intc)
    sym = _native.DeviceEnsemble(X, Y, d["w"], rho, d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    unw = _native.DeviceEnsemble(Xu, Yu, d["w"], rho_u, d["T"], one, blocks1, ids1)
    for case in ("case0", "case1", "case2"):
        f1, D1 = sym.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), precision)
        f2, D2 = unw.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), precision)
        assert np.abs(f1 - f2).max() <= tol * np.abs(f2).max(), case
        assert np.abs(D1 - D2).max() <= tol * np.abs(D2).max(), case
    sym.close()
    unw.close()


def test_static_limit_of_the_dynamical_operator(cuda, rocksalt_l2):
    from tdscha_b200 import DynamicalLanczos as DL
    torch = cuda
    d = rocksalt_l2
    n = d["X"].shape[1]
    ens = types.SimpleNamespace(T=d["T"], nat=16, m=np.ones(48), w=d["w"], pols=np.eye(48, n), N=len(d["rho"]),
                                rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"], deg_space=d["blocks"],
                                blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)
    L = DL.Lanczos(ens)
    L.init()
    Ldyn = L.get_full_L_operator_FT(overwrite_L_operator=False)
    ls = n + n * (n + 1) // 2
    E = torch.eye(ls, dtype=torch.float64, device="cuda")
    Lst = torch.empty_like(E)
    L_rows = []
    for c0 in range(0, ls, 64):
        out = L._static_apply_batched(E[c0:c0 + 64].contiguous())
        L_rows.append(out.cpu().numpy())
    Lstat = np.concatenate(L_rows).T                     # columns = static L applied to unit vectors
    del Lst
    Gdyn = np.linalg.inv(Ldyn)[:n, :n]
    Gst = np.linalg.inv(Lstat)[:n, :n]
    err = np.abs(Gdyn - Gst).max() / np.abs(Gst).max()
    print("static-limit relative difference:", err)
    assert err < 1e-8
