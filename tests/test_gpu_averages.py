"""Symmetrised perturbed averages on the GPU (C ABI) against the reference kernel's golden outputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# max-norm error relative to the max-norm of the golden output, per precision mode
TOL = {"fp64": 1e-12, "tf32x3": 2e-5, "bf16x3": 2e-4, "tf32": 2e-2, "bf16": 1e-1}


def _dev_ens(d):
    from tdscha_b200 import _native
    return _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("fixture", ["mode10", "rocksalt_l2"])
@pytest.mark.parametrize("precision", list(TOL))
def test_averages_match_reference_golden(request, cuda, fixture, precision):
    d = request.getfixturevalue(fixture)
    ens = _dev_ens(d)
    for case in ("case0", "case1", "case2"):
        f, dv = ens.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), precision)
        ef, ed = _rel(f, d[f"{case}_f"]), _rel(dv, d[f"{case}_d2v"])
        print(f"{fixture} {precision} {case}: f {ef:.2e} d2v {ed:.2e}")
        assert ef < TOL[precision] and ed < TOL[precision], (case, ef, ed)
    ens.close()


def test_one_shot_drop_in_matches_golden(cuda, mode10):
    """tdscha_GetPerturbAverageSym: the reference's argument list, outputs written in place."""
    from tdscha_b200 import _native
    d = mode10
    n = d["X"].shape[1]
    f = np.zeros(n)
    dv = np.zeros((n, n))
    _native.get_perturb_average_sym(d["X"], d["Y"], d["w"], d["rho"], d["case1_R1"], d["case1_Y1"], d["T"], 1,
                                    d["syms"][0].shape[0], d["syms"], d["n_deg"], d["blocks"], d["blocks_ids"], f, dv)
    assert _rel(f, d["case1_f"]) < 1e-12 and _rel(dv, d["case1_d2v"]) < 1e-12


def test_batched_device_averages_equal_single(cuda, rocksalt_l2):
    torch = cuda
    d = rocksalt_l2
    ens = _dev_ens(d)
    n = d["X"].shape[1]
    R = torch.as_tensor(np.stack([d[f"case{c}_R1"] for c in range(2)]), device="cuda")
    Y = torch.as_tensor(np.stack([d[f"case{c}_Y1"] for c in range(2)]), device="cuda")
    f = torch.empty((2, n), dtype=torch.float64, device="cuda")
    dv = torch.empty((2, n, n), dtype=torch.float64, device="cuda")
    ens.perturb_average_device(R, Y, f, dv, 1, "fp64")
    torch.cuda.synchronize()
    for c in range(2):
        assert _rel(f[c].cpu().numpy(), d[f"case{c}_f"]) < 1e-12
        assert _rel(dv[c].cpu().numpy(), d[f"case{c}_d2v"]) < 1e-12


def test_bad_blocks_raise_not_exit(cuda, mode10):
    """Argument errors come back as exceptions (the reference's binding calls exit())."""
    from tdscha_b200 import _native
    d = mode10
    blocks = [b.copy() for b in d["blocks"]]
    blocks[1] = blocks[1][::-1].copy()          # not ascending
    with pytest.raises(_native.TdschaError, match="contiguous"):
        _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], blocks, d["blocks_ids"])
    w = d["w"].copy()
    w[1] *= 1.001                               # breaks the degeneracy of block 0
    with pytest.raises(_native.TdschaError, match="degenerate"):
        _native.DeviceEnsemble(d["X"], d["Y"], w, d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    ens = _dev_ens(d)
    with pytest.raises(_native.TdschaError, match="apply_D4"):
        ens.perturb_average(d["case0_R1"], d["case0_Y1"], 2, "fp64")


@pytest.mark.parametrize("L,N", [(3, 40), (4, 24)])
@pytest.mark.parametrize("precision,tol", [("bf16x3", 2e-5), ("tf32x3", 2e-5), ("tf32", 5e-3)])
def test_mixed_modes_against_fp64_all_block_classes(cuda, L, N, precision, tol):
    """The tensor-core symmetry transform / fold (mixed modes) against the FP64 CUDA-core path on
    rock-salt 3x3x3 (blocks up to 42 modes) and 4x4x4 (up to 72): every padded block class."""
    torch = cuda
    from tdscha_b200 import _native
    from tdscha_b200 import rocksalt as RS
    s = RS.make_ensemble(L, N, seed=L)
    ens = _native.DeviceEnsemble(s.X, s.Y, s.w, s.rho, s.T, s.symmetries, s.deg_space, s.blocks_ids)
    n = s.X.shape[1]
    rng = np.random.default_rng(9)
    nb = 3
    R = torch.as_tensor(rng.standard_normal((nb, n)), device="cuda")
    A = rng.standard_normal((nb, n, n))
    Y1 = torch.as_tensor(A + A.transpose(0, 2, 1), device="cuda")
    out = {}
    for prec in ("fp64", precision):
        f = torch.empty((nb, n), dtype=torch.float64, device="cuda")
        dv = torch.empty((nb, n, n), dtype=torch.float64, device="cuda")
        ens.perturb_average_device(R, Y1, f, dv, 1, prec)
        torch.cuda.synchronize()
        out[prec] = (f.cpu().numpy(), dv.cpu().numpy())
    ens.close()
    assert _rel(out[precision][0], out["fp64"][0]) < tol
    assert _rel(out[precision][1], out["fp64"][1]) < tol


@pytest.mark.parametrize("fixture", ["mode10", "rocksalt_l2"])
def test_tcgen05_symmetry_kernels_match(request, cuda, fixture, monkeypatch):
    """The opt-in tcgen05 symmetry transform / fold of the bf16 formats (TDSCHA_SYM_UMMA=1,
    symmetry_umma.cu) against the reference kernel's golden outputs and the default mma.sync path."""
    d = request.getfixturevalue(fixture)
    ens = _dev_ens(d)
    for case in ("case0", "case1", "case2"):
        monkeypatch.delenv("TDSCHA_SYM_UMMA", raising=False)
        f0, d0 = ens.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), "bf16x3")
        monkeypatch.setenv("TDSCHA_SYM_UMMA", "1")
        f1, d1 = ens.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), "bf16x3")
        ef, ed = _rel(f1, d[f"{case}_f"]), _rel(d1, d[f"{case}_d2v"])
        print(f"{fixture} tcgen05 symmetry bf16x3 {case}: f {ef:.2e} d2v {ed:.2e}; vs mma.sync path "
              f"{_rel(f1, f0):.2e} {_rel(d1, d0):.2e}")
        assert ef < TOL["bf16x3"] and ed < TOL["bf16x3"]
        assert _rel(f1, f0) < 1e-4 and _rel(d1, d0) < 1e-4
    monkeypatch.delenv("TDSCHA_SYM_UMMA", raising=False)
    ens.close()


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_lean_symmetry_kernels_are_bit_identical(cuda, rocksalt_l2, precision, monkeypatch):
    """The half-shared-memory symmetry transform and fold (default) and the double-buffered ones
    (TDSCHA_SYM_LEAN=0) form the same tf32 hi / lo values and the same products: identical averages."""
    d = rocksalt_l2
    ens = _dev_ens(d)
    for case in ("case0", "case2"):
        monkeypatch.setenv("TDSCHA_SYM_LEAN", "0")
        f0, d0 = ens.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), precision)
        monkeypatch.delenv("TDSCHA_SYM_LEAN")
        f1, d1 = ens.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), precision)
        assert np.array_equal(f0, f1) and np.array_equal(d0, d1)
    ens.close()
