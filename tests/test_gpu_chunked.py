"""Configuration-chunked averages (the large-ensemble path: operands rebuilt per chunk of
configurations, Z and F accumulated across chunks) against the golden outputs and against the
resident-operand path.  TDSCHA_CONFIG_CHUNK forces the chunk size; it is read on every call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "tf32x3": 2e-5, "bf16x3": 2e-4, "tf32": 2e-2, "bf16": 1e-1}


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture
def chunk_env(monkeypatch):
    def set_chunk(nc):
        if nc is None:
            monkeypatch.delenv("TDSCHA_CONFIG_CHUNK", raising=False)
        else:
            monkeypatch.setenv("TDSCHA_CONFIG_CHUNK", str(nc))
    return set_chunk


@pytest.mark.parametrize("precision", list(TOL))
def test_chunked_matches_golden(cuda, mode10, chunk_env, precision):
    from tdscha_b200 import _native
    d = mode10
    ens = _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    chunk_env(3)                                   # chunks of 3, 3, 3, 1 configurations
    for case in ("case0", "case1", "case2"):
        f, dv = ens.perturb_average(d[f"{case}_R1"], d[f"{case}_Y1"], int(d[f"{case}_d4"]), precision)
        assert _rel(f, d[f"{case}_f"]) < TOL[precision], case
        assert _rel(dv, d[f"{case}_d2v"]) < TOL[precision], case
    chunk_env(None)
    ens.close()


@pytest.mark.parametrize("precision", ["fp64", "bf16x3", "tf32x3"])
def test_chunked_equals_resident(cuda, chunk_env, precision):
    """Batched device call on a 2x2x2 rock-salt ensemble of 777 configurations: chunks of 128
    (ragged last chunk of 9) against all configurations at once."""
    torch = cuda
    from tdscha_b200 import _native
    from tdscha_b200 import rocksalt as RS
    s = RS.make_ensemble(2, 777, seed=3)
    ens = _native.DeviceEnsemble(s.X, s.Y, s.w, s.rho, s.T, s.symmetries, s.deg_space, s.blocks_ids)
    n = s.X.shape[1]
    rng = np.random.default_rng(5)
    nb = 3
    R = torch.as_tensor(rng.standard_normal((nb, n)), device="cuda")
    A = rng.standard_normal((nb, n, n))
    Y1 = torch.as_tensor(A + A.transpose(0, 2, 1), device="cuda")
    out = {}
    for nc in (None, 128):
        chunk_env(nc)
        f = torch.empty((nb, n), dtype=torch.float64, device="cuda")
        dv = torch.empty((nb, n, n), dtype=torch.float64, device="cuda")
        ens.perturb_average_device(R, Y1, f, dv, 1, precision)
        torch.cuda.synchronize()
        out[nc] = (f.cpu().numpy(), dv.cpu().numpy())
    chunk_env(None)
    ens.close()
    tol = 1e-12 if precision == "fp64" else TOL[precision]
    assert _rel(out[128][0], out[None][0]) < tol
    assert _rel(out[128][1], out[None][1]) < tol


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3", "bf16"])
def test_split_k_equals_single_launch(cuda, rocksalt_l2, monkeypatch, precision):
    """The projection contraction split over K slices (TDSCHA_KSPLIT, accumulate epilogue) against
    one launch over the whole K: slices of 384, 384, 320 for K = 1088."""
    from tdscha_b200 import _native
    d = rocksalt_l2
    ens = _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    out = {}
    for ks in ("0", "400"):
        monkeypatch.setenv("TDSCHA_KSPLIT", ks)
        out[ks] = ens.perturb_average(d["case1_R1"], d["case1_Y1"], 1, precision)
        assert _rel(out[ks][1], d["case1_d2v"]) < TOL[precision]
    monkeypatch.delenv("TDSCHA_KSPLIT")
    ens.close()
    tol = 1e-5 if precision != "bf16" else 1e-2
    assert _rel(out["400"][0], out["0"][0]) < tol
    assert _rel(out["400"][1], out["0"][1]) < tol


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_symmetry_chunks_equal_one_chunk(cuda, rocksalt_l2, monkeypatch, precision):
    """The symmetry dimension in chunks (what a tight workspace budget gives): 384 operations in
    chunks of 80 (a multiple of the 16-operation fold group; last chunk 64) against one chunk."""
    from tdscha_b200 import _native
    d = rocksalt_l2
    out = {}
    for sc in (None, "80"):
        if sc is None:
            monkeypatch.delenv("TDSCHA_SYM_CHUNK", raising=False)
        else:
            monkeypatch.setenv("TDSCHA_SYM_CHUNK", sc)
        ens = _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
        out[sc] = ens.perturb_average(d["case2_R1"], d["case2_Y1"], int(d["case2_d4"]), precision)
        ens.close()
    monkeypatch.delenv("TDSCHA_SYM_CHUNK", raising=False)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert _rel(out["80"][0], out[None][0]) < tol
    assert _rel(out["80"][1], out[None][1]) < tol
    assert _rel(out["80"][1], d["case2_d2v"]) < (1e-12 if precision == "fp64" else TOL[precision])
