"""The averages' big contractions over the character classes of the translation subgroup.

On the factorised path (symmetries S_p D_t, D_t in the abelian subgroup of lattice translations)
the [a|b] and Z contractions of the averages run class by class over the characters of the
subgroup: every precision, FP64 included.  TDSCHA_SYM_FREQ=0 (read at every averages call) selects
the contractions over every symmetry row instead.  Checked against each other, against the
reference kernel's semantics (CModules/LanczosFunctions.c:2082-2754, GetPerturbAverageSym) through
the FP64 general path, in configuration and symmetry chunks, and batched.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _system(L, N, seed):
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(L, T=300.0)
    X, Y, rho = RS.sample_ensemble(s, N, seed=seed)
    return X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids


@pytest.fixture(scope="module")
def c1():
    d = np.load(os.path.join(GOLDEN, "c1_reference_chain.npz"))
    nb = int(d["n_blocks"])
    return (d["X"][:40], d["Y"][:40], d["w"], d["rho"][:40], float(d["T"]), [d[f"sym{b}"] for b in range(nb)],
            [d[f"block{b}"] for b in range(nb)], d["blocks_ids"])


def _perturbations(n, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        Y1 = rng.standard_normal((n, n))
        out.append((rng.standard_normal(n), Y1 + Y1.T, i % 2))
    return out


def _both(monkeypatch, ens, R1, Y1, d4, prec):
    monkeypatch.delenv("TDSCHA_SYM_FREQ", raising=False)
    fq = ens.perturb_average(R1, Y1, d4, prec)
    monkeypatch.setenv("TDSCHA_SYM_FREQ", "0")
    fg = ens.perturb_average(R1, Y1, d4, prec)
    monkeypatch.delenv("TDSCHA_SYM_FREQ")
    return fq, fg


@pytest.mark.parametrize("L,N,n_class", [(2, 40, 8), (3, 12, 14), (4, 4, 36)])
def test_fp64_classes_equal_the_symmetry_rows(cuda, monkeypatch, L, N, n_class):
    from tdscha_b200 import _native
    ens = _native.DeviceEnsemble(*_system(L, N, seed=L))
    info = ens.classes()
    assert info["n_class"] == n_class and info["flops_ratio"] < 0.5
    n = ens.n
    for R1, Y1, d4 in _perturbations(n, 2, L):
        (f1, d1), (f0, d0) = _both(monkeypatch, ens, R1, Y1, d4, "fp64")
        print(f"L={L} fp64 d4={d4}: f {_rel(f1, f0):.2e} D {_rel(d1, d0):.2e}")
        assert _rel(f1, f0) < 1e-12 and _rel(d1, d0) < 1e-12


@pytest.mark.parametrize("prec,tol", [("bf16x3", 2e-5), ("tf32x3", 2e-5), ("tf32", 5e-3), ("bf16", 2e-2)])
def test_mixed_classes_against_fp64(cuda, monkeypatch, prec, tol):
    from tdscha_b200 import _native
    ens = _native.DeviceEnsemble(*_system(4, 4, seed=9))
    n = ens.n
    for R1, Y1, d4 in _perturbations(n, 2, 21):
        fr, dr = ens.perturb_average(R1, Y1, d4, "fp64")
        (fq, dq), (fg, dg) = _both(monkeypatch, ens, R1, Y1, d4, prec)
        e_q, e_g = max(_rel(fq, fr), _rel(dq, dr)), max(_rel(fg, fr), _rel(dg, dr))
        print(f"4x4x4 {prec} d4={d4}: classes {e_q:.2e}  symmetry rows {e_g:.2e}")
        assert e_q < tol and e_q < max(3 * e_g, 2e-6), (e_q, e_g)


def test_classes_against_the_reference_fixture(cuda, c1):
    """FP64 on the 2x2x2 reference fixture (384 operations) against the oracle restatement of the
    reference kernel."""
    from oracle import lanczos_oracle as LO
    from tdscha_b200 import _native
    X, Y, w, rho, T, syms, deg, bid = c1
    ens = _native.DeviceEnsemble(X, Y, w, rho, T, syms, deg, bid)
    assert ens.classes()["n_class"] == 8
    n = len(w)
    n_deg = np.array([len(b) for b in deg], dtype=np.intc)
    for R1, Y1, d4 in _perturbations(n, 2, 4):
        fr, dr = LO.perturb_average_sym(X, Y, w, rho, R1, Y1, T, d4, syms, n_deg, deg, bid)
        f, d = ens.perturb_average(R1, Y1, d4, "fp64")
        assert _rel(f, fr) < 1e-12 and _rel(d, dr) < 1e-12


@pytest.mark.parametrize("prec,resident_rows", [("fp64", "0"), ("bf16x3", "0"), ("bf16x3", "1"), ("tf32x3", "1")])
def test_classes_in_configuration_and_coset_chunks(cuda, monkeypatch, prec, resident_rows):
    """Configuration chunks (32 + 18) and coset chunks (5) against the resident single pass: every
    class operand rebuilt per chunk (the default), or, with TDSCHA_CHUNK_RESIDENT_ROWS=1 and a split
    format, the row-major class operands of all configurations resident and the transposed ones
    formed per chunk."""
    from tdscha_b200 import _native
    ens = _native.DeviceEnsemble(*_system(3, 50, seed=2))
    n = ens.n
    (R1, Y1, d4), = _perturbations(n, 1, 8)
    f1, d1 = ens.perturb_average(R1, Y1, 1, prec)
    monkeypatch.setenv("TDSCHA_CONFIG_CHUNK", "32")    # chunks of 32 + 18 configurations
    monkeypatch.setenv("TDSCHA_SYM_CHUNK", "270")      # 10 cosets of 27 per chunk (5 chunks)
    monkeypatch.setenv("TDSCHA_CHUNK_RESIDENT_ROWS", resident_rows)
    f2, d2 = ens.perturb_average(R1, Y1, 1, prec)
    monkeypatch.delenv("TDSCHA_CONFIG_CHUNK")
    monkeypatch.delenv("TDSCHA_SYM_CHUNK")
    monkeypatch.delenv("TDSCHA_CHUNK_RESIDENT_ROWS")
    tol = 1e-12 if prec == "fp64" else 1e-6
    assert _rel(f2, f1) < tol and _rel(d2, d1) < tol


def test_batched_classes_equal_single_vectors(cuda):
    import torch
    from tdscha_b200 import _native
    ens = _native.DeviceEnsemble(*_system(3, 12, seed=4))
    n = ens.n
    rng = np.random.default_rng(3)
    R1 = rng.standard_normal((3, n))
    Y1 = rng.standard_normal((3, n, n))
    Y1 = Y1 + Y1.transpose(0, 2, 1)
    dev = torch.device("cuda")
    for prec in ("fp64", "bf16x3"):
        f = torch.zeros((3, n), dtype=torch.float64, device=dev)
        d = torch.zeros((3, n, n), dtype=torch.float64, device=dev)
        ens.perturb_average_device(torch.as_tensor(R1, device=dev), torch.as_tensor(Y1, device=dev), f, d, 1, prec)
        torch.cuda.synchronize()
        for k in range(3):
            fk, dk = ens.perturb_average(R1[k], Y1[k], 1, prec)
            tol = 1e-13 if prec == "fp64" else 1e-6
            assert _rel(f[k].cpu().numpy(), fk) < tol and _rel(d[k].cpu().numpy(), dk) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("bf16x3", 1e-4), ("tf32x3", 2e-5)])
def test_vjp_classes_equal_the_symmetry_rows(cuda, monkeypatch, prec, tol):
    """The averages' VJP (d<fbar, f_av> + <Dbar, D_av> / d(Y, rho)) on the character classes against
    the same VJP over every symmetry row in FP64 (TDSCHA_VJP_FREQ=0)."""
    import torch
    from tdscha_b200 import _native
    ens = _native.DeviceEnsemble(*_system(3, 24, seed=6))
    N, n = 24, ens.n
    rng = np.random.default_rng(17)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)   # noqa: E731
    R1, Y1 = rng.standard_normal((3, n)), rng.standard_normal((3, n, n))
    Ys = t(Y1 + Y1.transpose(0, 2, 1))
    fb, Db = rng.standard_normal((3, n)), rng.standard_normal((3, n, n))
    Db = t(Db + Db.transpose(0, 2, 1))

    def vjp(precision, rows):
        if rows:
            monkeypatch.setenv("TDSCHA_VJP_FREQ", "0")
        else:
            monkeypatch.delenv("TDSCHA_VJP_FREQ", raising=False)
        Yb = torch.zeros((N, n), dtype=torch.float64, device=dev)
        rb = torch.zeros(N, dtype=torch.float64, device=dev)
        ens.perturb_average_vjp(t(R1), Ys, t(fb), Db, Yb, rb, precision=precision)
        torch.cuda.synchronize()
        monkeypatch.delenv("TDSCHA_VJP_FREQ", raising=False)
        return Yb.cpu().numpy(), rb.cpu().numpy()

    Y0, r0 = vjp("fp64", True)
    Yc, rc = vjp(prec, False)
    print(f"{prec}: Ybar {_rel(Yc, Y0):.2e}  rhobar {_rel(rc, r0):.2e}")
    assert _rel(Yc, Y0) < tol and _rel(rc, r0) < tol


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_fused_cd_weights_equal_the_contraction(cuda, monkeypatch, prec):
    """The thin [c|d] contraction formed inside the weights kernel (TDSCHA_FREQ_FUSED_CD=1) against
    the grouped contraction plus the separate weights kernel (the default), and both against FP64."""
    from tdscha_b200 import _native
    ens = _native.DeviceEnsemble(*_system(4, 4, seed=12))
    n = ens.n
    for R1, Y1, d4 in _perturbations(n, 2, 31):
        fr, dr = ens.perturb_average(R1, Y1, d4, "fp64")
        monkeypatch.setenv("TDSCHA_FREQ_FUSED_CD", "1")
        ff, df = ens.perturb_average(R1, Y1, d4, prec)
        monkeypatch.delenv("TDSCHA_FREQ_FUSED_CD")
        fs, ds = ens.perturb_average(R1, Y1, d4, prec)
        e_f, e_s = max(_rel(ff, fr), _rel(df, dr)), max(_rel(fs, fr), _rel(ds, dr))
        print(f"{prec} d4={d4}: fused {e_f:.2e}  separate {e_s:.2e}")
        assert e_f < max(1.5 * e_s, 2e-6)
