"""The factorised symmetry path against the general one.

An ensemble whose symmetry group has the coset structure (the rock-salt fixtures: O_h x lattice
translations) is stored in the rotated mode basis, and its mixed-precision averages run the dense
symmetry transform / fold over the 48 coset representatives plus the four-term expansion over each
coset.  TDSCHA_SYM_COSETS=0 at creation keeps the given basis and the general per-symmetry kernels.
Both are checked against each other and against FP64 (reference semantics:
CModules/LanczosFunctions.c:2082-2754, the symmetrised averages of GetPerturbAverageSym).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _make(monkeypatch, general, X, Y, w, rho, T, syms, deg_space, blocks_ids):
    from tdscha_b200 import _native
    if general:
        monkeypatch.setenv("TDSCHA_SYM_COSETS", "0")
    else:
        monkeypatch.delenv("TDSCHA_SYM_COSETS", raising=False)
    ens = _native.DeviceEnsemble(X, Y, w, rho, T, syms, deg_space, blocks_ids)
    monkeypatch.delenv("TDSCHA_SYM_COSETS", raising=False)
    return ens


@pytest.fixture(scope="module")
def c1():
    d = np.load(os.path.join(GOLDEN, "c1_reference_chain.npz"))
    nb = int(d["n_blocks"])
    syms = [d[f"sym{b}"] for b in range(nb)]
    deg = [d[f"block{b}"] for b in range(nb)]
    return d["X"], d["Y"], d["w"], d["rho"], float(d["T"]), syms, deg, d["blocks_ids"]


@pytest.fixture(scope="module")
def l4():
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(4, T=300.0)
    X, Y, rho = RS.sample_ensemble(s, 16, seed=7)
    return X, Y, s.w, rho, s.T, s.symmetries, s.deg_space, s.blocks_ids


def _perturbations(n, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        Y1 = rng.standard_normal((n, n))
        out.append((rng.standard_normal(n), Y1 + Y1.T, i % 2))
    return out


def test_rotated_ensemble_reports_its_factorisation(cuda, monkeypatch, c1):
    on = _make(monkeypatch, False, *c1)
    off = _make(monkeypatch, True, *c1)
    info = on.cosets()
    assert info["rotated"] and (info["n_cosets"], info["coset_size"]) == (48, 8)
    assert info["offpattern"] < 1e-9
    assert off.cosets() == dict(rotated=False, n_cosets=0, coset_size=0, offpattern=0.0)


def test_fp64_averages_unchanged_by_the_rotated_basis(cuda, monkeypatch, c1):
    on = _make(monkeypatch, False, *c1)
    off = _make(monkeypatch, True, *c1)
    n = len(c1[2])
    for R1, Y1, d4 in _perturbations(n, 2, 3):
        f1, d1 = on.perturb_average(R1, Y1, d4, "fp64")
        f0, d0 = off.perturb_average(R1, Y1, d4, "fp64")
        assert _rel(f1, f0) < 1e-12 and _rel(d1, d0) < 1e-12


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_mixed_averages_on_the_cosets_2x2x2(cuda, monkeypatch, c1, prec):
    on = _make(monkeypatch, False, *c1)
    off = _make(monkeypatch, True, *c1)
    n = len(c1[2])
    for R1, Y1, d4 in _perturbations(n, 2, 5):
        fr, dr = off.perturb_average(R1, Y1, d4, "fp64")
        fc, dc = on.perturb_average(R1, Y1, d4, prec)
        fg, dg = off.perturb_average(R1, Y1, d4, prec)
        e_cos, e_gen = max(_rel(fc, fr), _rel(dc, dr)), max(_rel(fg, fr), _rel(dg, dr))
        print(f"2x2x2 {prec} d4={d4}: cosets {e_cos:.2e}  general {e_gen:.2e}")
        assert e_cos < max(3 * e_gen, 2e-6), (e_cos, e_gen)


def test_vjp_unchanged_by_the_rotated_basis(cuda, monkeypatch, c1):
    import torch
    on = _make(monkeypatch, False, *c1)
    off = _make(monkeypatch, True, *c1)
    X = c1[0]
    N, n = X.shape
    rng = np.random.default_rng(11)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    R1, Y1 = rng.standard_normal((2, n)), rng.standard_normal((2, n, n))
    Ys = t(Y1 + Y1.transpose(0, 2, 1))
    fb, Db = rng.standard_normal((2, n)), rng.standard_normal((2, n, n))
    Db = t(Db + Db.transpose(0, 2, 1))
    out = []
    for ens in (on, off):
        Yb = torch.zeros((N, n), dtype=torch.float64, device=dev)
        rb = torch.zeros(N, dtype=torch.float64, device=dev)
        ens.perturb_average_vjp(t(R1), Ys, t(fb), Db, Yb, rb)
        torch.cuda.synchronize()
        out.append((Yb.cpu().numpy(), rb.cpu().numpy()))
    assert _rel(out[0][0], out[1][0]) < 1e-10 and _rel(out[0][1], out[1][1]) < 1e-10


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_mixed_averages_on_the_cosets_4x4x4(cuda, monkeypatch, l4, prec):
    on = _make(monkeypatch, False, *l4)
    off = _make(monkeypatch, True, *l4)
    info = on.cosets()
    assert (info["n_cosets"], info["coset_size"]) == (48, 64)
    n = len(l4[2])
    for R1, Y1, d4 in _perturbations(n, 2, 9):
        fr, dr = off.perturb_average(R1, Y1, d4, "fp64")
        fc, dc = on.perturb_average(R1, Y1, d4, prec)
        fg, dg = off.perturb_average(R1, Y1, d4, prec)
        e_cos, e_gen = max(_rel(fc, fr), _rel(dc, dr)), max(_rel(fg, fr), _rel(dg, dr))
        print(f"4x4x4 {prec} d4={d4}: cosets {e_cos:.2e}  general {e_gen:.2e}")
        assert e_cos < 5e-5 and e_cos < max(3 * e_gen, 2e-6), (e_cos, e_gen)


def test_coset_path_in_symmetry_chunks(cuda, monkeypatch, l4):
    on = _make(monkeypatch, False, *l4)
    n = len(l4[2])
    (R1, Y1, d4), = _perturbations(n, 1, 13)
    f1, d1 = on.perturb_average(R1, Y1, d4, "bf16x3")
    monkeypatch.setenv("TDSCHA_SYM_CHUNK", "128")   # two cosets of 64 per chunk
    f2, d2 = on.perturb_average(R1, Y1, d4, "bf16x3")
    monkeypatch.delenv("TDSCHA_SYM_CHUNK")
    assert _rel(f2, f1) < 1e-6 and _rel(d2, d1) < 1e-6
