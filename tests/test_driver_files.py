"""Input / output files of the stand-alone Lanczos program (DynamicalLanczos.py:815-1000, 3572-3595):
the writer produces the reference's file set and formats, the loaders read them back.  No GPU."""
import json
import os
import types

import numpy as np


def _lanczos(d):
    from tdscha_b200 import DynamicalLanczos as DL
    n = d["X"].shape[1]
    ens = types.SimpleNamespace(T=d["T"], nat=16, m=np.linspace(1, 2, 48), w=d["w"], pols=np.eye(48, n),
                                N=len(d["rho"]), rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"],
                                deg_space=d["blocks"], blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)
    L = DL.Lanczos(ens)
    L.symmetries = [np.asarray(s, dtype=np.double) for s in d["syms"]]
    L.degenerate_space = [np.asarray(b, dtype=np.intc) for b in d["blocks"]]
    L.N_degeneracy = np.array([len(b) for b in d["blocks"]], dtype=np.intc)
    L.sym_block_id = np.asarray(d["blocks_ids"], dtype=np.intc)
    return L


def test_prepare_input_files_layout(tmp_path, rocksalt_l2):
    d = rocksalt_l2
    L = _lanczos(d)
    L.prepare_mode(2)
    L.reverse_L, L.shift_value = True, 1e-5
    L.prepare_input_files("run", n_steps=7, directory=str(tmp_path))
    root = os.path.join(str(tmp_path), "run")
    js = json.load(open(root + ".json"))
    assert js["n_steps"] == 7 and js["T"] == L.T and js["data"]["n_modes"] == L.n_modes
    assert js["data"]["n_syms"] == L.symmetries[0].shape[0] and js["data"]["n_blocks"] == len(L.symmetries)
    assert js["data"]["reverse"] is True and js["data"]["shift"] == 1e-5
    assert np.array_equal(np.loadtxt(root + ".X.dat"), L.X) and np.array_equal(np.loadtxt(root + ".Y.dat"), L.Y)
    assert np.array_equal(np.loadtxt(root + ".psi"), L.psi)
    assert np.array_equal(np.loadtxt(root + ".ndegs", dtype=int), L.N_degeneracy)
    assert np.array_equal(np.loadtxt(root + ".blockid", dtype=int), L.sym_block_id)
    for i, S in enumerate(L.symmetries):
        assert np.array_equal(np.atleast_1d(np.loadtxt(root + f".block{i}", dtype=int)), L.degenerate_space[i])
        text = open(root + f".symsb{i}").read()
        vals = np.array(text.split(), dtype=float).reshape(S.shape)
        assert np.abs(vals - S).max() <= 1e-15 + 1e-16 * np.abs(S).max()
        # one line per row of each table, a blank line after each symmetry, 23 characters per value
        lines = text.split("\n")
        assert len(lines[0]) == 23 * S.shape[2] and lines[S.shape[1]] == ""


def test_load_from_input_files_and_abc(tmp_path, rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    L.prepare_input_files("run", n_steps=3, directory=str(tmp_path))
    root = os.path.join(str(tmp_path), "run")
    abc = np.array([[1.5, 0.25, 0.5], [2.5, 0.125, 0.75]])
    np.savetxt(root + ".abc", abc)
    np.savetxt(root + ".snorm.out", [1.0, 0.9, 0.8])
    L.load_from_input_files("run", directory=str(tmp_path))
    assert np.array_equal(L.a_coeffs, abc[:, 0]) and np.array_equal(L.c_coeffs, abc[:, 2])
    assert np.array_equal(L.s_norm, [1.0, 0.9, 0.8])
    L.save_abc(root + ".abc2")
    L2 = _lanczos(rocksalt_l2)
    L2.load_abc(root + ".abc2")
    assert np.array_equal(L2.b_coeffs, abc[:, 1])
