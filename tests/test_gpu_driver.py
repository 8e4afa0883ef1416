"""The stand-alone Lanczos program tdscha_lanczos_b200 (the counterpart of the reference's
tdscha-lanczos.x, CModules/main.cpp + Lanczos.cpp) on files written by prepare_input_files:
same coefficients and basis as the Python chain, restart from its own output files, refusal of
the flag combinations on which the reference program and the Python class disagree."""
import json
import os
import subprocess
import types

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lanczos(d):
    from tdscha_b200 import DynamicalLanczos as DL
    n = d["X"].shape[1]
    ens = types.SimpleNamespace(T=d["T"], nat=16, m=np.ones(48), w=d["w"], pols=np.eye(48, n), N=len(d["rho"]),
                                rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"], deg_space=d["blocks"],
                                blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)
    L = DL.Lanczos(ens)
    L.init()
    return L


def _run(root, *args):
    from tdscha_b200 import build
    return subprocess.run([build.DRIVER_PATH, root, "--quiet", *args], capture_output=True, text=True, timeout=600)


def test_driver_matches_python_chain_and_restarts(cuda, tmp_path, rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    L.prepare_mode(3)
    L.prepare_input_files("run", n_steps=4, directory=str(tmp_path))
    root = os.path.join(str(tmp_path), "run")
    r = _run(root)
    assert r.returncode == 0, r.stderr
    js = json.load(open(root + ".json"))
    js.update(n_steps=8, restart=True, step_done=4)
    json.dump(js, open(root + ".json", "w"))
    r = _run(root)
    assert r.returncode == 0, r.stderr
    abc = np.loadtxt(root + ".abc")
    L.run_FT(8, verbose=False)
    a, b, c = (np.array(x) for x in (L.a_coeffs, L.b_coeffs, L.c_coeffs))
    assert abc.shape == (8, 3)
    for col, ref in ((0, a[:8]), (1, b[:8]), (2, c[:8])):
        assert np.abs(abc[:, col] - ref).max() <= 1e-10 * np.abs(ref).max()
    Q = np.loadtxt(root + ".qbasis.out")
    P = np.loadtxt(root + ".pbasis.out")
    assert Q.shape == (9, len(L.psi)) and P.shape == Q.shape
    # the program restarts from its files at step 4 in a process of its own, so its FP64 roundings
    # need not match the Python chain's bit for bit; on this 6-configuration ensemble the bi-conjugate
    # recurrence amplifies such differences to ~5e-9 of the vectors' size by step 8 (a, b, c above
    # agree to 1e-10)
    for got, ref in ((Q[-1], L.basis_Q[8]), (P[-1], L.basis_P[8])):
        assert np.abs(got - ref).max() <= 2e-8 * np.abs(ref).max()
    assert np.abs(np.loadtxt(root + ".snorm.out") - np.array(L.s_norm[:9])).max() <= 1e-9 * max(L.s_norm[:9])
    # the results load back into a Lanczos object and give the same G(w)
    L2 = _lanczos(rocksalt_l2)
    L2.load_from_input_files("run", directory=str(tmp_path))
    w = np.linspace(0, 4e-3, 50)
    L.a_coeffs, L.b_coeffs, L.c_coeffs = L.a_coeffs[:8], L.b_coeffs[:8], L.c_coeffs[:8]
    g1 = L.get_green_function_continued_fraction(w, smearing=1e-5)
    g2 = L2.get_green_function_continued_fraction(w, smearing=1e-5)
    assert np.abs(g1 - g2).max() <= 1e-9 * np.abs(g1).max()


def test_driver_refuses_wigner_and_quartic_only(cuda, tmp_path, rocksalt_l2):
    L = _lanczos(rocksalt_l2)
    L.prepare_mode(1)
    root = os.path.join(str(tmp_path), "run")
    L.use_wigner = True
    L.prepare_input_files("run", n_steps=2, directory=str(tmp_path))
    r = _run(root)
    assert r.returncode != 0 and "use_wigner" in r.stderr
    L.use_wigner, L.ignore_v3 = False, True
    L.prepare_input_files("run", n_steps=2, directory=str(tmp_path))
    r = _run(root)
    assert r.returncode != 0 and "ignore_v3" in r.stderr
