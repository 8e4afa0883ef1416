"""Full operator, bi-conjugate Lanczos and continued fraction on the GPU against the oracle and the
reference's golden chain."""
import types

import numpy as np
import pytest

from oracle import lanczos_oracle as LO

pytestmark = pytest.mark.gpu


def _ensemble_obj(d, nat=16):
    n = d["X"].shape[1]
    return types.SimpleNamespace(T=d["T"], nat=nat, m=np.ones(3 * nat), w=d["w"], pols=np.eye(3 * nat, n), N=len(d["rho"]),
                                 rho=d["rho"], X=d["X"], Y=d["Y"], symmetries=d["syms"], deg_space=d["blocks"],
                                 blocks_ids=d["blocks_ids"], supercell=(2, 2, 2), nat_uc=2)


def _lanczos(d, **kw):
    from tdscha_b200 import DynamicalLanczos as DL
    L = DL.Lanczos(_ensemble_obj(d), **kw)
    L.init()
    return L


def _oracle(d):
    return LO.OracleLanczos(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])


FLAGS = [dict(), dict(transpose=True), dict(use_wigner=True), dict(reverse_L=True, shift_value=3e-6),
         dict(ignore_v4=True), dict(ignore_harmonic=True), dict(ignore_v3=True), dict(use_wigner=True, transpose=True)]


@pytest.mark.parametrize("flags", FLAGS, ids=lambda f: "-".join(f) or "default")
def test_apply_full_L_matches_oracle(cuda, rocksalt_l2, flags):
    d = rocksalt_l2
    flags = dict(flags)
    transpose = flags.pop("transpose", False)
    L = _lanczos(d, use_wigner=flags.pop("use_wigner", False))
    O = _oracle(d)
    O.use_wigner = L.use_wigner
    for k, v in flags.items():
        setattr(L, k, v)
        setattr(O, k, v)
    n = L.n_modes
    psi = np.random.default_rng(5).standard_normal(n + n * (n + 1)) * 1e-2
    got = L.apply_full_L(psi.copy(), transpose=transpose)
    ref = O.apply_full_L(psi.copy(), transpose=transpose)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, err


def test_chain_replays_reference_run(cuda, mode10):
    """GPU FP64 chain from the reference's first Krylov vector reproduces its a, b, c (steps 0-6
    to 1e-11 relative; c_4 to the reference test constant, rel 1e-6)."""
    d = mode10
    L = _lanczos(d)
    L.psi = d["q0"].copy()
    L.run_FT(10, verbose=False)
    a, b, c = (np.array(x) for x in (L.a_coeffs, L.b_coeffs, L.c_coeffs))
    for got, ref in ((a, d["a_coeffs"]), (b, d["b_coeffs"]), (c, d["c_coeffs"])):
        rel = np.abs(got[:7] - ref[:7]) / np.abs(ref[:7])
        assert rel.max() < 1e-11, rel
    assert abs(c[4] - d["c4_test_constant"]) / d["c4_test_constant"] < 1e-6


def test_chain_matches_oracle_chain_rocksalt(cuda, rocksalt_l2):
    d = rocksalt_l2
    L = _lanczos(d)
    O = _oracle(d)
    L.prepare_mode(3)
    O.prepare_mode(3)
    L.run_FT(12, verbose=False)
    O.run_FT(12)
    a, ao = np.array(L.a_coeffs), np.array(O.a_coeffs)
    b, bo = np.array(L.b_coeffs), np.array(O.b_coeffs)
    k = min(len(a), len(ao), 8)
    assert np.abs(a[:k] - ao[:k]).max() / np.abs(ao[:k]).max() < 1e-10
    assert np.abs(b[:k] - bo[:k]).max() / np.abs(bo[:k]).max() < 1e-10


def test_batched_chains_equal_independent_chains(cuda, rocksalt_l2):
    from tdscha_b200 import DynamicalLanczos as DL
    d = rocksalt_l2
    base = _lanczos(d)
    chains = []
    for s in range(3):
        L = DL.Lanczos(_ensemble_obj(d))
        L.symmetries, L.degenerate_space, L.sym_block_id = base.symmetries, base.degenerate_space, base.sym_block_id
        L.N_degeneracy, L.initialized, L.device_ensemble = base.N_degeneracy, True, base.device_ensemble
        L.prepare_random(seed=s, sector="all")
        chains.append(L)
    DL.run_FT_batched(chains, 6)
    for s, L in enumerate(chains):
        S = _lanczos(d)
        S.prepare_random(seed=s, sector="all")
        S.run_FT(6, verbose=False)
        assert np.allclose(L.a_coeffs, S.a_coeffs, rtol=1e-10, atol=0)
        assert np.allclose(L.c_coeffs, S.c_coeffs, rtol=1e-10, atol=0)


@pytest.mark.parametrize("opts", [dict(use_terminator=True), dict(use_terminator=False, smearing=1e-5),
                                  dict(use_terminator=True, last_average=3), dict(wigner=True),
                                  dict(reverse=True, shift=1e-7), dict(symmetric=True)])
def test_continued_fraction_matches_oracle(cuda, mode10, opts):
    d = mode10
    L = _lanczos(d, use_wigner=opts.get("wigner", False))
    O = _oracle(d)
    O.use_wigner = L.use_wigner
    L.a_coeffs, L.b_coeffs = list(d["a_coeffs"][:8]), list(d["b_coeffs"][:8])
    L.c_coeffs = [] if opts.get("symmetric") else list(d["c_coeffs"][:8])
    O.a_coeffs, O.b_coeffs, O.c_coeffs = L.a_coeffs, L.b_coeffs, L.c_coeffs
    for obj in (L, O):
        obj.reverse_L = opts.get("reverse", False)
        obj.shift_value = opts.get("shift", 0.0)
        obj.perturbation_modulus = 2.5
    w = np.linspace(0, 4e-3, 257)
    kw = dict(use_terminator=opts.get("use_terminator", True), last_average=opts.get("last_average", 1),
              smearing=opts.get("smearing", 0.0))
    g = L.get_green_function_continued_fraction(w, **kw)
    go = O.get_green_function_continued_fraction(w, **kw)
    assert np.abs(g - go).max() <= 1e-10 * np.abs(go).max()


@pytest.mark.parametrize("n_rep_orth", [1, 2])
def test_gram_schmidt_step_matches_oracle(cuda, n_rep_orth):
    """The device Gram-Schmidt of one new Lanczos pair (DynamicalLanczos.py:6244-6316) against the
    oracle's restatement on the same inputs: a window of 4 basis pairs, with and without the
    symmetric Wigner mask."""
    torch = cuda
    from tdscha_b200 import DynamicalLanczos as DL
    rng = np.random.default_rng(3 + n_rep_orth)
    n = 12
    ln = n + n * (n + 1)
    basis_Q = [rng.standard_normal(ln) for _ in range(6)]
    basis_P = [rng.standard_normal(ln) for _ in range(6)]
    q, p = rng.standard_normal(ln), rng.standard_normal(ln)
    c = 0.37
    o = LO.OracleLanczos.__new__(LO.OracleLanczos)
    o.n_modes = n
    for mask in (None, o.mask_dot_wigner()):
        dot = (lambda a, b: a.dot(b)) if mask is None else (lambda a, b: a.dot(b * mask))   # noqa: E731
        rq, rp, rs, _ = LO.gram_schmidt(q, p, basis_Q, basis_P, n_rep_orth, 4, c, dot)
        window = [(torch.as_tensor(Q, device="cuda"), torch.as_tensor(P, device="cuda")) for Q, P in zip(basis_Q[-4:], basis_P[-4:])]
        tm = None if mask is None else torch.as_tensor(mask, device="cuda")
        gq, gp, gs, _ = DL._gram_schmidt(torch.as_tensor(q, device="cuda"), torch.as_tensor(p, device="cuda"), window,
                                         n_rep_orth, c, tm)
        assert np.abs(gq.cpu().numpy() - rq).max() <= 1e-12 * np.abs(rq).max()
        assert np.abs(gp.cpu().numpy() - rp).max() <= 1e-12 * np.abs(rp).max()
        assert abs(gs - rs) <= 1e-12 * abs(rs)


@pytest.mark.parametrize("n_rep_orth", [1, 2])
def test_chain_with_gram_schmidt_matches_oracle(cuda, rocksalt_l2, n_rep_orth):
    """run_FT with Gram-Schmidt re-orthogonalisation against the oracle's chain (n_ortho = 4, shorter
    than the chain); on this 6-configuration ensemble both chains agree to ~1e-11 over 10 steps, the
    size of the re-orthogonalisation's own effect, which the test above checks exactly."""
    d = rocksalt_l2
    L = _lanczos(d)
    O = _oracle(d)
    L.prepare_mode(3)
    O.prepare_mode(3)
    L.run_FT(10, verbose=False, n_rep_orth=n_rep_orth, n_ortho=4)
    O.run_FT(10, n_rep_orth=n_rep_orth, n_ortho=4)
    assert len(L.a_coeffs) == len(O.a_coeffs)
    for attr in ("a_coeffs", "b_coeffs", "c_coeffs", "s_norm"):
        ref = np.array(getattr(O, attr))
        assert np.abs(np.array(getattr(L, attr)) - ref).max() <= 1e-9 * np.abs(ref).max(), attr
