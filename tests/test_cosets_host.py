"""Host analysis of the factorised symmetry path (tdscha_symmetry_cosets), no device needed.

The averages' symmetry transform Y~_j = S_j^T Ys S_j and fold S_j W S_j^T (reference:
CModules/LanczosFunctions.c:2158-2170, the symmetry loop of GetPerturbAverageSym) are evaluated per
coset of the subgroup K that acts trivially on one degenerate block: S_j = S_p D_j with p the coset's
representative and D_j in K, and in the rotated basis of every degenerate block D_j has non-zeros only
on a 1 x 1 / 2 x 2 pattern (mode q and its partner).  These tests check that factorisation on the
symmetry tables of the rock-salt 2x2x2 reference fixture and of the 4x4x4 benchmark system.
"""
import os

import numpy as np
import pytest

from tdscha_b200 import _native

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixture_tables():
    d = np.load(os.path.join(HERE, "golden", "c1_reference_chain.npz"))
    return [d[f"sym{b}"] for b in range(int(d["n_blocks"]))]


def _check(tables, res, n_check=None, seed=0):
    N_sym = tables[0].shape[0]
    sub, ncos = res["coset_size"], res["n_cosets"]
    assert sub * ncos == N_sym
    assert sorted(res["order"].tolist()) == list(range(N_sym))
    partner = res["partner"]
    assert np.array_equal(partner[partner], np.arange(len(partner)))     # an involution
    rng = np.random.default_rng(seed)
    rows = np.arange(N_sym) if n_check is None else rng.choice(N_sym, n_check, replace=False)
    starts = np.cumsum([0] + [t.shape[1] for t in tables])
    worst_pattern, worst_transform = 0.0, 0.0
    Ys = {}
    for b, t in enumerate(tables):
        R = res["R"][b]
        d = R.shape[0]
        assert np.abs(R.T @ R - np.eye(d)).max() < 1e-10
        for c in range(b, len(tables)):
            Ys[b, c] = rng.standard_normal((d, tables[c].shape[1]))
    rot = [[R.T @ t[j] @ R for j in range(N_sym)] for R, t in zip(res["R"], tables)]
    for r in rows:
        j = res["order"][r]
        p = res["order"][(r // sub) * sub]
        for b in range(len(tables)):
            D = rot[b][p].T @ rot[b][j]
            d = D.shape[0]
            loc = partner[starts[b]:starts[b] + d] - starts[b]
            mask = np.zeros((d, d), bool)
            mask[np.arange(d), np.arange(d)] = True
            mask[loc, np.arange(d)] = True
            if (~mask).any():
                worst_pattern = max(worst_pattern, np.abs(D[~mask]).max())
        # transform of one block pair through the representative: D^T (S_p^T Y S_p) D
        b, c = 0, len(tables) - 1
        Db, Dc = rot[b][p].T @ rot[b][j], rot[c][p].T @ rot[c][j]
        U = rot[b][p].T @ Ys[b, c] @ rot[c][p]
        worst_transform = max(worst_transform, np.abs(Db.T @ U @ Dc - rot[b][j].T @ Ys[b, c] @ rot[c][j]).max())
    assert worst_pattern < 1e-9
    assert worst_transform < 1e-12
    assert res["offpattern"] < 1e-9


def test_cosets_of_the_reference_fixture():
    tables = _fixture_tables()
    res = _native.symmetry_cosets(tables)
    assert res is not None
    assert (res["n_cosets"], res["coset_size"]) == (48, 8)   # O_h x the 8 translations of 2x2x2
    _check(tables, res)


def test_cosets_of_the_benchmark_system():
    from tdscha_b200 import rocksalt as RS
    system = RS.build_system(4)
    res = _native.symmetry_cosets(system.symmetries)
    assert res is not None
    assert (res["n_cosets"], res["coset_size"]) == (48, 64)
    paired = int((res["partner"] != np.arange(len(res["partner"]))).sum())
    assert paired > 0                                          # complex characters: 2 x 2 blocks
    _check(system.symmetries, res, n_check=96)


def test_group_without_the_structure():
    # identity and inversion only: no proper kernel of order >= 4, the general path stays
    tables = [np.stack([np.eye(3), -np.eye(3)]), np.stack([np.eye(2), -np.eye(2)])]
    assert _native.symmetry_cosets(tables) is None
