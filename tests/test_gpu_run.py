"""The multi-system, graph-captured run (tdscha_lanczos_run_device through run_FT_multi) against
per-system run_FT_batched chains: same coefficients, graph replay identical to eager steps,
breakdowns ending a chain as run_FT does."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(L, N, seed, T=300.0):
    from tdscha_b200 import DynamicalLanczos as DL
    from tdscha_b200 import rocksalt as RS
    ens = RS.make_ensemble(L, N, T=T, seed=seed)
    base = DL.Lanczos(ens)
    base.init()
    return base


def _chains(base, seeds, sector="all"):
    out = []
    for s in seeds:
        L = base.new_chain()
        L.prepare_random(seed=s, sector=sector)
        out.append(L)
    return out


def _coeffs(chains):
    return [(np.array(L.a_coeffs), np.array(L.b_coeffs), np.array(L.c_coeffs)) for L in chains]


@pytest.fixture(scope="module")
def systems(cuda):
    # uneven: 2x2x2 with 300 and 3x3x3 with 120 configurations
    return _system(2, 300, seed=1), _system(3, 120, seed=2)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_multi_equals_batched_per_system(systems, precision):
    from tdscha_b200 import DynamicalLanczos as DL
    A, B = systems
    steps = 12
    ref = [_chains(A, [1, 2, 3]), _chains(B, [4, 5])]
    for chains in ref:
        DL.run_FT_batched(chains, steps, precision=precision)
    for use_graph in (False, True):
        got = [_chains(A, [1, 2, 3]), _chains(B, [4, 5])]
        DL.run_FT_multi(got, steps, precision=precision, use_graph=use_graph)
        for cg, cr in zip(got, ref):
            for (a, b, c), (ar, br, cr_) in zip(_coeffs(cg), _coeffs(cr)):
                assert len(a) == len(ar) == steps
                tol = 1e-10 if precision == "fp64" else 1e-8
                assert np.abs(a - ar).max() <= tol * np.abs(ar).max()
                assert np.abs(b - br).max() <= tol * np.abs(br).max()
                assert np.abs(c - cr_).max() <= tol * np.abs(cr_).max()
        # the final vectors are the batched run's last q
        for cg, cr in zip(got, ref):
            for Lg, Lr in zip(cg, cr):
                assert np.abs(Lg.psi - Lr.psi).max() <= 1e-8 * np.abs(Lr.psi).max()


def test_graph_replay_is_bitwise_the_eager_run(systems):
    from tdscha_b200 import DynamicalLanczos as DL
    A, B = systems
    runs = []
    for use_graph in (False, True):
        got = [_chains(A, [7, 8]), _chains(B, [9])]
        DL.run_FT_multi(got, 9, precision="bf16x3", use_graph=use_graph)
        runs.append([x for chains in got for t in _coeffs(chains) for x in t])
    for x, y in zip(*runs):
        assert np.array_equal(x, y)


def test_continuation_equals_one_run(systems):
    """Two runs of 5 + 7 steps give the 12-step run (state carried in the Lanczos objects)."""
    from tdscha_b200 import DynamicalLanczos as DL
    A, _ = systems
    one = _chains(A, [11, 12])
    DL.run_FT_multi([one], 12, precision="fp64")
    two = _chains(A, [11, 12])
    DL.run_FT_multi([two], 5, precision="fp64")
    DL.run_FT_multi([two], 7, precision="fp64")
    for (a, b, c), (a2, b2, c2) in zip(_coeffs(one), _coeffs(two)):
        assert np.abs(a - a2).max() <= 1e-10 * np.abs(a).max()
        assert np.abs(c - c2).max() <= 1e-10 * np.abs(c).max()


def test_breakdown_ends_only_that_chain(systems):
    """Harmonic operator (ignore_v3): a single-mode start is an eigenvector, so that chain breaks
    down at its first step (b = 0) while the random chains of the same batch go on, as in
    run_FT_batched."""
    from tdscha_b200 import DynamicalLanczos as DL
    A, _ = systems
    A.ignore_v3 = True
    try:
        def make():
            single = A.new_chain()
            single.prepare_mode(4)
            return [single] + _chains(A, [21, 22])
        got, ref = make(), make()
        DL.run_FT_multi([got], 8, precision="fp64")
        DL.run_FT_batched(ref, 8)
    finally:
        A.ignore_v3 = False
    assert len(got[0].a_coeffs) == len(ref[0].a_coeffs) == 1 and len(got[0].b_coeffs) == 0
    assert abs(got[0].a_coeffs[0] - ref[0].a_coeffs[0]) <= 1e-12 * abs(ref[0].a_coeffs[0])
    for Lg, Lr in zip(got[1:], ref[1:]):
        assert len(Lg.a_coeffs) == len(Lr.a_coeffs)
        assert np.allclose(Lg.a_coeffs, Lr.a_coeffs, rtol=1e-10, atol=0)
