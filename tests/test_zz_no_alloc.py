"""The Lanczos step entry point that allocates nothing (tdscha_lanczos_step_device_noalloc).

Some host programs cannot call cudaMalloc while they run the recurrence -- they hand out all device
memory from their own fixed arena, or must not trigger the implicit device synchronisation of
cudaMalloc/cudaFree.  This entry point keeps the step's reduction partials in a fixed array inside
the library instead.  Checked here through the C ABI against the allocating entry point on the same
inputs, on two calls in a row (the array keeps the previous call's contents).  Collected last so that
a run stopping at the first failure has already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(torch, nc, length, step, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    mk = lambda: torch.randn(nc, length, generator=g, dtype=torch.float64).cuda()   # noqa: E731
    Lq, pL, q, p, qp, pp = mk(), mk(), mk(), mk(), mk(), mk()
    sc = torch.tensor([[0.7, 0.9, 1.3, 1.1, 0.8, float(step)]] * nc, dtype=torch.float64).cuda()
    return Lq, pL, q, p, qp, pp, sc


def _run(torch, fn, args, mask=None):
    Lq, pL, q, p, qp, pp, sc = args
    qn, pn = torch.empty_like(q), torch.empty_like(p)
    sc_out = torch.empty((q.shape[0], 4), dtype=torch.float64, device="cuda")
    fn(Lq, pL, q, p, qp, pp, sc, mask, qn, pn, sc_out)
    torch.cuda.synchronize()
    return qn.cpu().numpy(), pn.cpu().numpy(), sc_out.cpu().numpy()


def test_noalloc_step_matches_allocating_step(cuda):
    torch = cuda
    from tdscha_b200 import _native
    for call, (nc, length, step) in enumerate([(5, 70001, 3), (32, 2115, 0)]):
        args = _inputs(torch, nc, length, step, seed=100 + call)
        ref = _run(torch, _native.lanczos_step, args)
        got = _run(torch, _native.lanczos_step_noalloc, args)
        for r, g in zip(ref, got):
            assert np.all(np.isfinite(g))
            assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()


def test_noalloc_step_with_mask_matches_allocating_step(cuda):
    """The weighted scalar products of the symmetric Wigner Lanczos (mask_dot_wigner) on both paths."""
    torch = cuda
    from tdscha_b200 import _native
    n = 45
    length = n + n * (n + 1)
    mask = np.ones(length)
    r, c = np.triu_indices(n)
    m = n * (n + 1) // 2
    mask[n:n + m][r < c] = 2
    mask[n + m:][r < c] = 2
    mask = torch.as_tensor(mask, device="cuda")
    args = _inputs(torch, 7, length, 2, seed=11)
    ref = _run(torch, _native.lanczos_step, args, mask)
    got = _run(torch, _native.lanczos_step_noalloc, args, mask)
    for rr, g in zip(ref, got):
        assert np.abs(g - rr).max() <= 1e-12 * np.abs(rr).max()


def test_noalloc_step_allocates_no_device_memory(cuda):
    """After one warm-up call (which may look up the array's address), further calls leave the
    device's free memory unchanged: nothing is allocated behind the caller's back."""
    torch = cuda
    from tdscha_b200 import _native
    args = _inputs(torch, 8, 100003, 4, seed=21)
    Lq, pL, q, p, qp, pp, sc = args
    qn, pn = torch.empty_like(q), torch.empty_like(p)
    sc_out = torch.empty((q.shape[0], 4), dtype=torch.float64, device="cuda")
    _native.lanczos_step_noalloc(Lq, pL, q, p, qp, pp, sc, None, qn, pn, sc_out)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        _native.lanczos_step_noalloc(Lq, pL, q, p, qp, pp, sc, None, qn, pn, sc_out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_step_rejects_too_many_chains(cuda):
    torch = cuda
    from tdscha_b200 import _native
    args = _inputs(torch, 33, 128, 1, seed=7)
    with pytest.raises(_native.TdschaError, match="at most 32"):
        _run(torch, _native.lanczos_step_noalloc, args)
