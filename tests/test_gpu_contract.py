"""tcgen05 contraction kernel (through the C ABI tdscha_tc_contract) against an FP64 torch product
of the same rounded operands."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def tf32_round(a):
    """Round float32 values to tf32 (nearest, ties away from zero) -- the cvt.rna.tf32.f32 rule."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    u = ((u + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).astype(np.uint32)
    return u.view(np.float32)


def split(torch, A, mode):
    """hi / lo operands (torch CUDA tensors) and their FP64 values."""
    if mode.startswith("bf16"):
        hi = A.to(torch.bfloat16)
        lo = (A - hi.double()).to(torch.bfloat16)
        return hi, lo, hi.double(), lo.double()
    a = A.cpu().numpy()
    hi = tf32_round(a.astype(np.float32))
    lo = tf32_round((a - hi.astype(np.float64)).astype(np.float32))
    th, tl = torch.as_tensor(hi, device="cuda"), torch.as_tensor(lo, device="cuda")
    return th, tl, th.double(), tl.double()


SHAPES = [(128, 256, 64), (256, 512, 256), (200, 300, 192), (384, 72, 128), (128, 256, 2048), (333, 129, 4096)]


@pytest.mark.parametrize("tile_n", ["256", "128"])
@pytest.mark.parametrize("mode", ["bf16", "bf16x3", "tf32", "tf32x3"])
@pytest.mark.parametrize("shape", SHAPES)
def test_tc_contract_matches_fp64(cuda, mode, shape, tile_n, monkeypatch):
    """Both tile configurations the autotuner chooses from (128 x 256 and 128 x 128 output tiles),
    forced through TDSCHA_TILE_N."""
    torch = cuda
    monkeypatch.setenv("TDSCHA_TILE_N", tile_n)
    from tdscha_b200 import _native
    M, N, K = shape
    if mode.startswith("tf32") and K % 32:
        pytest.skip("K multiple of 32 for tf32")
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).cuda()
    B = torch.randn(N, K, generator=g, dtype=torch.float64).cuda()
    ah, al, ahd, ald = split(torch, A, mode)
    bh, bl, bhd, bld = split(torch, B, mode)
    ldd = (N + 3) // 4 * 4
    D = torch.full((M, ldd), float("nan"), dtype=torch.float32, device="cuda")
    three = mode.endswith("x3")
    _native.tc_contract(mode, ah, al if three else None, bh, bl if three else None, D)
    torch.cuda.synchronize()
    ref = ahd @ bhd.T
    if three:
        ref = ref + ahd @ bld.T + ald @ bhd.T
    got = D[:, :N].double()
    scale = (ahd.abs() @ bhd.abs().T)
    err = ((got - ref).abs() / scale).max().item()
    assert torch.isfinite(got).all()
    # fp32 tensor-core accumulation of K exact products, relative to sum |a||b|; kind::tf32 accumulates
    # the three hi/lo products with a few units of 2^-22 per instruction group (measured ~5e-7 at K = 64)
    bound = (4e-7 if mode.startswith("bf16") else 1.2e-6) * np.sqrt(K / 64) + 2e-7
    assert err < bound, err
