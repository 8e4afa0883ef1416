"""Failure detection of the tensor-core contraction without a GPU fault.

Every pipeline wait of the tcgen05 kernel is bounded (tdscha_set_wait_budget).  A one-shot test hook
(tdscha_debug_stall_next_contraction) makes the next launch's producers issue no copy, so the MMA
warps' first wait on a full stage can only end by running out -- a flag that nothing sets.  The call
must come back with TDSCHA_ETIMEOUT (the kernel drained, freed its tensor memory and returned), and the
next contraction on the same context must give the correct result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _operands(torch, M, N, K, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).cuda()
    B = torch.randn(N, K, generator=g, dtype=torch.float64).cuda()
    ah = A.to(torch.bfloat16)
    al = (A - ah.double()).to(torch.bfloat16)
    bh = B.to(torch.bfloat16)
    bl = (B - bh.double()).to(torch.bfloat16)
    return ah, al, bh, bl


def test_stalled_contraction_times_out_and_the_next_one_is_correct(cuda):
    torch = cuda
    from tdscha_b200 import _native
    M, N, K = 1024, 768, 4096
    ah, al, bh, bl = _operands(torch, M, N, K, 3)
    D0 = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    _native.tc_contract("bf16x3", ah, al, bh, bl, D0)
    torch.cuda.synchronize()
    try:
        _native.set_wait_budget(0.02)
        _native.debug_stall_next_contraction()
        D1 = torch.zeros_like(D0)
        with pytest.raises(_native.TdschaError, match="ETIMEOUT"):
            _native.tc_contract("bf16x3", ah, al, bh, bl, D1)
    finally:
        _native.set_wait_budget(4.0)
    D2 = torch.zeros_like(D0)
    _native.tc_contract("bf16x3", ah, al, bh, bl, D2)
    torch.cuda.synchronize()
    assert torch.equal(D2, D0)
    ref = (ah.double() @ bh.double().T + ah.double() @ bl.double().T + al.double() @ bh.double().T)
    assert float((D2.double() - ref).abs().max() / ref.abs().max()) < 1e-5


def test_stalled_averages_report_timeout_and_recover(cuda, rocksalt_l2):
    """The same through a whole averages call: the stalled [a|b] launch flags the ensemble's error
    word, the call returns TDSCHA_ETIMEOUT, and the next call matches the reference golden output."""
    from tdscha_b200 import _native
    d = rocksalt_l2
    ens = _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    f0, dv0 = ens.perturb_average(d["case0_R1"], d["case0_Y1"], 1, "bf16x3")
    try:
        _native.set_wait_budget(0.02)
        _native.debug_stall_next_contraction()
        with pytest.raises(_native.TdschaError, match="ETIMEOUT"):
            ens.perturb_average(d["case0_R1"], d["case0_Y1"], 1, "bf16x3")
    finally:
        _native.set_wait_budget(4.0)
    f, dv = ens.perturb_average(d["case0_R1"], d["case0_Y1"], 1, "bf16x3")
    assert np.array_equal(f, f0) and np.array_equal(dv, dv0)
    gd = d["case0_d2v"]
    assert np.abs(dv - gd).max() / np.abs(gd).max() < 2e-4
    ens.close()


def test_wait_budget_rejects_out_of_range(cuda):
    from tdscha_b200 import _native
    with pytest.raises(_native.TdschaError, match="EINVAL"):
        _native.set_wait_budget(0.0)
    with pytest.raises(_native.TdschaError, match="EINVAL"):
        _native.set_wait_budget(1e3)


def test_deferred_error_check_reports_the_expiry_later(cuda, rocksalt_l2):
    """With the per-call check off (tdscha_set_error_check(0)) the stalled averages call returns at
    once; tdscha_check_errors reports the expiry afterwards, clears it, and later calls are exact."""
    from tdscha_b200 import _native
    d = rocksalt_l2
    ens = _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], d["T"], d["syms"], d["blocks"], d["blocks_ids"])
    f0, dv0 = ens.perturb_average(d["case0_R1"], d["case0_Y1"], 1, "bf16x3")
    try:
        _native.set_error_check(False)
        _native.set_wait_budget(0.02)
        _native.debug_stall_next_contraction()
        ens.perturb_average(d["case0_R1"], d["case0_Y1"], 1, "bf16x3")      # no error at return
        with pytest.raises(_native.TdschaError, match="ETIMEOUT"):
            _native.check_errors(ens.handle)
        _native.check_errors(ens.handle)                                      # cleared
        _native.set_wait_budget(4.0)
        f, dv = ens.perturb_average(d["case0_R1"], d["case0_Y1"], 1, "bf16x3")
        _native.check_errors(ens.handle)
    finally:
        _native.set_wait_budget(4.0)
        _native.set_error_check(True)
    assert np.array_equal(f, f0) and np.array_equal(dv, dv0)
    ens.close()
