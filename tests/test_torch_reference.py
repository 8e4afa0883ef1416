"""The float64 torch restatement of the averages (oracle/averages_torch.py, the autograd reference
for the gradients) against the C restatement pinned to the reference kernel.  No GPU."""
import numpy as np
import torch

from oracle import averages_torch as AT
from oracle import lanczos_oracle as LO


def test_torch_averages_match_c_oracle(rocksalt_l2):
    d = rocksalt_l2
    n = d["X"].shape[1]
    rng = np.random.default_rng(5)
    R1 = rng.standard_normal(n) * 1e-2
    A = rng.standard_normal((n, n)) * 1e-2
    Y1 = A + A.T
    for d4 in (0, 1):
        f_ref, D_ref = LO.perturb_average_sym(d["X"], d["Y"], d["w"], d["rho"], R1, Y1, d["T"], d4, d["syms"], d["n_deg"],
                                              d["blocks"], d["blocks_ids"], backend="port")
        S = AT.full_symmetries(d["syms"], d["blocks"], n)
        t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))   # noqa: E731
        f, D = AT.perturb_average(t(d["X"]), t(d["Y"]), d["w"], t(d["rho"]), t(R1), t(Y1), d["T"], d4, S)
        assert np.abs(f.numpy() - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
        assert np.abs(D.numpy() - D_ref).max() <= 1e-12 * np.abs(D_ref).max()
