"""Float64 torch restatement of the symmetrised perturbed ensemble averages, differentiable.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; tests/ use it as the
float64 autograd reference for the gradients of the averages with respect to the ensemble's forces
Y and weights rho (the reference has no derivatives, so these gradients are pinned by this
restatement and by finite differences).

It follows, vectorised over configurations, the same formulas as oracle/tdscha_oracle.c, i.e. the
reference's
  CModules/LanczosFunctions.c:2082-2254  get_f_average_from_Y_pert_sym_fast
  CModules/LanczosFunctions.c:2257-2438  get_d2v_dR2_from_R_pert_sym_fast
  CModules/LanczosFunctions.c:2615-2754  get_d2v_dR2_from_Y_pert_sym_fast
with the symmetry image u = S_j x_i, f = S_j y_i of LanczosFunctions.c:2158-2170:
  W1 = -u^T Y1 u / 2,  W2 = -(psi o f)^T (Y1 + Y1^T) u / 4
  f_av += rho (W1 f / 3 + 2 W2 (ups o u) / 3)
  D_av -= cf ((ups o u) f^T + f (ups o u)^T) + cu (ups o u)(ups o u)^T,
      cf = rho (R1 . (ups o u)) / 3 [- rho u^T Y1 u / 8],  cu = rho (R1 . f) / 3 [- rho W2' / 8]
(bracketed terms with apply_d4), both divided by N_eff N_sym, N_eff = sum(rho).  Small systems only.
"""
from __future__ import annotations

import numpy as np
import torch

RY_TO_K = 157887.32400374097


def thermal(w, T):
    w = torch.as_tensor(w, dtype=torch.float64)
    nb = 1.0 / torch.expm1(w * RY_TO_K / T) if T > 0 else torch.zeros_like(w)
    ups = 2 * w / (1 + 2 * nb)
    return ups, 1.0 / ups


def full_symmetries(symmetries, deg_space, n):
    """(N_sym, n, n) block-diagonal S_j from the per-block tables."""
    N_sym = np.asarray(symmetries[0]).shape[0]
    S = np.zeros((N_sym, n, n))
    for tab, blk in zip(symmetries, deg_space):
        blk = np.asarray(blk)
        S[:, blk[:, None], blk[None, :]] = np.asarray(tab)
    return torch.as_tensor(S)


def perturb_average(X, Y, w, rho, R1, Y1, T, apply_d4, S):
    """(f_av (n), D_av (n, n)); X, Y (N, n), rho (N), R1 (n), Y1 (n, n), S (N_sym, n, n) tensors."""
    ups, psi = thermal(w, T)
    n = X.shape[1]
    N_sym = S.shape[0]
    f_acc = torch.zeros(n, dtype=torch.float64)
    d_acc = torch.zeros((n, n), dtype=torch.float64)
    for j in range(N_sym):
        u = X @ S[j].T
        f = Y @ S[j].T
        ut = ups * u
        g = psi * f
        t = u @ Y1.T
        s = u @ Y1
        uYu = (u * t).sum(1)
        gYu = (g * (t + s)).sum(1)
        W1, W2 = -0.5 * uYu, -0.25 * gYu
        f_acc = f_acc + ((rho * W1 / 3.0)[:, None] * f + (rho * W2 * 2.0 / 3.0)[:, None] * ut).sum(0)
        cf = rho * (ut @ R1) / 3.0
        cu = rho * (f @ R1) / 3.0
        if apply_d4:
            cf = cf - rho / 8.0 * uYu
            cu = cu - rho / 8.0 * gYu
        d_acc = d_acc - (ut * cf[:, None]).T @ f - (f * cf[:, None]).T @ ut - (ut * cu[:, None]).T @ ut
    norm = rho.sum() * N_sym
    return f_acc / norm, d_acc / norm
