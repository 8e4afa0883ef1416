"""Gradients of the Lanczos Green function with respect to the ensemble: dG(w)/dY, dG(w)/drho and,
through the linear force dependence, dG(w)/d(k3, k4).

``apply_full_L`` is a torch.autograd.Function around the device apply (FP64):
  * the cotangent of its input vector is the transposed apply (L_T is the exact transpose of L);
  * the cotangent of the ensemble's forces Y and weights rho is the vector-Jacobian product of the
    averages (tdscha_perturb_average_vjp_device) at the prologue's (R1, Upsilon^(1)) of the input
    and the transposed epilogue of the output cotangent.
``green_function`` runs the bi-conjugate Lanczos recurrence (Modules/DynamicalLanczos.py:6059-6153,
n_rep_orth = 0) and the continued fraction (:4951-5047, no terminator) as torch operations on the
device, so torch autograd differentiates through them; every ``checkpoint_every`` steps the chain
is checkpointed (the forward of a segment is recomputed in the backward pass instead of kept).

Scope: the standard representation (use_wigner = False) without the terminator; the ensemble
arrays passed as Y and rho must be the ones the Lanczos object's device ensemble was built from
(they carry the gradient, the device copy does the arithmetic).
"""
from __future__ import annotations

import numpy as np

from . import _native
from .DynamicalLanczos import __EPSILON__, __RyToK__


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _native.TdschaError("gradients need a CUDA device (no CPU fallback)")
    return torch


class _Ctl:
    """What the autograd function needs besides tensors."""

    def __init__(self, lanc, precision="fp64", vjp_precision=None):
        torch = _torch()
        vjp_precision = precision if vjp_precision is None else vjp_precision
        for p in (precision, vjp_precision):
            if p not in _native.PREC:
                raise ValueError(f"precision must be one of {list(_native.PREC)}")
        self.precision = precision
        self.vjp_precision = vjp_precision
        if lanc.use_wigner:
            raise NotImplementedError("gradients are available in the standard representation (use_wigner = False)")
        lanc._check_init()
        self.lanc = lanc
        self.ens = lanc.device_ensemble
        self.opts = lanc._opts()
        n = lanc.n_modes
        self.n = n
        self.P = n * (n + 1) // 2
        w = np.asarray(lanc.w, dtype=np.float64)
        T = float(lanc.T)
        nb = 1.0 / np.expm1(w * __RyToK__ / T) if T > __EPSILON__ else np.zeros_like(w)   # as the epilogue
        Yw = 2 * w / (2 * nb + 1)
        RA = 2 * w * nb * (nb + 1) / (2 * nb + 1)
        r, c = np.triu_indices(n)
        off = r != c
        dev = "cuda"
        self.r, self.c = torch.as_tensor(r, device=dev), torch.as_tensor(c, device=dev)
        # coefficient of D_av[mu, nu] in the Y / A components of the output (epilogue), per packed pair
        self.cY = torch.as_tensor(Yw[r] + Yw[c], device=dev)
        self.cA = torch.as_tensor(RA[r] + RA[c], device=dev)
        self.cYt = torch.as_tensor(0.5 / (Yw[r] * Yw[c]) * np.where(off, 2.0, 1.0), device=dev)
        self.half = torch.as_tensor(np.where(off, 0.5, 1.0), device=dev)   # symmetric Frobenius convention
        self.sign = -1.0 if lanc.reverse_L else 1.0
        self.apply_d4 = 0 if lanc.ignore_v4 else 1
        self.anharmonic = not lanc.ignore_v3

    def epilogue_transpose(self, gout, transpose):
        """(fbar, Dbar) with <gout, epilogue(f, D)> = <fbar, f> + <Dbar, D>_F for symmetric D."""
        torch = _torch()
        n, P = self.n, self.P
        kb = gout.shape[0]
        fbar = -self.sign * gout[:, :n]
        gY, gA = gout[:, n:n + P], gout[:, n + P:]
        tr = torch.as_tensor(transpose, device=gout.device, dtype=torch.bool)[:, None]
        kappa = torch.where(tr, -gY * self.cYt, -(gY * self.cY + gA * self.cA)) * self.sign
        Dbar = torch.zeros((kb, n, n), dtype=torch.float64, device=gout.device)
        vals = kappa * self.half
        Dbar[:, self.r, self.c] = vals
        Dbar[:, self.c, self.r] = vals
        return fbar.contiguous(), Dbar.contiguous()


def _make_function():
    torch = _torch()

    class ApplyFullL(torch.autograd.Function):
        @staticmethod
        def forward(ctx, psi, Y, rho, ctl, transpose):
            out = torch.empty_like(psi)
            ctl.ens.apply_full_L(psi.contiguous(), out, transpose, ctl.opts, ctl.precision)
            ctx.save_for_backward(psi)
            ctx.ctl, ctx.transpose = ctl, list(transpose)
            return out

        @staticmethod
        def backward(ctx, gout):
            (psi,) = ctx.saved_tensors
            ctl, tr = ctx.ctl, ctx.transpose
            gout = gout.contiguous()
            psi_bar = None
            if ctx.needs_input_grad[0]:
                psi_bar = torch.empty_like(gout)
                ctl.ens.apply_full_L(gout, psi_bar, [1 - t for t in tr], ctl.opts, ctl.precision)
            Y_bar = rho_bar = None
            if (ctx.needs_input_grad[1] or ctx.needs_input_grad[2]) and ctl.anharmonic:
                kb, n = psi.shape[0], ctl.n
                R1 = torch.empty((kb, n), dtype=torch.float64, device=psi.device)
                Y1 = torch.empty((kb, n, n), dtype=torch.float64, device=psi.device)
                ctl.ens.apply_prologue(psi.contiguous(), R1, Y1, tr, ctl.opts)
                fbar, Dbar = ctl.epilogue_transpose(gout, tr)
                Y_bar = torch.empty((ctl.ens.N, n), dtype=torch.float64, device=psi.device)
                rho_bar = torch.empty(ctl.ens.N, dtype=torch.float64, device=psi.device)
                ctl.ens.perturb_average_vjp(R1, Y1, fbar, Dbar, Y_bar, rho_bar, apply_d4=ctl.apply_d4,
                                            precision=ctl.vjp_precision)
            elif ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
                Y_bar = torch.zeros((ctl.ens.N, ctl.n), dtype=torch.float64, device=psi.device)
                rho_bar = torch.zeros(ctl.ens.N, dtype=torch.float64, device=psi.device)
            return psi_bar, Y_bar, rho_bar, None, None

    return ApplyFullL


_FN = None


def apply_full_L(psi, Y, rho, lanc, transpose, ctl=None):
    """Differentiable batched apply: psi (nb, len) CUDA float64, Y (N, n), rho (N) the ensemble's
    arrays as CUDA float64 tensors (requires_grad as needed), transpose a list of nb flags."""
    global _FN
    if _FN is None:
        _FN = _make_function()
    return _FN.apply(psi, Y, rho, ctl or _Ctl(lanc), list(transpose))


def green_function(lanc, omega, smearing, n_steps, Y, rho, psi0=None, checkpoint_every=10, precision="fp64",
                   vjp_precision=None):
    """G(omega) (complex, CUDA) of the bi-conjugate chain of n_steps steps from psi0 (default
    lanc.psi), differentiable with respect to Y and rho.  `precision` is the arithmetic of the
    ensemble contractions inside the forward and transposed applies, `vjp_precision` (default the
    same) that of the contractions of the averages' vector-Jacobian product; the recurrence, the
    continued fraction and the rest of the VJP are FP64."""
    torch = _torch()
    from torch.utils.checkpoint import checkpoint
    ctl = _Ctl(lanc, precision, vjp_precision)
    dev = "cuda"
    v = torch.as_tensor(np.asarray(lanc.psi if psi0 is None else psi0, dtype=np.float64), device=dev)
    q = v / torch.sqrt((v * v).sum())
    p = q.clone()
    zero = torch.zeros_like(q)
    one = torch.ones((), dtype=torch.float64, device=dev)
    # running state: q, p, q_prev, p_prev, s_norm[-1], s_norm[-2], c[-1], c[-2], b[-1]
    state = (q, p, zero, zero, one, one, one, one, one * 0)
    a_list, b_list, c_list = [], [], []

    def segment(k0, k1, *st):
        q, p, qp, pp, sn1, sn2, c1, c2, b1 = st
        out_a, out_b, out_c = [], [], []
        for k in range(k0, k1):
            L = apply_full_L(torch.stack([q, p]), Y, rho, lanc, [0, 1], ctl)
            Lq, pL = L[0], L[1]
            c_old = c1 if k > 0 else one
            p_norm = sn1 / c_old
            a = (p * Lq).sum() * p_norm
            rk = Lq - a * q
            sk = pL - a * p
            if k > 0:
                rk = rk - c1 * qp
                old_p_norm = sn2 if k < 2 else sn2 / c2
                sk = sk - b1 * pp * (old_p_norm / p_norm)
            s_raw = torch.sqrt((sk * sk).sum())
            sk_t = sk / s_raw
            s_new = s_raw * p_norm
            b = torch.sqrt((rk * rk).sum())
            c = (sk_t * (rk / b)).sum() * s_new
            out_a.append(a)
            out_b.append(b)
            out_c.append(c)
            qp, pp = q, p
            q, p = rk / b, sk_t
            sn2, sn1 = sn1, s_new
            c2, c1 = c1, c
            b1 = b
        return (q, p, qp, pp, sn1, sn2, c1, c2, b1, torch.stack(out_a), torch.stack(out_b), torch.stack(out_c))

    for k0 in range(0, n_steps, checkpoint_every):
        k1 = min(n_steps, k0 + checkpoint_every)
        res = checkpoint(segment, k0, k1, *state, use_reentrant=False)
        state = res[:9]
        a_list.append(res[9])
        b_list.append(res[10])
        c_list.append(res[11])
    a = torch.cat(a_list)
    b = torch.cat(b_list)[:-1]
    c = torch.cat(c_list)[:-1]
    if torch.any(b.abs() < __EPSILON__) or torch.any(c.abs() < __EPSILON__):
        raise ValueError("the chain broke down before n_steps; reduce n_steps")
    return continued_fraction(a, b, c, omega, smearing, lanc)


def continued_fraction(a, b, c, omega, smearing, lanc):
    """The continued fraction without terminator, as get_green_function_continued_fraction."""
    torch = _torch()
    sign = -1.0 if lanc.reverse_L else 1.0
    shift = float(lanc.shift_value)
    w = torch.as_tensor(np.asarray(omega, dtype=np.float64), device=a.device)
    eta = float(smearing)
    A = a * sign - sign * shift
    B = b * sign
    C = c * sign
    g = 1.0 / torch.complex(A[-1] - w * w, 2 * w * eta)
    for i in range(len(a) - 2, -1, -1):
        g = 1.0 / (torch.complex(A[i] - w * w, 2 * w * eta) - B[i] * C[i] * g)
    return g * float(lanc.perturbation_modulus)


def force_gradient_to_k(Y_bar, Y3, Y4):
    """dG/dk3, dG/dk4 from dG/dY for forces linear in (k3, k4): Y = k3 Y3 + k4 Y4."""
    return float((Y_bar * Y3).sum()), float((Y_bar * Y4).sum())
