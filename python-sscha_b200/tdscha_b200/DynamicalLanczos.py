"""
B200 compute mode for the TD-SCHA Lanczos linear response.

Host-side mirror of ``tdscha.DynamicalLanczos.Lanczos`` (Modules/DynamicalLanczos.py:182) for the
hot path: same attribute names, method names, argument meanings and checkpoint (npz) schema, with
one more compute mode ``MODE_B200 = 4`` next to the reference's 0-3 (:166-169).  Every operator
application, Lanczos step and continued fraction runs on the GPU through the C ABI
(include/tdscha_b200.h); there is no CPU fallback.

Differences from the reference that a user sees:
  * the ensemble argument is any object exposing the arrays the reference extracts from an
    ``sscha.Ensemble`` (X, Y, rho, w, pols, m, T, ...), e.g. ``rocksalt.SyntheticEnsemble``;
    cellconstructor/sscha are not needed;
  * ``precision`` selects the arithmetic of the two ensemble contractions
    ("fp64", "tf32", "bf16x3", "tf32x3", "bf16"); the recurrence is always FP64;
  * errors raise exceptions where the reference's C binding calls exit().
"""
from __future__ import annotations

import difflib
import json
import os
import sys
import time
import warnings

import numpy as np

from . import _native

MODE_SLOW_SERIAL = 0
MODE_FAST_SERIAL = 1
MODE_FAST_MPI = 2
MODE_FAST_JULIA = 3
MODE_B200 = 4

TYPE_DP = np.double
__EPSILON__ = 1e-12          # DynamicalLanczos.py:121
__RyToK__ = 157887.32400374097


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _native.TdschaError("MODE_B200 needs a CUDA device (no CPU fallback)")
    return torch


class Lanczos(object):
    def __init__(self, ensemble=None, mode=None, unwrap_symmetries=False, select_modes=None, use_wigner=False,
                 lo_to_split="random", precision="fp64"):
        self.mode = MODE_B200
        if mode is not None and mode != MODE_B200:
            raise ValueError(f"this package implements only MODE_B200 = {MODE_B200} (got {mode})")
        self.verbose = True
        self.T = 0
        self.nat = 0
        self.m = []
        self.w = []
        self.pols = []
        self.n_modes = 0
        self.ignore_harmonic = False
        self.ignore_v3 = False
        self.ignore_v4 = False
        self.N = 0
        self.rho = []
        self.N_eff = 0
        self.X = []
        self.Y = []
        self.psi = []
        self.eigvals = None
        self.eigvects = None
        self.a_coeffs = []
        self.b_coeffs = []
        self.c_coeffs = []
        self.krilov_basis = []
        self.basis_P = []
        self.basis_Q = []
        self.s_norm = []
        self.arnoldi_matrix = []
        self.reverse_L = False
        self.shift_value = 0
        self.symmetrize = False
        self.symmetries = None
        self.degenerate_space = None
        self.N_degeneracy = None
        self.initialized = False
        self.perturbation_modulus = 1
        self.dyn = None
        self.uci_structure = None
        self.super_structure = None
        self.qe_sym = None
        self.L_linop = None
        self.M_linop = None
        self.unwrapped = False
        self.sym_julia = None
        self.deg_julia = None
        self.n_syms = 1
        self.u_tilde = None
        self.f_tilde = None
        self.sym_block_id = None
        self.use_wigner = use_wigner
        self.ignore_small_w = False
        self.precision = precision
        self.effective_charges = None
        self.raman_tensor = None
        self.supercell = (1, 1, 1)
        self.nat_uc = 0
        self.device_ensemble = None
        self.__total_attributes__ = [item for item in self.__dict__.keys()]
        self.fixed_attributes = True

        if ensemble is None:
            return
        if precision not in _native.PREC:
            raise ValueError(f"precision must be one of {list(_native.PREC)}")
        self.T = float(ensemble.T)
        self.nat = int(ensemble.nat)
        self.m = np.asarray(ensemble.m, dtype=TYPE_DP)
        self.w = np.asarray(ensemble.w, dtype=TYPE_DP)
        self.pols = np.asarray(ensemble.pols, dtype=TYPE_DP)
        if select_modes is not None:
            raise NotImplementedError("select_modes: pass the already reduced mode set in the ensemble")
        self.n_modes = len(self.w)
        self.N = int(ensemble.N)
        self.rho = np.asarray(ensemble.rho, dtype=TYPE_DP).copy()
        self.N_eff = float(np.sum(self.rho))
        self.X = np.ascontiguousarray(ensemble.X, dtype=TYPE_DP)
        self.Y = np.ascontiguousarray(ensemble.Y, dtype=TYPE_DP)
        self.effective_charges = getattr(ensemble, "effective_charges", None)
        self.raman_tensor = getattr(ensemble, "raman_tensor", None)
        self.supercell = tuple(getattr(ensemble, "supercell", (1, 1, 1)))
        self.nat_uc = int(getattr(ensemble, "nat_uc", self.nat))
        self._ens_symmetries = (getattr(ensemble, "symmetries", None), getattr(ensemble, "deg_space", None),
                                getattr(ensemble, "blocks_ids", None))
        self.psi = np.zeros(self.n_modes + self.n_modes * (self.n_modes + 1), dtype=TYPE_DP)

    def __setattr__(self, name, value):
        if "fixed_attributes" in self.__dict__:
            if name in self.__total_attributes__ or name.startswith("_"):
                super(Lanczos, self).__setattr__(name, value)
            elif self.fixed_attributes:
                similar = str(difflib.get_close_matches(name, self.__total_attributes__))
                raise AttributeError(f"""
        Error, the attribute '{name}' is not a member of '{type(self).__name__}'.
        Suggested similar attributes: {similar} ?
        """)
        else:
            super(Lanczos, self).__setattr__(name, value)

    # ------------------------------------------------------------------------------------------
    def reset(self):
        n = self.n_modes
        self.psi = np.zeros(n + n * (n + 1), dtype=TYPE_DP)
        self.eigvals = None
        self.eigvects = None
        self.a_coeffs = []
        self.b_coeffs = []
        self.c_coeffs = []
        self.basis_P = []
        self.basis_Q = []
        self.s_norm = []
        self.krilov_basis = []
        self.arnoldi_matrix = []

    def new_chain(self):
        """Another chain on this initialised object's device ensemble: same ensemble, symmetries and
        flags, fresh Lanczos state (for run_FT_batched / run_FT_multi, whose chains share an ensemble)."""
        import copy
        self._check_init()
        L = copy.copy(self)
        L.reset()
        L.perturbation_modulus = 1
        return L

    def init(self, use_symmetries=True):
        self.prepare_symmetrization(no_sym=not use_symmetries)
        self.initialized = True
        self._make_linops()

    def prepare_symmetrization(self, no_sym=False, verbose=True, symmetries=None):
        """Mode-space symmetry blocks (DynamicalLanczos.py:686-782).  ``symmetries`` may be a tuple
        (per-block tables, per-block mode lists, blocks_ids); by default the ensemble's are used."""
        n = self.n_modes
        self.initialized = True
        if no_sym or self.unwrapped:
            self.symmetries = [np.ones((1, 1, 1), dtype=np.double)] * n
            self.N_degeneracy = np.ones(n, dtype=np.intc)
            self.degenerate_space = [np.array([i], dtype=np.intc) for i in range(n)]
            self.sym_block_id = np.arange(n).astype(np.intc)
        else:
            syms, degs, bids = symmetries if symmetries is not None else self._ens_symmetries
            if syms is None:
                raise ValueError("no symmetry tables available: pass symmetries=(tables, blocks, ids) or no_sym=True")
            self.symmetries = [np.asarray(s, dtype=np.double) for s in syms]
            self.degenerate_space = [np.array(d, dtype=np.intc) for d in degs]
            self.N_degeneracy = np.array([len(d) for d in degs], dtype=np.intc)
            self.sym_block_id = np.asarray(bids, dtype=np.intc)
        self.n_syms = self.symmetries[0].shape[0]
        self._upload()

    def _upload(self):
        if self.device_ensemble is not None:
            self.device_ensemble.close()
        self.device_ensemble = _native.DeviceEnsemble(self.X, self.Y, self.w, self.rho, self.T, self.symmetries,
                                                      self.degenerate_space, self.sym_block_id)

    def _opts(self, harmonic=True, anharmonic=True, post=True):
        return _native.ApplyOpts(int(self.use_wigner), int(self.ignore_harmonic or not harmonic),
                                 int(self.ignore_v3 or not anharmonic), int(self.ignore_v4),
                                 int(self.reverse_L) if post else 0, float(self.shift_value) if post else 0.0)

    def _check_init(self):
        if not self.initialized or self.device_ensemble is None:
            raise ValueError("Error, this class must be initialized before lunching the computation:\n Use the .init()")

    def _apply_host(self, psi, transpose, opts):
        torch = _torch()
        self._check_init()
        x = torch.as_tensor(np.asarray(psi, dtype=TYPE_DP), device="cuda").reshape(1, -1).contiguous()
        out = torch.empty_like(x)
        self.device_ensemble.apply_full_L(x, out, [int(transpose)], opts, self.precision)
        return out.reshape(-1).cpu().numpy()

    # ---- operator (DynamicalLanczos.py:2227-2385, 2891-3281, 3467-3570) ----------------------
    def apply_L1_FT(self, transpose=False):
        if self.ignore_harmonic:
            return np.zeros(np.shape(self.psi), dtype=TYPE_DP)
        return self._apply_host(self.psi, transpose, self._opts(anharmonic=False, post=False))

    def apply_anharmonic_FT(self, transpose=False, test_weights=True, use_old_version=False):
        if use_old_version:
            raise NotImplementedError("the pre-symmetrisation averages are not part of the B200 path")
        o = self._opts(harmonic=False, post=False)
        o.ignore_v3 = 0
        return self._apply_host(self.psi, transpose, o)

    def apply_full_L(self, target=None, force_t_0=False, force_FT=True, transpose=False, fast_lanczos=True):
        if force_t_0 and force_FT:
            raise ValueError("Error, only one between force_t_0 and force_FT can be True")
        if target is not None:
            self.psi = target
        self._check_init()
        if (force_t_0 or self.T < __EPSILON__) and not force_FT:
            raise NotImplementedError("the T = 0 operator (apply_L1) is not part of the B200 path")
        opts = self._opts(anharmonic=fast_lanczos)
        self.psi = self._apply_host(self.psi, transpose, opts)
        return self.psi

    # ---- perturbations (DynamicalLanczos.py:1963-2031, 1647-1689, 1003-1124) -----------------
    def prepare_perturbation(self, vector, masses_exp=1, add=False):
        if not add:
            self.reset()
            self.psi = np.zeros(self.psi.shape, dtype=TYPE_DP)
        m_on = np.sqrt(self.m) ** masses_exp
        new_v = np.einsum("a, a, ab->b", m_on, vector, self.pols)
        self.psi[:self.n_modes] += new_v
        self.perturbation_modulus = new_v.dot(new_v)

    def prepare_mode(self, index):
        self.reset()
        self.psi[:] = 0
        self.psi[index] = 1
        self.perturbation_modulus = 1

    def prepare_ir(self, effective_charges=None, pol_vec=np.array([1, 0, 0])):
        ec = self.effective_charges if effective_charges is None else effective_charges
        assert ec is not None, "Error, no effective charge found. Cannot initialize IR responce"
        ec = np.asarray(ec)
        assert len(ec.shape) == 3 and ec.shape[1] == ec.shape[2] == 3, f"Error, effective charges of the wrong shape: {ec.shape}"
        n_supercell = int(np.prod(self.supercell))
        if not self.ignore_small_w:
            assert ec.shape[0] * ec.shape[2] * n_supercell == self.n_modes + 3
        z_eff = np.einsum("abc, b", ec, pol_vec)
        self.prepare_perturbation(np.tile(z_eff.ravel(), n_supercell), masses_exp=-1)

    def prepare_raman(self, pol_vec_in=np.array([1, 0, 0]), pol_vec_out=np.array([1, 0, 0]), mixed=False,
                      pol_in_2=None, pol_out_2=None, unpolarized=None):
        """Raman perturbation.  As in the reference (DynamicalLanczos.py:1124), the final call
        re-prepares the perturbation from the last vector without ``add``."""
        from .rocksalt import raman_vector
        assert self.raman_tensor is not None, "Error, no Raman tensor found. Cannot initialize the Raman responce"
        rv = lambda a, b: raman_vector(self.raman_tensor, np.asarray(a, float), np.asarray(b, float))   # noqa: E731
        n_supercell = int(np.prod(self.supercell))
        raman_v = rv(pol_vec_in, pol_vec_out)
        if mixed:
            raman_v += rv(pol_in_2, pol_out_2)
        px, py, pz = np.eye(3)
        if unpolarized is None:
            new_raman_v = np.tile(rv(pol_vec_in, pol_vec_out).ravel(), n_supercell)
            self.prepare_perturbation(new_raman_v, masses_exp=-1)
        else:
            plan = {0: [((px, px), 1 / 3), ((py, py), 1 / 3), ((pz, pz), 1 / 3)],
                    1: [((px, px), 1 / np.sqrt(2)), ((py, py), -1 / np.sqrt(2))],
                    2: [((px, px), 1 / np.sqrt(2)), ((pz, pz), -1 / np.sqrt(2))],
                    3: [((py, py), 1 / np.sqrt(2)), ((pz, pz), -1 / np.sqrt(2))],
                    4: [((px, py), np.sqrt(3))], 5: [((py, pz), np.sqrt(3))], 6: [((px, pz), np.sqrt(3))]}
            if unpolarized not in plan:
                raise ValueError(f"Error, unpolarized must be between [0, ... ,6] got invalid {unpolarized}.")
            for t, ((a, b), s) in enumerate(plan[unpolarized]):
                new_raman_v = np.tile(rv(a, b).ravel(), n_supercell) * s
                self.prepare_perturbation(new_raman_v, masses_exp=-1, add=t > 0)
        self.prepare_perturbation(new_raman_v, masses_exp=-1)

    def prepare_random(self, seed=0, sector="R"):
        """Seeded random unit perturbation on R^(1) (sector "R") or on the whole vector ("all")."""
        rng = np.random.default_rng(seed)
        self.reset()
        v = np.zeros_like(self.psi)
        if sector == "R":
            v[:self.n_modes] = rng.standard_normal(self.n_modes)
        else:
            v[:] = rng.standard_normal(len(v))
        v /= np.linalg.norm(v)
        self.psi = v
        self.perturbation_modulus = 1

    def mask_dot_wigner(self, debug=False):
        n = self.n_modes
        mask = np.ones(n + n * (n + 1))
        r, c = np.triu_indices(n)
        m = n * (n + 1) // 2
        mask[n:n + m][r < c] = 2
        mask[n + m:][r < c] = 2
        return mask

    # ---- Lanczos (DynamicalLanczos.py:5843-6374) ---------------------------------------------
    def run_FT(self, n_iter, save_dir=None, save_each=5, verbose=True, n_rep_orth=0, n_ortho=10, flush_output=True,
               debug=False, prefix="LANCZOS", run_simm=False, optimized=False):
        run_FT_batched([self], n_iter, save_dir=save_dir, save_each=save_each, verbose=verbose, n_rep_orth=n_rep_orth,
                       run_simm=run_simm, prefix=[prefix], n_ortho=n_ortho)

    # ---- Green function (DynamicalLanczos.py:4951-5047) --------------------------------------
    def get_green_function_continued_fraction(self, w_array, use_terminator=True, last_average=1, smearing=0):
        torch = _torch()
        w_array = np.asarray(w_array, dtype=np.float64)
        a = torch.as_tensor(np.asarray(self.a_coeffs, dtype=np.float64), device="cuda")
        b = torch.as_tensor(np.asarray(self.b_coeffs, dtype=np.float64), device="cuda") if len(self.b_coeffs) else None
        c = torch.as_tensor(np.asarray(self.c_coeffs, dtype=np.float64), device="cuda") if len(self.c_coeffs) else None
        om = torch.as_tensor(w_array.ravel(), device="cuda")
        gf = torch.empty(2 * om.numel(), dtype=torch.float64, device="cuda")
        _native.continued_fraction(a, b, c, om, gf, use_terminator, last_average, smearing, self.use_wigner,
                                   self.reverse_L, self.shift_value, self.perturbation_modulus)
        g = gf.cpu().numpy()
        return (g[0::2] + 1j * g[1::2]).reshape(w_array.shape)

    # ---- consumers of apply_full_L (DynamicalLanczos.py:2391-2502, 3761-3972, 4571-4613, 5273-5307,
    #      5454-5789, 6381-6421) -------------------------------------------------------------------
    def _make_linops(self):
        """L_linop / M_linop as the reference builds them (DynamicalLanczos.py:468-479, 3749-3759):
        matvec = apply_full_L, rmatvec = its transpose, preconditioner = the harmonic inverse.  The
        matvec here leaves self.psi untouched."""
        import scipy.sparse.linalg as sla
        ln = len(self.psi)
        self.L_linop = sla.LinearOperator((ln, ln), matvec=lambda x: self._apply_host(x, False, self._opts()),
                                          rmatvec=lambda x: self._apply_host(x, True, self._opts()), dtype=TYPE_DP)
        self.M_linop = sla.LinearOperator((ln, ln), matvec=self.apply_L1_inverse_FT,
                                          rmatvec=lambda x: self.apply_L1_inverse_FT(x, transpose=True), dtype=TYPE_DP)

    def _l1_inverse_coefficients(self):
        """Pair-sector coefficients of the inverse free propagator (DynamicalLanczos.py:2391-2502).
        Pairs follow the packed order of psi: row-major upper triangle (mu <= nu), w_a = w[nu], w_b = w[mu]."""
        n = self.n_modes
        r, c = np.triu_indices(n)
        w_a, w_b = self.w[c], self.w[r]
        n_a = np.zeros(np.shape(w_a), dtype=TYPE_DP)
        n_b = np.zeros(np.shape(w_a), dtype=TYPE_DP)
        not_populated_a = 0.01 * w_a * __RyToK__ > self.T
        not_populated_b = 0.01 * w_a * __RyToK__ > self.T      # the reference tests w_a for both (:2434)
        if self.T > 0:
            with np.errstate(over="ignore"):
                n_a = 1 / (np.exp(w_a / np.double(self.T / __RyToK__)) - 1)
                n_b = 1 / (np.exp(w_b / np.double(self.T / __RyToK__)) - 1)
            n_a[not_populated_a] = 0
            n_b[not_populated_b] = 0
        X_ab = -w_a ** 2 - w_b ** 2 - (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
        Y_ab = -(8 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
        X1_ab = -(2 * n_a * n_b + n_a + n_b) * (2 * n_a * n_b + n_a + n_b + 1) * (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
        Y1_ab = -w_a ** 2 - w_b ** 2 + (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
        den = X_ab * Y1_ab - X1_ab * Y_ab
        den_mask = den < __EPSILON__
        den[den_mask] = np.inf
        X_new, Y_new, X1_new, Y1_new = -Y1_ab / den, Y_ab / den, X1_ab / den, -X_ab / den
        X_new[den_mask] = -1 / X_ab[den_mask]
        if self.T > __EPSILON__:
            new_mask = (w_a == w_b) & (n_a > __EPSILON__)
            Y1_new[new_mask] = -1 / Y1_ab[new_mask]
        return X_new, Y_new, X1_new, Y1_new

    def apply_L1_inverse_FT(self, psi, transpose=False):
        """Inverse of the harmonic (free) part of L, the preconditioner of the static solvers
        (DynamicalLanczos.py:2391-2502); host, O(n^2)."""
        n = self.n_modes
        out = np.zeros(np.shape(self.psi), dtype=TYPE_DP)
        if self.ignore_harmonic:
            return out
        psi = np.asarray(psi, dtype=TYPE_DP)
        m = n * (n + 1) // 2
        sY, sA = n, n + m
        assert len(psi) == sA + m, ("ERROR, the initial vector for the Lanczos algorithm has a wrong dimension. "
                                    "This may be caused by the Lanczos initialized at the wrong temperature.")
        X_new, Y_new, X1_new, Y1_new = self._l1_inverse_coefficients()
        out[:n] = (psi[:n] / self.w) / self.w
        out[sY:sA] = X_new * psi[sY:sA]
        if not transpose:
            out[sY:sA] += Y_new * psi[sA:]
            out[sA:] += X1_new * psi[sY:sA]
        else:
            out[sA:] += Y_new * psi[sY:sA]
            out[sY:sA] += X1_new * psi[sA:]
        out[sA:] += Y1_new * psi[sA:]
        return out

    def _bicgstab_batched(self, B, X0, rtol, maxiter, use_preconditioning, callback=None):
        """BiCGSTAB for the columns of B (k, |psi|) at once on the device, one batched apply of the
        still-active columns per operator application.  Per column it is scipy's bicgstab
        (scipy.sparse.linalg, rtol / atol = 0 semantics, breakdown tolerances eps^2); returns the
        solutions and scipy-style info codes (0 converged, maxiter, -10 / -11 breakdown)."""
        torch = _torch()
        dev = "cuda"
        n = self.n_modes
        m = n * (n + 1) // 2
        opts = self._opts()
        if use_preconditioning and not self.ignore_harmonic:
            co = [torch.as_tensor(a, device=dev) for a in self._l1_inverse_coefficients()]
            inv_w2 = torch.as_tensor(1.0 / self.w / self.w, device=dev)

            def psolve(x):
                y = torch.empty_like(x)
                y[:, :n] = x[:, :n] * inv_w2
                xY, xA = x[:, n:n + m], x[:, n + m:]
                y[:, n:n + m] = co[0] * xY + co[1] * xA
                y[:, n + m:] = co[2] * xY + co[3] * xA
                return y
        else:
            def psolve(x):
                return x.clone()

        def matvec(x):
            out = torch.empty_like(x)
            self.device_ensemble.apply_full_L(x.contiguous(), out, [0] * x.shape[0], opts, self.precision)
            return out

        def dot(a, b):
            return (a * b).sum(dim=1)

        b = torch.as_tensor(np.asarray(B, dtype=TYPE_DP), device=dev)
        x = torch.as_tensor(np.asarray(X0, dtype=TYPE_DP), device=dev).clone()
        k = b.shape[0]
        bnrm = torch.linalg.norm(b, dim=1)
        atol = rtol * bnrm
        info = np.full(k, maxiter, dtype=np.int64)
        active = (bnrm > 0).cpu().numpy()
        info[~active] = 0
        r = b - matvec(x) if bool((x != 0).any()) else b.clone()
        rt = r.clone()
        p = torch.zeros_like(r)
        v = torch.zeros_like(r)
        rho_prev = torch.ones(k, dtype=torch.float64, device=dev)
        alpha = torch.ones_like(rho_prev)
        omega = torch.ones_like(rho_prev)
        tiny = np.finfo(np.float64).eps ** 2
        first = np.ones(k, dtype=bool)
        for _ in range(maxiter):
            done = (torch.linalg.norm(r, dim=1) < atol).cpu().numpy() & active
            info[done] = 0
            active &= ~done
            idx = np.nonzero(active)[0]
            if len(idx) == 0:
                break
            it = torch.as_tensor(idx, device=dev)
            ra, rta = r[it], rt[it]
            rho = dot(rta, ra)
            bad = (rho.abs() < tiny).cpu().numpy()
            om_bad = ((omega[it].abs() < tiny).cpu().numpy()) & ~first[idx]
            info[idx[bad]] = -10
            info[idx[om_bad & ~bad]] = -11
            keep = ~(bad | om_bad)
            active[idx[~keep]] = False
            idx = idx[keep]
            if len(idx) == 0:
                continue
            it = torch.as_tensor(idx, device=dev)
            kt = torch.as_tensor(keep, device=dev)
            rho, ra, rta = rho[kt], ra[kt], rta[kt]
            fr = torch.as_tensor(first[idx], device=dev)
            beta = torch.where(fr, torch.zeros_like(rho), (rho / rho_prev[it]) * (alpha[it] / omega[it]))
            pa = torch.where(fr[:, None], ra, (p[it] - omega[it][:, None] * v[it]) * beta[:, None] + ra)
            first[idx] = False
            phat = psolve(pa)
            va = matvec(phat)
            rv = dot(rta, va)
            zero_rv = (rv == 0).cpu().numpy()
            if zero_rv.any():
                info[idx[zero_rv]] = -11
                active[idx[zero_rv]] = False
            al = rho / torch.where(rv == 0, torch.ones_like(rv), rv)
            sa = ra - al[:, None] * va
            conv = (torch.linalg.norm(sa, dim=1) < atol[it]).cpu().numpy() & ~zero_rv
            xa = x[it] + al[:, None] * phat
            # columns that converged on s take x + alpha phat and stop here
            cidx = np.nonzero(conv)[0]
            if len(cidx):
                ct = torch.as_tensor(cidx, device=dev)
                x[it[ct]] = xa[ct]
                info[idx[cidx]] = 0
                active[idx[cidx]] = False
            go = np.nonzero(~conv & ~zero_rv)[0]
            p[it], v[it], alpha[it], rho_prev[it] = pa, va, al, rho
            if len(go) == 0:
                continue
            gt = torch.as_tensor(go, device=dev)
            ig = it[gt]
            shat = psolve(sa[gt])
            t = matvec(shat)
            sg = sa[gt]
            om = dot(t, sg) / dot(t, t)
            omega[ig] = om
            x[ig] = xa[gt] + om[:, None] * shat
            r[ig] = sg - om[:, None] * t
            if callback is not None:
                callback(x)
        return x.cpu().numpy(), info

    def run_biconjugate_gradient(self, verbose=True, tol=5e-4, maxiter=1000, save_g=None, save_each=1,
                                 use_preconditioning=True, algorithm="bicgstab", batched=True, batch=16):
        """Static response by solving L x = e_i for every mode i (DynamicalLanczos.py:3761-3972);
        returns G^-1, the mass-rescaled free energy Hessian.  ``batched`` (default) solves ``batch``
        right-hand sides at a time with a device BiCGSTAB in which every operator application is
        one batched GPU apply; ``batched=False`` runs scipy's solver (``algorithm`` bicgstab | bicg |
        cg-minimize) with one GPU apply per matvec, as the reference does."""
        import scipy.optimize
        import scipy.sparse.linalg as sla
        self._check_init()
        if self.L_linop is None or self.M_linop is None:
            self._make_linops()
        n = self.n_modes
        G_one_phonon = np.zeros((n, n), dtype=np.double)
        if verbose:
            print("\n====================\nBICONJUGATE GRADIENT\n====================\n")
        if batched:
            if algorithm.lower() != "bicgstab":
                raise ValueError(f"batched=True runs bicgstab; got algorithm '{algorithm}' (pass batched=False)")
            for i0 in range(0, n, batch):
                cols = list(range(i0, min(n, i0 + batch)))
                B = np.zeros((len(cols), len(self.psi)), dtype=TYPE_DP)
                for q, i in enumerate(cols):
                    B[q, i] = 1.0
                X0 = np.stack([self.apply_L1_inverse_FT(bq) for bq in B])
                t1 = time.time()
                X, info = self._bicgstab_batched(B, X0, tol, maxiter, use_preconditioning)
                if verbose:
                    print(f"modes {cols[0] + 1}-{cols[-1] + 1} / {n}: solved in {time.time() - t1:.2f} s, info {info.tolist()}")
                assert np.all(info >= 0), f"Error on input or breakdown of biconjugate gradient algorithm (info = {info})"
                if verbose and np.any(info > 0):
                    print(f"The biconjugate gradient did not converge after {maxiter} iterations for modes "
                          f"{[cols[q] + 1 for q in np.nonzero(info > 0)[0]]}: reduce the tolerance or raise maxiter")
                G_one_phonon[cols, :] = X[:, :n]
                if save_g is not None:
                    np.save(save_g, G_one_phonon)
        else:
            for i in range(n):
                b = np.zeros(len(self.psi), dtype=TYPE_DP)
                b[i] = 1
                x0 = self.M_linop.matvec(b)
                M_prec = self.M_linop if use_preconditioning else None
                alg = algorithm.lower()
                if alg == "bicgstab":
                    res, info = sla.bicgstab(self.L_linop, b, x0=x0, rtol=tol, maxiter=maxiter, M=M_prec)
                elif alg == "bicg":
                    res, info = sla.bicg(self.L_linop, b, x0=x0, rtol=tol, maxiter=maxiter, M=M_prec)
                elif alg == "cg-minimize":
                    def func(x, bb):
                        r = self.L_linop.matvec(x) - bb
                        Hinv_r = self.M_linop.matvec(self.M_linop.rmatvec(r)) if use_preconditioning else r
                        return 0.5 * np.sum(r * Hinv_r), self.L_linop.rmatvec(Hinv_r)
                    opt = scipy.optimize.minimize(func, x0, args=(b.copy(),), method="bfgs", jac=True,
                                                  options={"gtol": tol, "maxiter": maxiter, "disp": verbose, "norm": 2})
                    res, info = opt.x.copy(), (0 if opt.success else 1)
                else:
                    raise ValueError(f"Error, algorithm type '{algorithm}' in subroutine run_biconjugate_gradient not "
                                     "implemented. the only supported algorithms are ['bicgstab', 'bicg', 'cg-minimize']")
                assert info >= 0, f"Error on input or breakdown of biconjugate gradient algorithm (info = {info})"
                G_one_phonon[i, :] = res[:n]
                if save_g is not None and i % save_each == 0:
                    np.save(save_g, G_one_phonon)
        if save_g is not None:
            np.save(save_g, G_one_phonon)
        disp = np.max(np.abs(G_one_phonon - G_one_phonon.T))
        assert disp < 1e-4, "Error, the resulting one-phonon Green function is not Hermitian."
        G = 0.5 * (G_one_phonon + G_one_phonon.T)
        return np.linalg.inv(G)

    def get_full_L_operator_FT(self, verbose=False, debug_d3=None, symmetrize=True, overwrite_L_operator=True,
                               batch=64, max_bytes=16 << 30):
        """The full L matrix (DynamicalLanczos.py:5454-5789).  Memory |psi|^2 x 8 B on the host.

        * symmetrize=False, or a debug_d3 tensor: the reference's analytic operator from the explicit
          d3 / d4 tensors of the ensemble, unsymmetrised (explicit_L_operator_FT).
        * symmetrize=True without debug_d3: the reference raises NotImplementedError unless
          ignore_v3 and ignore_v4 (it cannot symmetrise d3 / d4); here the symmetrised operator is
          built column by column from batched device applies of unit vectors, i.e. exactly the
          operator that apply_full_L applies (current flags)."""
        torch = _torch()
        self._check_init()
        ln = len(self.psi)
        if ln * ln * 8 > max_bytes:
            raise MemoryError(f"the full L operator needs {ln * ln * 8 / 2**30:.1f} GiB (limit {max_bytes / 2**30:.1f} GiB)")
        if debug_d3 is not None or not symmetrize:
            L = self.explicit_L_operator_FT(debug_d3=debug_d3, symmetrize=symmetrize, verbose=verbose)
            if overwrite_L_operator:
                import scipy.sparse.linalg as sla
                self.L_linop = sla.LinearOperator(L.shape, matvec=L.dot, rmatvec=lambda x: x.dot(L))
            return L
        L = np.zeros((ln, ln), dtype=TYPE_DP)
        opts = self._opts()
        for c0 in range(0, ln, batch):
            k = min(batch, ln - c0)
            E = torch.zeros((k, ln), dtype=torch.float64, device="cuda")
            E[torch.arange(k, device="cuda"), torch.arange(c0, c0 + k, device="cuda")] = 1.0
            out = torch.empty_like(E)
            self.device_ensemble.apply_full_L(E, out, [0] * k, opts, self.precision)
            L[:, c0:c0 + k] = out.cpu().numpy().T
        if overwrite_L_operator:
            import scipy.sparse.linalg as sla
            self.L_linop = sla.LinearOperator(L.shape, matvec=L.dot, rmatvec=L.T.dot, dtype=TYPE_DP)
        return L

    def explicit_tensors_FT(self, debug_d3=None, need_d3=True, need_d4=True):
        """The pair-space third- and fourth-order tensors of the reference's analytic operator
        (DynamicalLanczos.py:5578-5700), with x = X o ups, y = rho Y, N_eff = sum rho and the packed
        pairs p = (a_p, b_p) = (col, row) of the upper triangle:
          d3[p, c] = -(1 / 3 N_eff) sum_i (x_a x_b y_c + x_a x_c y_b + x_b x_c y_a)
                     (the six-permutation average of -x_a x_b y_c / N_eff)
          d4[p, q] = -(1 / 4 N_eff) sum_i [ (x_a x_b)_p (x y + y x)_q + (x y + y x)_p (x_a x_b)_q ]
        Both are FP64 GEMMs over the configurations on the device (O(P N n) and O(P^2 N)).
        debug_d3 (n, n, n), when given, replaces d3 as in the reference."""
        torch = _torch()
        n = self.n_modes
        r, c = np.triu_indices(n)
        dev = "cuda"
        n_w = 1 / (np.exp(self.w * __RyToK__ / self.T) - 1) if self.T > 0 else 0    # f_ups, :144-163
        ups = 2 * self.w / (1 + 2 * n_w)
        x = torch.as_tensor(np.asarray(self.X) * ups[None, :], device=dev)
        y = torch.as_tensor(np.asarray(self.Y) * np.asarray(self.rho)[:, None], device=dev)
        N_eff = float(np.sum(self.rho))
        ra, cb = torch.as_tensor(c, device=dev), torch.as_tensor(r, device=dev)   # a = col, b = row
        XX = (x[:, ra] * x[:, cb]).T.contiguous()                       # (P, N)
        XY = (x[:, ra] * y[:, cb] + y[:, ra] * x[:, cb]).T.contiguous()   # (P, N)
        d3 = d4 = None
        if need_d3:
            if debug_d3 is not None:
                d3 = np.asarray(debug_d3)[c, r, :].copy()
            else:
                d3 = (-(XX @ y + XY @ x) / (3.0 * N_eff)).cpu().numpy()
        if need_d4:
            d4 = (-(XX @ XY.T + XY @ XX.T) / (4.0 * N_eff)).cpu().numpy()
        return d3, d4

    def explicit_L_operator_FT(self, debug_d3=None, symmetrize=False, verbose=False):
        """The reference's analytic L operator (DynamicalLanczos.py:5454-5789) from the explicit,
        unsymmetrised d3 / d4 tensors: harmonic blocks, d3 couplings between R and the pair
        sectors, d4 couplings within the pair sectors, standard or Wigner representation, with the
        reference's double-counting factors.  As in the reference, symmetrize=True raises for the
        tensors it needs (no symmetrisation of d3 / d4 exists there)."""
        n = self.n_modes
        r, c = np.triu_indices(n)
        w_a, w_b = self.w[c], self.w[r]
        N_w2 = len(w_a)
        start_Y, start_A = n, n + N_w2
        L = np.zeros((n + 2 * N_w2, n + 2 * N_w2), dtype=TYPE_DP)
        if not self.ignore_harmonic:
            L[:n, :n] = np.diag(self.w ** 2) if not self.use_wigner else -np.diag(self.w ** 2)
        n_a = np.zeros(w_a.shape, dtype=TYPE_DP)
        n_b = np.zeros(w_a.shape, dtype=TYPE_DP)
        if self.T > 0:
            n_a = 1 / (np.exp(w_a * 157887.32400374097 / self.T) - 1)
            n_b = 1 / (np.exp(w_b * 157887.32400374097 / self.T) - 1)
        if not self.ignore_harmonic:
            if not self.use_wigner:
                X_ab_NI = -w_a ** 2 - w_b ** 2 - (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
                L[start_Y:start_A, start_Y:start_A] = -np.diag(X_ab_NI)
                Y_ab_NI = -(8 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
                L[start_Y:start_A, start_A:] = -np.diag(Y_ab_NI)
                X1_ab_NI = -(2 * n_a * n_b + n_a + n_b) * (2 * n_a * n_b + n_a + n_b + 1) * (2 * w_a * w_b) / (
                    (2 * n_a + 1) * (2 * n_b + 1))
                L[start_A:, start_Y:start_A] = -np.diag(X1_ab_NI)
                Y1_ab_NI = -w_a ** 2 - w_b ** 2 + (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1))
                L[start_A:, start_A:] = -np.diag(Y1_ab_NI)
            else:
                L[start_Y:start_A, start_Y:start_A] = np.diag(-(w_a ** 2 + w_b ** 2 - 2 * w_a * w_b))
                L[start_A:, start_A:] = np.diag(-(w_a ** 2 + w_b ** 2 + 2. * w_a * w_b))
        need_d3, need_d4 = not self.ignore_v3, not self.ignore_v4
        if need_d3 and symmetrize and debug_d3 is None:
            raise NotImplementedError('The symmetrizaiton on d3 is not implemented')
        if need_d4 and symmetrize:
            raise NotImplementedError('The symmetrizaiton on d4 is not implemented')
        d3, d4 = self.explicit_tensors_FT(debug_d3, need_d3, need_d4)
        double = np.where(c != r, 2, 1)
        if need_d3:
            if not self.use_wigner:
                Z_coeff = 2 * ((2 * n_a + 1) * w_b + (2 * n_b + 1) * w_a) / ((2 * n_a + 1) * (2 * n_b + 1))
                L[start_Y:start_A, :start_Y] = -d3 * Z_coeff[:, None]
                Z1_coeff = 2 * ((2 * n_a + 1) * w_b * n_b * (n_b + 1) + (2 * n_b + 1) * w_a * n_a * (n_a + 1)) / (
                    (2 * n_a + 1) * (2 * n_b + 1))
                L[start_A:, :start_Y] = -d3 * Z1_coeff[:, None]
                X2_coeff = (2 * n_b + 1) * (2 * n_a + 1) / (8 * w_a * w_b)
                L[:start_Y, start_Y:start_A] = -(d3 * (X2_coeff * double)[:, None]).T
            else:
                chi_minus = (n_a - n_b) * (w_a - w_b) / (2 * w_a * w_b)
                chi_plus = (1 + n_a + n_b) * (w_a + w_b) / (2 * w_a * w_b)
                L[:start_Y, start_Y:start_A] = (d3 * (np.sqrt(-0.5 * chi_minus) * double)[:, None]).T
                L[:start_Y, start_A:] = -(d3 * (np.sqrt(0.5 * chi_plus) * double)[:, None]).T
                L[start_Y:start_A, :start_Y] = d3 * np.sqrt(-0.5 * chi_minus)[:, None]
                L[start_A:, :start_Y] = -d3 * np.sqrt(0.5 * chi_plus)[:, None]
        if need_d4:
            if not self.use_wigner:
                X_left = -(2 * w_a * n_b + 2 * w_b * n_a + w_a + w_b) / (4 * (2 * n_a + 1) * (2 * n_b + 1))
                right = (2 * n_a + 1) * (2 * n_b + 1) / (w_a * w_b) * double
                L[start_Y:start_A, start_Y:start_A] += -(X_left[:, None] * d4 * right[None, :])
                X1_left = -(w_a * n_a * (n_a + 1) * (2 * n_b + 1) + w_b * n_b * (n_b + 1) * (2 * n_a + 1)) / (
                    4 * (2 * n_a + 1) * (2 * n_b + 1))
                L[start_A:, start_Y:start_A] += -(X1_left[:, None] * d4 * right[None, :])
            else:
                chi_plus = (1 + n_a + n_b) * (w_a + w_b) / (2 * w_a * w_b)
                chi_minus = (n_a - n_b) * (w_a - w_b) / (2 * w_a * w_b)
                sp, sm = np.sqrt(0.5 * chi_plus), np.sqrt(-0.5 * chi_minus)
                L[start_Y:start_A, start_Y:start_A] += -(sm[:, None] * d4 * (sm * double)[None, :])
                L[start_A:, start_A:] += -(sp[:, None] * d4 * (sp * double)[None, :])
                L[start_Y:start_A, start_A:] += sm[:, None] * d4 * (sp * double)[None, :]
                L[start_A:, start_Y:start_A] += sp[:, None] * d4 * (sm * double)[None, :]
        return L

    def run_full_diag(self, number, discard_dyn=True, n_iter=100):
        """ARPACK (scipy eigsh) on L_linop (DynamicalLanczos.py:6381-6421)."""
        import scipy.sparse.linalg as sla
        self._check_init()
        if self.L_linop is None:
            self._make_linops()
        eigvals, eigvects = sla.eigsh(self.L_linop, k=number, v0=self.psi, ncv=n_iter)
        self.eigvals = eigvals
        self.eigvects = eigvects
        if discard_dyn:
            eigvects = eigvects[:self.n_modes, :]
        return eigvals, eigvects

    def build_lanczos_matrix_from_coeffs(self, use_arnoldi=False):
        """Tridiagonal (bi-conjugate: b below, c above the diagonal) Lanczos matrix, sign-reversed
        and shifted like L (DynamicalLanczos.py:4571-4613)."""
        N_size = len(self.a_coeffs)
        matrix = np.zeros((N_size, N_size), dtype=TYPE_DP)
        if not use_arnoldi:
            for i in range(N_size):
                matrix[i, i] = self.a_coeffs[i]
                if i >= 1:
                    c_coeff = self.b_coeffs[i - 1]
                    if len(self.c_coeffs) == len(self.b_coeffs):
                        c_coeff = self.c_coeffs[i - 1]
                    matrix[i - 1, i] = c_coeff
                    matrix[i, i - 1] = self.b_coeffs[i - 1]
        else:
            assert len(self.b_coeffs) > len(self.c_coeffs), "Error, cannot Arnoldi with non-symmetric Lanczos not implemented"
            for i in range(N_size):
                matrix[:i + 1, i] = self.arnoldi_matrix[i]
                matrix[i, :i + 1] = self.arnoldi_matrix[i]
        sign = -1 if self.reverse_L else 1
        return sign * matrix - sign * np.eye(N_size) * self.shift_value

    # ---- static response: the free-energy Hessian (DynamicalLanczos.py:2502-2565, 3287-3354,
    #      3973-4235) --------------------------------------------------------------------------
    def _static_len(self):
        n = self.n_modes
        return n + n * (n + 1) // 2

    def apply_L1_static(self, psi, inverse=False, power=1):
        """Harmonic part of the static L: w^(2 power) on R, 1/Lambda^power on the packed Upsilon
        (tdscha_apply_L1_static_device, with the reference's Bose-mask quirks)."""
        torch = _torch()
        self._check_init()
        psi = np.asarray(psi, dtype=TYPE_DP)
        expected_dim = self._static_len()
        assert len(psi) == expected_dim, f"\nError, for the static calculation the vector must be of dimension {expected_dim}, got {len(psi)}\n"
        if inverse:
            power *= -1
        x = torch.as_tensor(psi, device="cuda").reshape(1, -1).contiguous()
        out = torch.empty_like(x)
        _native.apply_L1_static(self.device_ensemble, x, out, power)
        return out.cpu().numpy().ravel()

    def apply_anharmonic_static(self):
        """Anharmonic part of the static L on the static vector self.psi = (R, packed Upsilon):
        (-f_av, packed D_av) of R1 = R, Upsilon1 = -2 Yw Upsilon Yw."""
        torch = _torch()
        self._check_init()
        x = torch.as_tensor(np.asarray(self.psi[:self._static_len()], dtype=TYPE_DP), device="cuda").reshape(1, -1).contiguous()
        out = torch.empty_like(x)
        _native.apply_static_L(self.device_ensemble, x, out, ignore_v4=self.ignore_v4, include_L1=False,
                               precision=self.precision)
        res = np.zeros(self.psi.shape, dtype=TYPE_DP)
        res[:x.shape[1]] = out.cpu().numpy().ravel()
        return res

    def _static_apply_batched(self, X, eigen_shift=1.0, with_L1=True):
        """The matvec of run_hessian_calculation on a (k, len) device batch."""
        torch = _torch()
        n = self.n_modes
        Xs = X.clone()
        Xs[:, n:] *= eigen_shift
        out = torch.empty_like(Xs)
        _native.apply_static_L(self.device_ensemble, Xs, out, ignore_v4=self.ignore_v4, include_L1=with_L1,
                               precision=self.precision)
        out[:, n:] *= eigen_shift
        return out

    def _static_precond_batched(self, X, power=0.5):
        torch = _torch()
        out = torch.empty_like(X)
        _native.apply_L1_static(self.device_ensemble, X.contiguous(), out, -power)
        return out

    def run_hessian_calculation(self, verbose=True, eigen_shift=1, tol=5e-4, max_iters=1000, save_g=None, save_each=1,
                                use_preconditioning=True, algorithm="cg"):
        """Static susceptibility by one linear solve per mode, then its inverse: the mass-rescaled
        free-energy Hessian (DynamicalLanczos.py:3973-4235).  With algorithm "cg" (the reference's
        minimum-residual method, Tools.py:265-471) the n solves advance together: every iteration
        applies the static L to all still-unconverged right-hand sides in batches of 64 on the
        device.  "minimize" / "minimize-quad" run scipy's BFGS per mode on the device matvec, as
        the reference does."""
        G_one_phonon = self.static_green_function(verbose, eigen_shift, tol, max_iters, save_g, save_each,
                                                  use_preconditioning, algorithm)
        disp = np.max(np.abs(G_one_phonon - G_one_phonon.T))
        assert disp < 1e-4, "Error, the resulting one-phonon Green function is not Hermitian."
        G = 0.5 * (G_one_phonon + G_one_phonon.T)
        return np.linalg.inv(G)

    def static_green_function(self, verbose=True, eigen_shift=1, tol=5e-4, max_iters=1000, save_g=None, save_each=1,
                              use_preconditioning=True, algorithm="cg"):
        """The rows G[i, :] = (L_static^-1 e_i)[:n] that run_hessian_calculation symmetrises and
        inverts (DynamicalLanczos.py:4024-4218), before its absolute hermiticity check (1e-4, which
        trips on Green functions of order 1/w^2 in Rydberg units)."""
        torch = _torch()
        self._check_init()
        n = self.n_modes
        ln = self._static_len()
        if verbose:
            print("\n=====================\n HESSIAN CALCULATION \n=====================\n")
        G_one_phonon = np.zeros((n, n), dtype=np.double)
        alg = algorithm.lower()
        if alg == "cg":
            B = torch.zeros((n, ln), dtype=torch.float64, device="cuda")
            B[torch.arange(n), torch.arange(n)] = 1.0
            A = lambda X: self._static_apply_batched(X, eigen_shift)                  # noqa: E731
            if not use_preconditioning:
                res = minimum_residual_batched(A, B, B.clone(), max_iters=max_iters, verbose=verbose)
            else:
                M = self._static_precond_batched
                res = minimum_residual_batched_precond(A, B, M, max_iters=max_iters, verbose=verbose)
            G_one_phonon[:, :] = res[:, :n].cpu().numpy()
        elif alg in ("minimize", "minimize-quad"):
            import scipy.optimize

            def matvec(x):
                X = torch.as_tensor(x, device="cuda").reshape(1, -1).contiguous()
                return self._static_apply_batched(X, eigen_shift).cpu().numpy().ravel()

            for i in range(n):
                b = np.zeros(ln)
                b[i] = 1

                def func_standard(x, b):
                    Lx = matvec(x)
                    return 0.5 * x.dot(Lx) - b.dot(x), Lx - b

                def func_quad(x, b):
                    r = matvec(x) - b
                    return 0.5 * np.sum(r ** 2), matvec(r)

                options = {"gtol": tol, "maxiter": max_iters, "disp": verbose, "norm": 2}
                fn = func_standard if alg == "minimize" else func_quad
                results = scipy.optimize.minimize(fn, b.copy(), args=(b,), method="bfgs", jac=True, options=options)
                G_one_phonon[i, :] = results.x[:n]
                if save_g is not None and i % save_each == 0:
                    np.save(save_g, G_one_phonon)
        else:
            raise ValueError(f"""
Error, algorithm type '{algorithm}' in subroutine run_biconjugate_gradient not implemented.
       the only supported algorithms are ['bicgstab', 'bicg']
""")
        if save_g is not None:
            np.save(save_g, G_one_phonon)
        return G_one_phonon

    def get_static_frequency(self, smearing=0):
        """sqrt(1 / Re G(omega -> 0 + i eta)), negative when imaginary (DynamicalLanczos.py:5273-5307)."""
        gf = self.get_green_function_continued_fraction(np.array([0]), False, smearing=smearing)
        w2 = 1 / np.real(gf[0])
        return np.float64(np.sqrt(np.abs(w2)) * np.sign(w2))

    # ---- input / output files of the stand-alone Lanczos program (DynamicalLanczos.py:815-1000,
    #      3572-3595; CModules/Lanczos.cpp:47-269, 533-800) ---------------------------------------
    def prepare_input_files(self, root_name="tdscha", n_steps=100, start_from_scratch=True, directory=".", run_symm=False):
        """Write <root>.json, .ndegs, .blockid, .masses, .freqs, .rho, .X.dat, .Y.dat, .psi,
        .block<i>, .symsb<i> for the stand-alone program (tdscha_lanczos_b200 here, tdscha-lanczos.x
        in the reference), in the reference's formats."""
        Nsyms = np.shape(self.symmetries[0])[0]
        json_data = {"T": self.T, "n_steps": n_steps, "ignore_v2": self.ignore_harmonic, "ignore_v3": self.ignore_v3,
                     "ignore_v4": self.ignore_v4, "use_wigner": self.use_wigner, "run_sym": run_symm,
                     "data": {"n_configs": int(self.N), "n_modes": int(self.n_modes), "n_syms": int(Nsyms),
                              "n_blocks": len(self.symmetries), "perturbation_modulus": float(self.perturbation_modulus),
                              "reverse": bool(self.reverse_L), "shift": float(self.shift_value)}}
        if not start_from_scratch:
            raise NotImplementedError("Error, restarting from a previous calculation is not yet implemented.")
        root_fname = os.path.join(directory, root_name)
        os.makedirs(directory, exist_ok=True)
        with open(root_fname + ".json", "w") as fp:
            json.dump(json_data, fp)
        np.savetxt(root_fname + ".ndegs", self.N_degeneracy, fmt="%d")
        np.savetxt(root_fname + ".blockid", self.sym_block_id, fmt="%d")
        np.savetxt(root_fname + ".masses", self.m)
        np.savetxt(root_fname + ".freqs", self.w)
        np.savetxt(root_fname + ".rho", self.rho)
        np.savetxt(root_fname + ".X.dat", self.X)
        np.savetxt(root_fname + ".Y.dat", self.Y)
        np.savetxt(root_fname + ".psi", self.psi)
        for i in range(len(self.symmetries)):
            np.savetxt(root_fname + ".block{:d}".format(i), self.degenerate_space[i], fmt="%d")
            ns, b1, b2 = self.symmetries[i].shape
            with open(root_fname + ".symsb{:d}".format(i), "w") as fp:
                for isym in range(ns):
                    for k1 in range(b1):
                        fp.write("".join(" {:22.16f}".format(v) for v in self.symmetries[i][isym, k1]))
                        fp.write("\n")
                    fp.write("\n")

    def load_from_input_files(self, root_name="tdscha", directory="."):
        """Read the program's results (<root>.abc, and .qbasis.out / .pbasis.out / .snorm.out when
        present) and the general variables of <root>.json."""
        if not os.path.exists(directory):
            raise IOError("Error, the specified directory '{}' does not exist".format(directory))
        abc_file = os.path.join(directory, "{}.abc".format(root_name))
        if not os.path.exists(abc_file):
            raise IOError(f"Error, the file '{abc_file}' does not exist. please, check if you correctly run the "
                          "stand-alone Lanczos program.")
        data_abc = np.loadtxt(abc_file, dtype=np.double)
        self.a_coeffs = data_abc[:, 0]
        self.b_coeffs = data_abc[:, 1]
        self.c_coeffs = data_abc[:, 2]
        for attr, suffix in (("basis_Q", "qbasis.out"), ("basis_P", "pbasis.out"), ("s_norm", "snorm.out")):
            fname = os.path.join(directory, "{}.{}".format(root_name, suffix))
            if os.path.exists(fname):
                v = np.loadtxt(fname, dtype=np.double)
                setattr(self, attr, v.ravel() if attr == "s_norm" else v)
            else:
                warnings.warn(f"File {fname} not found. {attr} not loaded.")
        with open(os.path.join(directory, root_name + ".json"), "r") as fp:
            json_data = json.load(fp)
        self.perturbation_modulus = json_data["data"]["perturbation_modulus"]
        self.T = json_data["T"]
        self.ignore_harmonic = json_data["ignore_v2"]
        self.ignore_v3 = json_data["ignore_v3"]
        self.ignore_v4 = json_data["ignore_v4"]
        self.N = json_data["data"]["n_configs"]
        self.n_modes = json_data["data"]["n_modes"]
        self.reverse_L = json_data["data"]["reverse"]
        self.shift_value = json_data["data"]["shift"]

    def save_abc(self, file):
        total_len = len(self.c_coeffs)
        abc = np.zeros((total_len, 3), dtype=np.double)
        abc[:, 0] = self.a_coeffs[:total_len]
        abc[:, 1] = self.b_coeffs
        abc[:, 2] = self.c_coeffs
        np.savetxt(file, abc, header="a; b; c")

    def load_abc(self, file):
        abc = np.loadtxt(file)
        self.a_coeffs = abc[:, 0]
        self.b_coeffs = abc[:, 1]
        self.c_coeffs = abc[:, 2]

    # ---- checkpoints (DynamicalLanczos.py:3597-3758) -----------------------------------------
    def save_status(self, file):
        if ".npz" not in file.lower():
            file += ".npz"
        np.savez_compressed(file, T=self.T, nat=self.nat, m=self.m, w=self.w, pols=self.pols, n_modes=self.n_modes,
                            ignore_v3=self.ignore_v3, ignore_v4=self.ignore_v4, N=self.N, rho=self.rho, X=self.X,
                            Y=self.Y, psi=self.psi, a_coeffs=self.a_coeffs, b_coeffs=self.b_coeffs,
                            c_coeffs=self.c_coeffs, basis_Q=self.basis_Q, basis_P=self.basis_P, s_norm=self.s_norm,
                            krilov_basis=self.krilov_basis, arnoldi_matrix=self.arnoldi_matrix, reverse=self.reverse_L,
                            shift=self.shift_value, perturbation_modulus=self.perturbation_modulus,
                            use_wigner=self.use_wigner, ignore_small_w=self.ignore_small_w, sym_julia=self.sym_julia,
                            deg_julia=self.deg_julia, n_syms=self.n_syms)

    def load_status(self, file, is_file_instance=False):
        if not is_file_instance:
            if ".npz" not in file.lower():
                file += ".npz"
            if not os.path.exists(file):
                raise IOError("Error while loading %s" % file)
        data = dict(np.load(file, allow_pickle=True))
        self.T = np.double(data["T"])
        self.nat = np.intc(data["nat"])
        self.m = data["m"]
        self.w = data["w"]
        self.pols = data["pols"]
        self.n_modes = np.intc(data["n_modes"])
        self.ignore_v3 = bool(data["ignore_v3"])
        self.ignore_v4 = bool(data["ignore_v4"])
        self.N = np.intc(data["N"])
        self.rho = data["rho"]
        self.X = data["X"]
        self.Y = data["Y"]
        self.psi = data["psi"]
        self.a_coeffs = list(data["a_coeffs"])
        self.b_coeffs = list(data["b_coeffs"])
        self.c_coeffs = list(data["c_coeffs"]) if "c_coeffs" in data else []
        self.krilov_basis = data["krilov_basis"]
        self.arnoldi_matrix = data["arnoldi_matrix"]
        self.sym_julia = data.get("sym_julia")
        self.deg_julia = data.get("deg_julia")
        self.n_syms = data.get("n_syms", 1)
        self.basis_Q = data["basis_Q"]
        self.basis_P = data["basis_P"]
        self.s_norm = data["s_norm"]
        self.use_wigner = bool(data["use_wigner"])
        self.ignore_small_w = bool(data.get("ignore_small_w", False))
        if "reverse" in data:
            self.reverse_L = bool(data["reverse"])
            self.shift_value = float(data["shift"])
        if "perturbation_modulus" in data:
            self.perturbation_modulus = float(data["perturbation_modulus"])
        self.N_eff = float(np.sum(self.rho))


def _gram_schmidt(q, p, window, n_rep_orth, c_coeff, mask):
    """Gram-Schmidt of the new pair (q, p) against the last basis pairs `window` (device vectors),
    DynamicalLanczos.py:6244-6316 with its conventions: sequential updates, q normalised by its norm
    and p by its squared norm, s_norm re-derived from p . q, and the stop test on the q coefficients
    only.  Returns (q, p, s_norm, next_converged)."""
    def dot(a, b):
        return float((a * b).sum()) if mask is None else float((a * b * mask).sum())

    next_converged = False
    s_norm = None
    for _ in range(n_rep_orth):
        ortho_q = 0.0
        for Qj, Pj in window:
            c1 = dot(Pj, q)
            c2 = dot(Qj, p)
            q = q - c1 * Pj
            p = p - c2 * Qj
            ortho_q += abs(c1)
        normq = np.sqrt(dot(q, q))
        if normq < __EPSILON__:
            next_converged = True
        q = q / normq
        normp = dot(p, p)
        if abs(normp) < __EPSILON__:
            next_converged = True
        p = p / normp
        s_norm = c_coeff / dot(p, q)
        if ortho_q < __EPSILON__:
            break
    return q, p, s_norm, next_converged


def run_FT_batched(lanczos_list, n_iter, save_dir=None, save_each=5, verbose=False, n_rep_orth=0, run_simm=False,
                   prefix=None, precision=None, n_ortho=10):
    """Advance several bi-conjugate Lanczos chains that share one ensemble in lockstep: each step
    is ONE batched apply over [L q_c, L^T p_c for every active chain] plus one batched recurrence
    launch; all vectors stay in HBM.  Chains stop independently on breakdown (|b| or |c| < 1e-12)."""
    torch = _torch()
    L0 = lanczos_list[0]
    dev_ens = L0.device_ensemble
    for L in lanczos_list:
        L._check_init()
        if L.device_ensemble is not dev_ens:
            raise ValueError("batched chains must share one initialised ensemble (set lanc.device_ensemble)")
        if run_simm and not L.use_wigner:
            raise NotImplementedError('The symmetric Lanczos works only with Wigner. Set use_wigner to True')
        psi = np.asarray(L.psi)
        if np.isnan(np.sum(psi ** 2)) or np.sum(psi ** 2) == 0:
            raise ValueError("Error, you must initialize a perturbation to start the Lanczos.")
    prec = precision or L0.precision
    nc = len(lanczos_list)
    n = L0.n_modes
    length = n + n * (n + 1)
    mask = torch.as_tensor(L0.mask_dot_wigner(), device="cuda") if run_simm else None
    dev = "cuda"
    # per chain device state: current q, p, previous q, p
    state = []
    for L in lanczos_list:
        if len(L.a_coeffs) == 0:
            v = torch.as_tensor(np.asarray(L.psi, dtype=np.float64), device=dev)
            nrm = torch.sqrt((v * v * (mask if mask is not None else 1.0)).sum())
            first = v / nrm
            L.basis_Q, L.basis_P, L.s_norm = [first.cpu().numpy()], [first.cpu().numpy()], [1]
        L.basis_Q, L.basis_P, L.s_norm = list(L.basis_Q), list(L.basis_P), list(L.s_norm)
        L.a_coeffs, L.b_coeffs, L.c_coeffs = list(L.a_coeffs), list(L.b_coeffs), list(L.c_coeffs)
        q = torch.as_tensor(np.asarray(L.basis_Q[-1]), device=dev)
        p = torch.as_tensor(np.asarray(L.basis_P[-1]), device=dev)
        qp = torch.as_tensor(np.asarray(L.basis_Q[-2]), device=dev) if len(L.basis_Q) > 1 else torch.zeros_like(q)
        pp = torch.as_tensor(np.asarray(L.basis_P[-2]), device=dev) if len(L.basis_P) > 1 else torch.zeros_like(p)
        window = []
        if n_rep_orth:      # the last n_ortho basis pairs, for the Gram-Schmidt of the next vectors
            start = max(0, len(L.basis_P) - n_ortho) if n_ortho is not None else 0
            window = [(torch.as_tensor(np.asarray(L.basis_Q[j]), device=dev),
                       torch.as_tensor(np.asarray(L.basis_P[j]), device=dev)) for j in range(start, len(L.basis_P))]
        state.append({"q": q, "p": p, "qp": qp, "pp": pp, "done": False, "L": L, "window": window,
                      "next_converged": False})
    opts = L0._opts()
    for it in range(n_iter):
        active = [s for s in state if not s["done"]]
        if not active:
            break
        na = len(active)
        if run_simm:
            vecs = torch.stack([s["q"] for s in active])
            tr = [0] * na
        else:
            vecs = torch.stack([s["q"] for s in active] + [s["p"] for s in active])
            tr = [0] * na + [1] * na
        out = torch.empty_like(vecs)
        dev_ens.apply_full_L(vecs, out, tr, opts, prec)
        Lq = out[:na]
        pL = out[:na].clone() if run_simm else out[na:]
        sc_in = torch.tensor([[s["L"].c_coeffs[-1] if s["L"].c_coeffs else 0.0,
                               s["L"].b_coeffs[-1] if s["L"].b_coeffs else 0.0,
                               s["L"].s_norm[-1],
                               s["L"].s_norm[-2] if len(s["L"].s_norm) > 1 else 0.0,
                               s["L"].c_coeffs[-2] if len(s["L"].c_coeffs) > 1 else 1.0,
                               float(len(s["L"].a_coeffs))] for s in active], dtype=torch.float64, device=dev)
        Q = torch.stack([s["q"] for s in active]).contiguous()
        Pm = torch.stack([s["p"] for s in active]).contiguous()
        QP = torch.stack([s["qp"] for s in active]).contiguous()
        PP = torch.stack([s["pp"] for s in active]).contiguous()
        qn = torch.empty_like(Q)
        pn = torch.empty_like(Pm)
        sc_out = torch.empty((na, 4), dtype=torch.float64, device=dev)
        _native.lanczos_step(Lq.contiguous(), pL.contiguous(), Q, Pm, QP, PP, sc_in, mask, qn, pn, sc_out)
        sc = sc_out.cpu().numpy()
        for ci, s in enumerate(active):
            L = s["L"]
            a, b, c, snew = (float(x) for x in sc[ci])
            if np.isnan(a):
                raise ValueError("Invalid value encountered during the Lanczos.")
            L.a_coeffs.append(a)
            if abs(b) < __EPSILON__ or abs(c) < __EPSILON__ or s["next_converged"]:
                s["done"] = True
                continue
            q_new, p_new = qn[ci], pn[ci]
            if n_rep_orth:
                q_new, p_new, s_gs, s["next_converged"] = _gram_schmidt(q_new.clone(), p_new.clone(), s["window"],
                                                                        n_rep_orth, c, mask)
                if s_gs is not None:
                    snew = s_gs
                s["window"].append((q_new, p_new))
                if n_ortho is not None and len(s["window"]) > n_ortho:
                    s["window"].pop(0)
            s["qp"], s["pp"] = s["q"], s["p"]
            s["q"], s["p"] = q_new, p_new
            L.basis_Q.append(q_new.cpu().numpy())
            L.basis_P.append(p_new.cpu().numpy())
            L.b_coeffs.append(b)
            L.c_coeffs.append(c)
            L.s_norm.append(snew)
            if save_dir is not None and len(L.a_coeffs) % save_each == 0:
                os.makedirs(save_dir, exist_ok=True)
                pre = prefix[state.index(s)] if prefix else "LANCZOS"
                L.save_status(os.path.join(save_dir, f"{pre}_STEP{len(L.a_coeffs)}"))
        if verbose:
            print(f"Lanczos step {it + 1}: " + ", ".join(f"a={s['L'].a_coeffs[-1]:.6e}" for s in active))
            sys.stdout.flush()
    for s in state:
        s["L"].psi = s["q"].cpu().numpy()


def run_FT_multi(groups, n_iter, precision=None, use_graph=True):
    """Advance the bi-conjugate chains of several systems together for n_iter steps without returning
    to the host (tdscha_lanczos_run_device): ``groups`` has one entry per system, a list of at most
    32 Lanczos objects sharing that system's initialised device ensemble.  Every step is one batched
    apply per system (all its chains' L q and L^T p), one batched recurrence and the history update;
    systems run on their own streams and, with use_graph, all steps after the first two are one CUDA
    graph launch.

    Afterwards every chain holds its coefficients up to its first breakdown (|b| or |c| < 1e-12, where
    run_FT stops, DynamicalLanczos.py:6129-6141) and psi = its last q.  Unlike run_FT the basis is not
    kept: basis_Q / basis_P end with the last two vectors only (the full basis is only needed for
    Gram-Schmidt re-orthogonalisation, n_rep_orth > 0, which MODE_B200 does not provide)."""
    torch = _torch()
    from . import _native
    dev = "cuda"
    systems, meta = [], []
    for g, chains in enumerate(groups):
        if not chains or len(chains) > 32:
            raise ValueError(f"system {g}: 1..32 chains per system (got {len(chains)})")
        L0 = chains[0]
        for L in chains:
            L._check_init()
            if L.device_ensemble is not L0.device_ensemble:
                raise ValueError(f"system {g}: the chains of one system must share its device ensemble")
            flags = lambda o: (o.use_wigner, o.ignore_harmonic, o.ignore_v3, o.ignore_v4, o.reverse_L, o.shift_value)  # noqa: E731
            if flags(L._opts()) != flags(L0._opts()):
                raise ValueError(f"system {g}: the chains of one system must share the apply flags")
            psi = np.asarray(L.psi)
            if np.isnan(np.sum(psi ** 2)) or np.sum(psi ** 2) == 0:
                raise ValueError("Error, you must initialize a perturbation to start the Lanczos.")
        nc = len(chains)
        ln = len(L0.psi)
        qp = torch.zeros((4, nc, ln), dtype=torch.float64, device=dev)
        sc = torch.zeros((nc, 6), dtype=torch.float64, device=dev)
        for ci, L in enumerate(chains):
            if len(L.a_coeffs) == 0:
                v = np.asarray(L.psi, dtype=np.float64)
                first = v / np.sqrt(np.sum(v * v))
                L.basis_Q, L.basis_P, L.s_norm = [first], [first], [1]
            L.basis_Q, L.basis_P, L.s_norm = list(L.basis_Q), list(L.basis_P), list(L.s_norm)
            L.a_coeffs, L.b_coeffs, L.c_coeffs = list(L.a_coeffs), list(L.b_coeffs), list(L.c_coeffs)
            qp[0, ci] = torch.as_tensor(np.asarray(L.basis_Q[-1]), device=dev)
            qp[1, ci] = torch.as_tensor(np.asarray(L.basis_P[-1]), device=dev)
            if len(L.basis_Q) > 1:
                qp[2, ci] = torch.as_tensor(np.asarray(L.basis_Q[-2]), device=dev)
                qp[3, ci] = torch.as_tensor(np.asarray(L.basis_P[-2]), device=dev)
            sc[ci] = torch.tensor([L.c_coeffs[-1] if L.c_coeffs else 0.0, L.b_coeffs[-1] if L.b_coeffs else 0.0,
                                   L.s_norm[-1], L.s_norm[-2] if len(L.s_norm) > 1 else 0.0,
                                   L.c_coeffs[-2] if len(L.c_coeffs) > 1 else 1.0, float(len(L.a_coeffs))],
                                  dtype=torch.float64)
        coef = torch.zeros((n_iter, nc, 4), dtype=torch.float64, device=dev)
        systems.append((L0.device_ensemble, qp, sc, coef, L0._opts(), precision or L0.precision))
        meta.append(chains)
    _native.lanczos_run(systems, n_iter, use_graph=use_graph)
    torch.cuda.synchronize()
    for (ens, qp, sc, coef, _, _), chains in zip(systems, meta):
        cf = coef.cpu().numpy()
        q_host = qp.cpu().numpy()
        for ci, L in enumerate(chains):
            for k in range(n_iter):
                a, b, c, snew = (float(x) for x in cf[k, ci])
                if np.isnan(a):
                    raise ValueError("Invalid value encountered during the Lanczos.")
                L.a_coeffs.append(a)
                if abs(b) < __EPSILON__ or abs(c) < __EPSILON__:
                    break
                L.b_coeffs.append(b)
                L.c_coeffs.append(c)
                L.s_norm.append(snew)
            L.basis_Q = [q_host[2, ci], q_host[0, ci]]
            L.basis_P = [q_host[3, ci], q_host[1, ci]]
            L.psi = q_host[0, ci]


# ---- the reference's minimum-residual solver (Modules/Tools.py:265-471), batched over rows ----
def minimum_residual_batched(A, B, X0, max_iters=100, conv_thr=1e-6, verbose=False, callback=None):
    """Tools.minimum_residual_algorithm (precond = None) for every row of B at once: A maps a
    (k, len) device batch to A applied to each row.  Each row runs the reference's iteration and
    stops when its residual |r| / |b| falls below conv_thr (or at max_iters); the apply of one
    iteration covers only the rows still running."""
    torch = _torch()
    r1 = B - A(X0)
    b_norm = torch.sqrt((B * B).sum(1))
    r1_bar = A(r1)
    z1 = r1.clone()
    p1 = r1.clone()
    p1_bar = r1_bar.clone()
    x = X0.clone()
    active = torch.ones(B.shape[0], dtype=torch.bool, device=B.device)
    iters = 1
    while iters < max_iters:
        idx = torch.nonzero(active).ravel()
        if idx.numel() == 0:
            break
        Ap = p1_bar[idx]
        Ap_bar = A(Ap.contiguous())
        alpha = (r1_bar[idx] * z1[idx]).sum(1) / (Ap * Ap).sum(1)
        x[idx] += alpha[:, None] * p1[idx]
        if callback is not None:
            callback(x, iters)
        r = r1[idx] - alpha[:, None] * Ap
        rbar = r1_bar[idx] - alpha[:, None] * Ap_bar
        r_norm = torch.sqrt((r * r).sum(1)) / b_norm[idx]
        beta = (rbar * r).sum(1) / (r1_bar[idx] * z1[idx]).sum(1)
        p1[idx] = r + beta[:, None] * p1[idx]
        p1_bar[idx] = rbar + beta[:, None] * p1_bar[idx]
        r1[idx] = r
        r1_bar[idx] = rbar
        z1[idx] = r
        active[idx[r_norm < conv_thr]] = False
        if verbose:
            print(f"Iteration {iters}: {int(active.sum())} of {B.shape[0]} still running, max residual "
                  f"{float(r_norm.max()):.3e}")
        iters += 1
    if bool(active.any()):
        print(f"WARNING: cg did not converge after {max_iters} iterations for {int(active.sum())} right-hand sides.")
    return x


def minimum_residual_batched_precond(A, B, precond_half, X0=None, **kwargs):
    """Tools.minimum_residual_algorithm_precond, batched: solve M A M x~ = M b, x = M x~."""
    A_tilde = lambda X: precond_half(A(precond_half(X)))     # noqa: E731
    B_tilde = precond_half(B)
    if X0 is None:
        X0 = B_tilde.clone()
    return precond_half(minimum_residual_batched(A_tilde, B_tilde, X0, **kwargs))
