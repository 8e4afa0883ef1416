"""
CPU oracle for the TD-SCHA Lanczos hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, always as the checker or the timed
CPU baseline, never by the product package.

It restates, in numpy, the FP64 host-side code of the reference ``tdscha.DynamicalLanczos.Lanczos``
around the C kernel, following these reference lines (Modules/DynamicalLanczos.py):

  apply_L1_FT                              :2227-2385
  get_Y1 / get_ReA1                        :2827-2888
  get_chi_minus / get_chi_plus             :2572-2627
  get_alpha1_beta1_wigner                  :2713-2822
  apply_anharmonic_FT (standard + Wigner)  :2891-3281
  apply_full_L                             :3467-3570
  mask_dot_wigner                          :5790-5839
  run_FT (bi-conjugate Lanczos, with the optional Gram-Schmidt of :6244-6316)    :5843-6374
  get_green_function_continued_fraction    :4951-5047
  prepare_perturbation / prepare_mode      :1963-2031
  apply_L1_static / apply_anharmonic_static :2502-2565, 3287-3354
  run_hessian_calculation ("cg")           :3973-4235
and Modules/Tools.py:265-471 (minimum_residual_algorithm[_precond]), Modules/StaticHessian.py:561-690
(the system matrix of StaticHessian), and the analytic L operator from explicit d3 / d4 tensors
(get_full_L_operator_FT, :5454-5789).

The symmetrised averages (the reference's ``sscha_HP_odd.GetPerturbAverageSym``,
CModules/odd_corr_module.c:491-634) come from one of two C back ends:

  "port"      -- oracle/tdscha_oracle.c, our pair-by-pair restatement (OpenMP over configs);
  "reference" -- oracle/_ref/sscha_HP_odd*.so, the reference's own C compiled from its sources.
"""
from __future__ import annotations

import ctypes
import glob
import os
import sys

import numpy as np

RY_TO_K = 157887.32400374097      # Modules/DynamicalLanczos.py:134, CModules/LanczosFunctions.h:9
EPSILON = 1e-12                   # Modules/DynamicalLanczos.py:121

_HERE = os.path.dirname(os.path.abspath(__file__))


# ----------------------------------------------------------------------------------------------
# C back ends for the averages
# ----------------------------------------------------------------------------------------------
_port_lib = None
_ref_mod = None


def port_library():
    """Load oracle/_build/libtdscha_oracle.so (built by ``make -C oracle``)."""
    global _port_lib
    if _port_lib is None:
        path = os.path.join(_HERE, "_build", "libtdscha_oracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.oracle_perturb_average_sym.argtypes = [
            dp, dp, dp, dp, dp, dp, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, dp, ip,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        lib.oracle_perturb_average_sym.restype = ctypes.c_int
        _port_lib = lib
    return _port_lib


def reference_module():
    """Import the reference's own ``sscha_HP_odd`` built into oracle/_ref (``make -C oracle ref``)."""
    global _ref_mod
    if _ref_mod is None:
        refdir = os.path.join(_HERE, "_ref")
        if not glob.glob(os.path.join(refdir, "sscha_HP_odd*.so")):
            raise FileNotFoundError(f"reference kernel not built in {refdir}: run `make -C oracle ref`")
        if refdir not in sys.path:
            sys.path.insert(0, refdir)
        import sscha_HP_odd  # noqa: E402
        _ref_mod = sscha_HP_odd
    return _ref_mod


class _SilenceStdout:
    """The reference kernel prints one line per call (LanczosFunctions.c:2139); drop it."""

    def __enter__(self):
        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        try:
            ctypes.CDLL(None).fflush(None)
        except Exception:
            pass
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def perturb_average_sym(X, Y, w, rho, R1, Y1, T, apply_d4, symmetries, n_deg, deg_space, blocks_ids,
                        backend="port", i_range=None, n_threads=0):
    """Symmetrised perturbed averages (f_av (n), d2v_av (n, n)) with the semantics of
    CModules/odd_corr_module.c:491-634.  ``symmetries`` is the list of per-block (N_sym, d, d)
    tables, ``deg_space`` the list of per-block mode-index arrays."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    R1 = np.ascontiguousarray(R1, dtype=np.float64)
    Y1 = np.ascontiguousarray(Y1, dtype=np.float64)
    N, n = X.shape
    N_sym = int(symmetries[0].shape[0])
    f_out = np.zeros(n, dtype=np.float64)
    d_out = np.zeros((n, n), dtype=np.float64)
    if backend == "reference":
        if i_range is not None:
            raise ValueError("the reference kernel always runs on the whole ensemble")
        mod = reference_module()
        syms = [np.ascontiguousarray(s, dtype=np.float64) for s in symmetries]
        degs = [np.ascontiguousarray(d, dtype=np.intc) for d in deg_space]
        with _SilenceStdout():
            mod.GetPerturbAverageSym(X, Y, w, rho, R1, Y1, float(T), int(apply_d4), N_sym, syms,
                                     np.ascontiguousarray(n_deg, dtype=np.intc), degs,
                                     np.ascontiguousarray(blocks_ids, dtype=np.intc), f_out, d_out)
        return f_out, d_out
    lib = port_library()
    sym_flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64).ravel() for s in symmetries]))
    deg_flat = np.ascontiguousarray(np.concatenate([np.asarray(d, dtype=np.intc).ravel() for d in deg_space]).astype(np.intc))
    n_deg = np.ascontiguousarray(n_deg, dtype=np.intc)
    bid = np.ascontiguousarray(blocks_ids, dtype=np.intc)
    i0, i1 = (0, N) if i_range is None else i_range
    rc = lib.oracle_perturb_average_sym(_dptr(X), _dptr(Y), _dptr(w), _dptr(rho), _dptr(R1), _dptr(Y1),
                                        float(T), int(apply_d4), N, n, N_sym, len(n_deg), _iptr(n_deg),
                                        _iptr(deg_flat), _dptr(sym_flat), _iptr(bid), int(i0), int(i1),
                                        int(n_threads), _dptr(f_out), _dptr(d_out))
    if rc != 0:
        raise ValueError(f"oracle_perturb_average_sym failed with code {rc}")
    return f_out, d_out


_POOL_DATA = {}


def _pool_init(data):
    _POOL_DATA.clear()
    _POOL_DATA.update(data)


def _pool_slice(args):
    """Averages of one slice of (configuration, symmetry) pairs, scaled back to a partial sum (x the
    slice's N_eff x its number of symmetries): what each MPI rank contributes to the reference's
    MPI_Allreduce (LanczosFunctions.c:2123-2136, 2236-2248)."""
    i0, i1, sym0, sym1, R1, Y1, apply_d4 = args
    d = _POOL_DATA
    syms = d["syms"] if sym0 is None else [s[sym0:sym1] for s in d["syms"]]
    f, dv = perturb_average_sym(d["X"][i0:i1], d["Y"][i0:i1], d["w"], d["rho"][i0:i1], R1, Y1, d["T"], apply_d4, syms,
                                d["n_deg"], d["degs"], d["bid"], backend=d["backend"], n_threads=1)
    scale = float(np.sum(d["rho"][i0:i1])) * int(syms[0].shape[0])
    return f * scale, dv * scale


class SlicedAverages:
    """The averages of the whole ensemble from P worker processes (``spawn``: safe after a CUDA
    context exists; callers' scripts need an ``if __name__ == "__main__"`` guard), each running the
    C kernel on a contiguous slice of the configurations -- the reference's MPI partition and
    Allreduce (LanczosFunctions.c:2123-2136, 2236-2248) on the host cores.  With fewer
    configurations than processes the symmetry group is sliced too (the averages are plain sums
    over (configuration, symmetry) pairs divided by N_eff * N_sym).  Use as a context manager."""

    def __init__(self, X, Y, w, rho, T, symmetries, n_deg, deg_space, blocks_ids, backend="reference", procs=None):
        import multiprocessing as mp
        self.N = X.shape[0]
        self.N_sym = int(symmetries[0].shape[0])
        self.rho = np.asarray(rho, dtype=np.float64)
        self.procs = max(1, procs or (os.cpu_count() or 1))
        data = dict(X=np.ascontiguousarray(X, dtype=np.float64), Y=np.ascontiguousarray(Y, dtype=np.float64),
                    w=np.ascontiguousarray(w, dtype=np.float64), rho=self.rho, T=float(T),
                    syms=[np.ascontiguousarray(s, dtype=np.float64) for s in symmetries],
                    n_deg=np.ascontiguousarray(n_deg, dtype=np.intc),
                    degs=[np.ascontiguousarray(d_, dtype=np.intc) for d_ in deg_space],
                    bid=np.ascontiguousarray(blocks_ids, dtype=np.intc), backend=backend)
        if self.N >= self.procs:
            edges = np.linspace(0, self.N, self.procs + 1).round().astype(int)
            self.tasks = [(int(a), int(b), None, None) for a, b in zip(edges[:-1], edges[1:]) if b > a]
        else:
            per = max(1, -(-self.procs // self.N))
            sedges = np.linspace(0, self.N_sym, per + 1).round().astype(int)
            self.tasks = [(i, i + 1, int(a), int(b)) for i in range(self.N)
                          for a, b in zip(sedges[:-1], sedges[1:]) if b > a]
        self._pool = mp.get_context("spawn").Pool(self.procs, initializer=_pool_init, initargs=(data,))

    def __call__(self, R1, Y1, apply_d4):
        R1 = np.ascontiguousarray(R1, dtype=np.float64)
        Y1 = np.ascontiguousarray(Y1, dtype=np.float64)
        parts = self._pool.map(_pool_slice, [t + (R1, Y1, int(apply_d4)) for t in self.tasks], chunksize=1)
        norm = float(np.sum(self.rho)) * self.N_sym
        f = sum(p[0] for p in parts) / norm
        dv = sum(p[1] for p in parts) / norm
        return f, dv

    def close(self):
        self._pool.close()
        self._pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False


# ----------------------------------------------------------------------------------------------
# helpers on the packed (R | Y-triangle | A-triangle) vector
# ----------------------------------------------------------------------------------------------
def bose(w, T):
    if T > 0:
        return 1.0 / (np.exp(w * RY_TO_K / T) - 1.0)
    return np.zeros_like(w)


def upper_pairs(n):
    """(row, col) with col >= row, row-major: the packing of get_Y1 (DynamicalLanczos.py:2840-2848)."""
    r, c = np.triu_indices(n)
    return r, c


def unpack_sym(packed, n, half_off_diagonal=False):
    r, c = upper_pairs(n)
    M = np.zeros((n, n), dtype=np.float64)
    M[r, c] = packed
    M[c, r] = packed
    if half_off_diagonal:
        mask = np.full((n, n), 0.5)
        np.fill_diagonal(mask, 1.0)
        M *= mask
    return M


def pack_upper(M):
    r, c = upper_pairs(M.shape[0])
    return M[r, c].copy()


# ----------------------------------------------------------------------------------------------
# the oracle Lanczos
# ----------------------------------------------------------------------------------------------
class OracleLanczos:
    """numpy restatement of the reference ``Lanczos`` object's hot-path methods."""

    def __init__(self, X, Y, w, rho, T, symmetries=None, deg_space=None, blocks_ids=None,
                 backend="port", n_threads=0):
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.Y = np.ascontiguousarray(Y, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.T = float(T)
        self.N, self.n_modes = self.X.shape
        n = self.n_modes
        if symmetries is None:     # prepare_symmetrization(no_sym=True), DynamicalLanczos.py:719-724
            symmetries = [np.ones((1, 1, 1))] * n
            deg_space = [np.array([i], dtype=np.intc) for i in range(n)]
            blocks_ids = np.arange(n, dtype=np.intc)
        self.symmetries = [np.asarray(s, dtype=np.float64) for s in symmetries]
        self.degenerate_space = [np.asarray(d, dtype=np.intc) for d in deg_space]
        self.N_degeneracy = np.array([len(d) for d in self.degenerate_space], dtype=np.intc)
        self.sym_block_id = np.asarray(blocks_ids, dtype=np.intc)
        self.backend = backend
        self.n_threads = n_threads
        self.ignore_harmonic = False
        self.ignore_v3 = False
        self.ignore_v4 = False
        self.use_wigner = False
        self.reverse_L = False
        self.shift_value = 0.0
        self.perturbation_modulus = 1.0
        self.psi = np.zeros(n + n * (n + 1), dtype=np.float64)
        self.reset()

    def reset(self):
        n = self.n_modes
        self.psi = np.zeros(n + n * (n + 1), dtype=np.float64)
        self.a_coeffs, self.b_coeffs, self.c_coeffs = [], [], []
        self.basis_Q, self.basis_P, self.s_norm = [], [], []

    # ---- perturbations (DynamicalLanczos.py:1963-2031) ----
    def prepare_mode(self, index):
        self.reset()
        self.psi[:] = 0
        self.psi[index] = 1
        self.perturbation_modulus = 1

    def prepare_perturbation_modes(self, v_modes, add=False):
        """prepare_perturbation after the projection on the polarisation vectors: psi[:n] += v."""
        if not add:
            self.reset()
        self.psi[: self.n_modes] += v_modes
        self.perturbation_modulus = float(v_modes.dot(v_modes))

    # ---- harmonic part (DynamicalLanczos.py:2227-2385) ----
    def apply_L1_FT(self, transpose=False):
        n = self.n_modes
        out = np.zeros_like(self.psi)
        if self.ignore_harmonic:
            return out
        r, c = upper_pairs(n)
        w_a, w_b = self.w[c], self.w[r]
        if not self.use_wigner:
            out[:n] = (self.psi[:n] * self.w) * self.w
        else:
            out[:n] = -(self.psi[:n] * self.w) * self.w
        if self.T > 0:
            n_a = 1 / (np.exp(w_a / np.double(self.T / RY_TO_K)) - 1)
            n_b = 1 / (np.exp(w_b / np.double(self.T / RY_TO_K)) - 1)
        else:
            n_a = np.zeros_like(w_a)
            n_b = np.zeros_like(w_a)
        sY, sA = n, n + len(w_a)
        pY, pA = self.psi[sY:sA], self.psi[sA:]
        if not self.use_wigner:
            den = (2 * n_a + 1) * (2 * n_b + 1)
            X_ab = -w_a ** 2 - w_b ** 2 - (2 * w_a * w_b) / den
            out[sY:sA] = -X_ab * pY
            Y_ab = -(8 * w_a * w_b) / den
            if not transpose:
                out[sY:sA] += -Y_ab * pA
            else:
                out[sA:] += -Y_ab * pY
            X1_ab = -(2 * n_a * n_b + n_a + n_b) * (2 * n_a * n_b + n_a + n_b + 1) * (2 * w_a * w_b) / den
            if not transpose:
                out[sA:] += -X1_ab * pY
            else:
                out[sY:sA] += -X1_ab * pA
            Y1_ab = -w_a ** 2 - w_b ** 2 + (2 * w_a * w_b) / den
            out[sA:] += -Y1_ab * pA
        else:
            out[sY:sA] = -(w_a ** 2 + w_b ** 2 - 2 * w_a * w_b) * pY
            out[sA:] = -(w_a ** 2 + w_b ** 2 + 2 * w_a * w_b) * pA
        return out

    # ---- packed-vector views (DynamicalLanczos.py:2827-2888) ----
    def get_Y1(self, half_off_diagonal=False):
        n = self.n_modes
        return unpack_sym(self.psi[n: n + n * (n + 1) // 2], n, half_off_diagonal)

    def get_ReA1(self, half_off_diagonal=False):
        n = self.n_modes
        return unpack_sym(self.psi[n + n * (n + 1) // 2:], n, half_off_diagonal)

    # ---- Wigner helpers (DynamicalLanczos.py:2572-2627, 2713-2822) ----
    def _bose_matrix(self):
        n = self.n_modes
        w = np.tile(self.w, (n, 1))
        nn = np.zeros((n, n))
        if self.T > EPSILON:
            nn = 1.0 / (np.exp(w * RY_TO_K / self.T) - 1.0)
        return w, nn

    def get_chi_minus(self):
        w, nn = self._bose_matrix()
        return (w - w.T) * (nn - nn.T) / (2. * w * w.T)

    def get_chi_plus(self):
        w, nn = self._bose_matrix()
        return (w + w.T) * (1 + nn + nn.T) / (2. * w * w.T)

    def get_alpha1_beta1_wigner(self, get_alpha=True):
        n = self.n_modes
        sa, sb = n, n + n * (n + 1) // 2
        a_all, b_all = self.psi[sa:sb], self.psi[sb:]
        r, c = upper_pairs(n)
        w_a, w_b = self.w[c], self.w[r]
        if self.T > 0:
            n_a = 1 / (np.exp(w_a / np.double(self.T / RY_TO_K)) - 1)
            n_b = 1 / (np.exp(w_b / np.double(self.T / RY_TO_K)) - 1)
        else:
            n_a = np.zeros_like(w_a)
            n_b = np.zeros_like(w_a)
        Xf = (1 + 2 * n_a) * (1 + 2 * n_b) / 8
        w2_on_X = (w_a * w_b) / Xf
        chi_m = ((w_a - w_b) * (n_a - n_b)) / (2 * w_a * w_b)
        chi_p = ((w_a + w_b) * (1 + n_a + n_b)) / (2 * w_a * w_b)
        if get_alpha:
            new = w2_on_X * np.sqrt(-0.5 * chi_m) * a_all - w2_on_X * np.sqrt(0.5 * chi_p) * b_all
        else:
            new = (np.sqrt(-0.5 * chi_m) / Xf) * a_all + (np.sqrt(0.5 * chi_p) / Xf) * b_all
        return unpack_sym(new, n)

    # ---- the averages (odd_corr_module.c:491-634) ----
    def averages(self, R1, Y1, apply_d4):
        return perturb_average_sym(self.X, self.Y, self.w, self.rho, R1, Y1, self.T, apply_d4,
                                   self.symmetries, self.N_degeneracy, self.degenerate_space,
                                   self.sym_block_id, backend=self.backend, n_threads=self.n_threads)

    # ---- static operator of the free-energy Hessian (DynamicalLanczos.py:2502-2565, 3287-3354) ----
    def apply_L1_static(self, psi, inverse=False, power=1):
        """apply_L1_static: w^(2 power) on R, 1/Lambda^power on the packed Upsilon, with the
        reference's quirks (both Bose factors masked by w_a; the equal-frequency branch multiplies
        by an all-zero array taken before the factors are filled)."""
        n = self.n_modes
        assert len(psi) == n + n * (n + 1) // 2
        out = np.zeros(psi.shape, dtype=np.float64)
        if inverse:
            power *= -1
        out[:n] = psi[:n] * (self.w ** (2 * power))
        b, a = upper_pairs(n)                  # i_b = row, i_a = col >= row
        w_a, w_b = self.w[a], self.w[b]
        n_a = np.zeros(w_a.shape)
        n_b = np.zeros(w_a.shape)
        mask_a = 0.01 * w_a * RY_TO_K > self.T
        mask_b = 0.01 * w_a * RY_TO_K > self.T
        diff = np.zeros(w_a.shape)
        equal = np.abs(w_a - w_b) < 1e-8
        w_equal = w_a[equal]
        n_equal = n_a[equal]
        if self.T > 0:
            beta = RY_TO_K / self.T
            with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
                n_a = 1 / (np.exp(w_a * beta) - 1)
                n_b = 1 / (np.exp(w_b * beta) - 1)
                n_a[mask_a] = 0
                n_b[mask_b] = 0
                diff[:] = (n_a - n_b) / (w_a - w_b)
                diff[equal] = -beta * np.exp(w_equal * beta) * n_equal ** 2
        lam = (n_a + n_b + 1) / (w_a + w_b) - diff
        lam /= 4 * w_a * w_b
        out[n:] = psi[n:] / lam ** power
        return out

    def apply_anharmonic_static(self):
        """apply_anharmonic_static on the static vector self.psi = (R, packed Upsilon)."""
        n = self.n_modes
        Y1 = unpack_sym(self.psi[n:n + n * (n + 1) // 2], n)
        R1 = self.psi[:n].copy()
        n_mu = bose(self.w, self.T) if self.T > 1e-12 else np.zeros(n)
        Y_w = 2 * self.w / (2 * n_mu + 1)
        Y1 = -2 * np.einsum("ab, a, b -> ab", Y1, Y_w, Y_w)
        f, d = self.averages(R1, Y1, 0 if self.ignore_v4 else 1)
        out = np.zeros(self.psi.shape, dtype=np.float64)
        out[:n] = -f
        out[n:] = pack_upper(d)
        return out

    def apply_static_L(self, psi, eigen_shift=1.0):
        """The matvec of run_hessian_calculation (DynamicalLanczos.py:4041-4051)."""
        n = self.n_modes
        self.psi = psi.copy()
        self.psi[n:] *= eigen_shift
        ret = self.apply_L1_static(self.psi)
        ret += self.apply_anharmonic_static()
        ret[n:] *= eigen_shift
        return ret

    def static_green_function(self, eigen_shift=1, max_iters=1000, use_preconditioning=True):
        """The rows of the one-phonon static Green function of run_hessian_calculation with
        algorithm "cg" (DynamicalLanczos.py:3973-4218): one minimum-residual solve per mode."""
        n = self.n_modes
        ln = n + n * (n + 1) // 2
        A = lambda x: self.apply_static_L(x, eigen_shift)                         # noqa: E731
        M = lambda x: self.apply_L1_static(x, inverse=True, power=0.5)             # noqa: E731
        G = np.zeros((n, n))
        for i in range(n):
            b = np.zeros(ln)
            b[i] = 1
            if not use_preconditioning:
                res = minimum_residual_algorithm(A, b.copy(), b.copy(), max_iters=max_iters)
            else:
                res = minimum_residual_algorithm_precond(A, b.copy(), M, max_iters=max_iters)
            G[i, :] = res[:n]
        return G

    # ---- anharmonic part (DynamicalLanczos.py:2891-3281) ----
    def apply_anharmonic_FT(self, transpose=False):
        n = self.n_modes
        R1 = self.psi[:n].copy()
        if not self.use_wigner:
            Y1 = self.get_Y1(half_off_diagonal=transpose)
            n_mu = 0
            if self.T > EPSILON:
                n_mu = 1.0 / (np.exp(self.w * RY_TO_K / self.T) - 1.0)
            Y_w = 2 * self.w / (2 * n_mu + 1)
            ReA_w = 2 * self.w * n_mu * (n_mu + 1) / (2 * n_mu + 1)
            if transpose:
                ReA1 = self.get_ReA1(half_off_diagonal=True)
                coeff_Y = 2 * (np.einsum("a,b,b->ab", Y_w, Y_w, Y_w) + np.einsum("a,a,b->ab", Y_w, Y_w, Y_w))
                coeff_RA = 2 * (np.einsum("a,b,b->ab", Y_w, ReA_w, Y_w) + np.einsum("a,a,b->ab", Y_w, ReA_w, Y_w))
                Y1 = Y1 * coeff_Y + ReA1 * coeff_RA
        else:
            Y1 = self.get_alpha1_beta1_wigner(get_alpha=True)
            chi_minus = self.get_chi_minus()
            chi_plus = self.get_chi_plus()
        apply_d4 = 0 if self.ignore_v4 else 1
        if self.ignore_v3:
            R1[:] = 0.0
        f_av, d2v = self.averages(R1, Y1, apply_d4)
        out = np.zeros_like(self.psi)
        out[:n] = f_av
        if not self.use_wigner:
            if not transpose:
                pert_Y = d2v * Y_w[:, None] + d2v * Y_w[None, :]
                pert_RA = d2v * ReA_w[:, None] + d2v * ReA_w[None, :]
            else:
                Y_inv = 1 / Y_w
                pert_Y = 0.5 * Y_inv[:, None] * d2v * Y_inv[None, :]
                pert_RA = np.zeros_like(pert_Y)
                sym_mask = np.full(pert_Y.shape, 2.0)
                np.fill_diagonal(sym_mask, 1.0)
                pert_Y = pert_Y * sym_mask
                pert_RA = pert_RA * sym_mask
        else:
            pert_Y = np.sqrt(-0.5 * chi_minus) * d2v
            pert_RA = -np.sqrt(0.5 * chi_plus) * d2v
        r, c = upper_pairs(n)
        m = n * (n + 1) // 2
        out[n: n + m] = pert_Y[r, c]
        out[n + m:] = pert_RA[r, c]
        return -out if not self.use_wigner else out

    # ---- full apply (DynamicalLanczos.py:3467-3570) ----
    def apply_full_L(self, target=None, transpose=False):
        if target is not None:
            self.psi = np.array(target, dtype=np.float64, copy=True)
        out = self.apply_L1_FT(transpose)
        if not self.ignore_v3:
            out = out + self.apply_anharmonic_FT(transpose)
        if self.reverse_L:
            out *= -1
        out += self.shift_value * self.psi
        self.psi = out
        return out

    # ---- mask for the symmetric Wigner Lanczos (DynamicalLanczos.py:5790-5839) ----
    def mask_dot_wigner(self):
        n = self.n_modes
        mask = np.ones(n + n * (n + 1))
        r, c = upper_pairs(n)
        m = n * (n + 1) // 2
        off = r < c
        mask[n: n + m][off] = 2
        mask[n + m:][off] = 2
        return mask

    # ---- bi-conjugate Lanczos (DynamicalLanczos.py:5843-6374) ----
    def run_FT(self, n_iter, run_simm=False, step_callback=None, n_rep_orth=0, n_ortho=10):
        psi_norm = np.sum(self.psi ** 2)
        if np.isnan(psi_norm) or psi_norm == 0:
            raise ValueError("initialise a perturbation before running")
        if run_simm and not self.use_wigner:
            raise NotImplementedError("the symmetric Lanczos works only with Wigner")
        mask = self.mask_dot_wigner() if run_simm else None

        def dot(a, b):
            return a.dot(b) if mask is None else a.dot(b * mask)

        i_step = len(self.a_coeffs)
        if i_step == 0:
            first = self.psi / np.sqrt(dot(self.psi, self.psi))
            self.basis_Q, self.basis_P, self.s_norm = [first], [first], [1]
        psi_q, psi_p = self.basis_Q[-1], self.basis_P[-1]
        next_converged = False
        for _ in range(i_step, i_step + n_iter):
            L_q = self.apply_full_L(psi_q, transpose=False)
            if self.use_wigner and run_simm:
                p_L = np.copy(L_q)
            else:
                p_L = self.apply_full_L(psi_p, transpose=True)
            c_old = self.c_coeffs[-1] if len(self.c_coeffs) > 0 else 1
            p_norm = self.s_norm[-1] / c_old
            a_coeff = dot(psi_p, L_q) * p_norm
            if np.isnan(a_coeff):
                raise ValueError("invalid value encountered during the Lanczos")
            rk = L_q - a_coeff * psi_q
            if len(self.basis_Q) > 1:
                rk -= self.c_coeffs[-1] * self.basis_Q[-2]
            sk = p_L - a_coeff * psi_p
            if len(self.basis_P) > 1:
                old_p_norm = self.s_norm[-2] if len(self.c_coeffs) < 2 else self.s_norm[-2] / self.c_coeffs[-2]
                sk -= self.b_coeffs[-1] * self.basis_P[-2] * (old_p_norm / p_norm)
            s_norm = np.sqrt(dot(sk, sk))
            sk_tilde = sk / s_norm
            s_norm *= p_norm
            b_coeff = np.sqrt(dot(rk, rk))
            c_coeff = dot(sk_tilde, rk / b_coeff) * s_norm
            self.a_coeffs.append(a_coeff)
            if np.abs(b_coeff) < EPSILON or np.abs(c_coeff) < EPSILON or next_converged:
                break
            psi_q = rk / b_coeff
            psi_p = sk_tilde.copy()
            if n_rep_orth > 0:
                psi_q, psi_p, s_gs, conv = gram_schmidt(psi_q, psi_p, self.basis_Q, self.basis_P, n_rep_orth, n_ortho,
                                                        c_coeff, dot)
                next_converged = next_converged or conv
                if s_gs is not None:
                    s_norm = s_gs
            self.basis_Q.append(psi_q.copy())
            self.basis_P.append(psi_p.copy())
            self.b_coeffs.append(b_coeff)
            self.c_coeffs.append(c_coeff)
            self.s_norm.append(s_norm)
            if step_callback is not None:
                step_callback(self)

    # ---- continued fraction (DynamicalLanczos.py:4951-5047) ----
    def get_green_function_continued_fraction(self, w_array, use_terminator=True, last_average=1, smearing=0.0):
        w_array = np.asarray(w_array, dtype=np.float64)
        n_iters = len(self.a_coeffs)
        sign = -1 if self.reverse_L else 1
        if use_terminator:
            a_av = np.mean(self.a_coeffs[-last_average:])
            b_av = np.mean(self.b_coeffs[-last_average:])
            c_av = b_av
            if len(self.c_coeffs) == len(self.b_coeffs):
                c_av = np.mean(self.c_coeffs[-last_average:])
            a = a_av * sign - sign * self.shift_value
            b = b_av * sign
            c = c_av * sign
            if not self.use_wigner:
                gf = (a - w_array ** 2 - np.sqrt((a - w_array ** 2) ** 2 - 4 * b * c + 0j)) / (2 * b * c)
            else:
                gf = (a + w_array ** 2 + np.sqrt((a + w_array ** 2) ** 2 - 4 * b * c + 0j)) / (2 * b * c)
        else:
            a = self.a_coeffs[-1] * sign - sign * self.shift_value
            if not self.use_wigner:
                gf = 1 / (a - w_array ** 2 + 2j * w_array * smearing)
            else:
                gf = 1 / (a + w_array ** 2 + 2j * w_array * smearing)
        for i in range(n_iters - 2, -1, -1):
            a = self.a_coeffs[i] * sign - sign * self.shift_value
            b = self.b_coeffs[i] * sign
            c = b
            if len(self.c_coeffs) == len(self.b_coeffs):
                c = self.c_coeffs[i] * sign
            if not self.use_wigner:
                gf = 1. / (a - w_array ** 2 + 2j * w_array * smearing - b * c * gf)
            else:
                gf = 1. / (a + w_array ** 2 + 2j * w_array * smearing - b * c * gf)
        if not self.use_wigner:
            return gf * self.perturbation_modulus
        return (-np.real(gf) + 1j * np.imag(gf)) * self.perturbation_modulus


def gram_schmidt(new_q, new_p, basis_Q, basis_P, n_rep_orth, n_ortho, c_coeff, dot):
    """Gram-Schmidt of the new Lanczos pair against the last n_ortho basis pairs
    (DynamicalLanczos.py:6244-6316), with the reference's own conventions: sequential updates, q
    normalised by its norm, p by its squared norm, s_norm re-derived from p . q, and the stop test on
    the q coefficients only (its p accumulator adds |0| to itself).  Returns (q, p, s_norm or None,
    next_converged)."""
    new_q, new_p = np.array(new_q, copy=True), np.array(new_p, copy=True)
    s_norm = None
    next_converged = False
    for _rep in range(n_rep_orth):
        ortho_q = 0.0
        start = max(0, len(basis_P) - n_ortho) if n_ortho is not None else 0
        for j in range(start, len(basis_P)):
            coeff1 = dot(basis_P[j], new_q)
            coeff2 = dot(basis_Q[j], new_p)
            new_q = new_q - coeff1 * basis_P[j]
            new_p = new_p - coeff2 * basis_Q[j]
            ortho_q += np.abs(coeff1)
        normq = np.sqrt(dot(new_q, new_q))
        if normq < EPSILON:
            next_converged = True
        new_q = new_q / normq
        normp = dot(new_p, new_p)
        if np.abs(normp) < EPSILON:
            next_converged = True
        new_p = new_p / normp
        s_norm = c_coeff / dot(new_p, new_q)
        if ortho_q < EPSILON:
            break
    return new_q, new_p, s_norm, next_converged


# ----------------------------------------------------------------------------------------------
# the reference's minimum residual solver (Modules/Tools.py:265-471), on plain callables
# ----------------------------------------------------------------------------------------------
def minimum_residual_algorithm(A, b, x0, max_iters=100, conv_thr=1e-6, callback=None):
    """Tools.minimum_residual_algorithm with precond = None (the only form its callers use)."""
    r1 = b - A(x0)
    b_prec = b.copy()
    r1_bar = A(r1)
    z1 = r1.copy()
    p1 = r1.copy()
    p1_bar = r1_bar.copy()
    x = x0.copy()
    iters = 1
    converged = False
    while iters < max_iters and not converged:
        Ap = p1_bar
        Ap_bar = A(p1_bar)
        alpha = r1_bar.dot(z1) / (p1_bar.dot(Ap))
        x[:] += alpha * p1
        if callback is not None:
            callback(x, iters)
        r = r1 - alpha * Ap
        rbar = r1_bar - alpha * Ap_bar
        r_norm = np.sqrt(r.dot(r)) / np.sqrt(b_prec.dot(b_prec))
        z = r.copy()
        zbar = rbar.copy()
        beta = rbar.dot(z) / (r1_bar.dot(z1))
        p1[:] = z + beta * p1
        p1_bar[:] = zbar + beta * p1_bar
        r1[:] = r
        r1_bar[:] = rbar
        z1[:] = z
        converged = r_norm < conv_thr
        iters += 1
    return x


def minimum_residual_algorithm_precond(A, b, precond_half, x0=None, **kwargs):
    """Tools.minimum_residual_algorithm_precond: the solve of M A M x~ = M b, x = M x~."""
    A_tilde = lambda x: precond_half(A(precond_half(x)))     # noqa: E731
    b_tilde = precond_half(b)
    if x0 is None:
        x0 = b_tilde.copy()
    x_tilde = minimum_residual_algorithm(A_tilde, b_tilde, x0, **kwargs)
    return precond_half(x_tilde)


# ----------------------------------------------------------------------------------------------
# StaticHessian's system matrix (Modules/StaticHessian.py:561-690), plain loops, small n only
# ----------------------------------------------------------------------------------------------
def static_hessian_get_G_W(vector, n, ignore_W=False):
    G = np.zeros((n, n))
    counter = 0
    for i in range(n):
        for j in range(i, n):
            G[i, j] = vector[counter]
            G[j, i] = vector[counter]
            counter += 1
    if ignore_W:
        return G
    W = np.zeros((n, n, n))
    for i in range(n):
        for j in range(i, n):
            for k in range(j, n):
                v = vector[counter]
                W[i, j, k] = W[i, k, j] = W[j, i, k] = W[j, k, i] = W[k, i, j] = W[k, j, i] = v
                counter += 1
    return G, W


def static_hessian_get_vector(G, W):
    n = G.shape[0]
    out = []
    for i in range(n):
        for j in range(i, n):
            out.append(G[i, j])
    for i in range(n):
        for j in range(i, n):
            for k in range(j, n):
                out.append(W[i, j, k])
    return np.array(out)


def static_hessian_apply_L(oracle, vect, preconditioner=False, inverse_preconditioner=False):
    """StaticHessian.apply_L: the static L on each row (G^-1[i, :], W[i] packed)."""
    n = oracle.n_modes
    Ginv, W = static_hessian_get_G_W(vect, n)
    for i in range(n):
        vector = np.zeros(n + n * (n + 1) // 2)
        vector[:n] = Ginv[i, :]
        vector[n:] = pack_upper(W[i])
        oracle.psi = vector
        if not preconditioner and not inverse_preconditioner:
            outv = oracle.apply_L1_static(vector)
            outv += oracle.apply_anharmonic_static()
        else:
            power = 0.5 if preconditioner else -0.5
            outv = oracle.apply_L1_static(vector, inverse=True, power=power)
        Ginv[i, :] = outv[:n]
        W[i] = unpack_sym(outv[n:], n)
    return static_hessian_get_vector(Ginv, W)


# ----------------------------------------------------------------------------------------------
# the reference's analytic L operator from explicit d3 / d4 tensors (DynamicalLanczos.py:5454-5789)
# ----------------------------------------------------------------------------------------------
def explicit_L_operator_FT(o, debug_d3=None):
    """get_full_L_operator_FT(symmetrize=False) of the reference, with its full n^3 / n^4 einsums
    (small n only).  `o` carries X, Y, rho, w, T, n_modes and the flags use_wigner,
    ignore_harmonic, ignore_v3, ignore_v4."""
    n = o.n_modes
    i_a = np.tile(np.arange(n), (n, 1)).ravel()
    i_b = np.tile(np.arange(n), (n, 1)).T.ravel()
    new_i_a = np.array([i_a[i] for i in range(len(i_a)) if i_a[i] >= i_b[i]])
    new_i_b = np.array([i_b[i] for i in range(len(i_a)) if i_a[i] >= i_b[i]])
    w_a, w_b = o.w[new_i_a], o.w[new_i_b]
    N_w2 = len(w_a)
    L = np.zeros((n + 2 * N_w2, n + 2 * N_w2))
    if not o.ignore_harmonic:
        L[:n, :n] = np.diag(o.w ** 2) if not o.use_wigner else -np.diag(o.w ** 2)
    n_a = np.zeros(w_a.shape)
    n_b = np.zeros(w_a.shape)
    if o.T > 0:
        n_a = 1 / (np.exp(w_a * 157887.32400374097 / o.T) - 1)
        n_b = 1 / (np.exp(w_b * 157887.32400374097 / o.T) - 1)
    sY, sA = n, n + N_w2
    if not o.ignore_harmonic:
        if not o.use_wigner:
            L[sY:sA, sY:sA] = -np.diag(-w_a ** 2 - w_b ** 2 - (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1)))
            L[sY:sA, sA:] = -np.diag(-(8 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1)))
            L[sA:, sY:sA] = -np.diag(-(2 * n_a * n_b + n_a + n_b) * (2 * n_a * n_b + n_a + n_b + 1) * (2 * w_a * w_b)
                                     / ((2 * n_a + 1) * (2 * n_b + 1)))
            L[sA:, sA:] = -np.diag(-w_a ** 2 - w_b ** 2 + (2 * w_a * w_b) / ((2 * n_a + 1) * (2 * n_b + 1)))
        else:
            L[sY:sA, sY:sA] = np.diag(-(w_a ** 2 + w_b ** 2 - 2 * w_a * w_b))
            L[sA:, sA:] = np.diag(-(w_a ** 2 + w_b ** 2 + 2. * w_a * w_b))
    N_eff = np.sum(o.rho)
    Y_weighted = np.einsum("ia, i -> ia", o.Y, o.rho)
    n_w = bose(o.w, o.T)
    X_ups = np.einsum("ia, a -> ia", o.X, 2 * o.w / (1 + 2 * n_w))
    ec = np.ones(N_w2)
    ec[new_i_a != new_i_b] = 2
    if not o.ignore_v3:
        if debug_d3 is not None:
            d3 = debug_d3
        else:
            d3n = np.einsum("ia, ib, ic -> abc", X_ups, X_ups, Y_weighted) / -N_eff
            d3 = (d3n + np.einsum("abc->acb", d3n) + np.einsum("abc->bac", d3n) + np.einsum("abc->bca", d3n)
                  + np.einsum("abc->cab", d3n) + np.einsum("abc->cba", d3n)) / 6
        d3s = d3[new_i_a, new_i_b, :]
        if not o.use_wigner:
            L[sY:sA, :sY] = -np.einsum("ab, a -> ab", d3s, 2 * ((2 * n_a + 1) * w_b + (2 * n_b + 1) * w_a)
                                       / ((2 * n_a + 1) * (2 * n_b + 1)))
            L[sA:, :sY] = -np.einsum("ab, a -> ab", d3s, 2 * ((2 * n_a + 1) * w_b * n_b * (n_b + 1) + (2 * n_b + 1) * w_a
                                                             * n_a * (n_a + 1)) / ((2 * n_a + 1) * (2 * n_b + 1)))
            L[:sY, sY:sA] = -np.einsum("ab, a -> ba", d3s, (2 * n_b + 1) * (2 * n_a + 1) / (8 * w_a * w_b) * ec)
        else:
            chi_minus = (n_a - n_b) * (w_a - w_b) / (2 * w_a * w_b)
            chi_plus = (1 + n_a + n_b) * (w_a + w_b) / (2 * w_a * w_b)
            L[:sY, sY:sA] = np.einsum("ab, a -> ab", d3s, np.sqrt(-0.5 * chi_minus) * ec).T
            L[:sY, sA:] = -np.einsum("ab, a -> ab", d3s, np.sqrt(0.5 * chi_plus) * ec).T
            L[sY:sA, :sY] = np.einsum("ab, a -> ab", d3s, np.sqrt(-0.5 * chi_minus))
            L[sA:, :sY] = -np.einsum("ab, a -> ab", d3s, np.sqrt(0.5 * chi_plus))
    if not o.ignore_v4:
        d4 = np.einsum("ia, ib, ic, id -> abcd", X_ups, X_ups, X_ups, Y_weighted)
        d4 += np.einsum("ia, ib, ic, id -> abcd", X_ups, X_ups, Y_weighted, X_ups)
        d4 += np.einsum("ia, ib, ic, id -> abcd", X_ups, Y_weighted, X_ups, X_ups)
        d4 += np.einsum("ia, ib, ic, id -> abcd", Y_weighted, X_ups, X_ups, X_ups)
        d4 /= -4 * N_eff
        d4s = d4[new_i_a, new_i_b, :, :][:, new_i_a, new_i_b]
        if not o.use_wigner:
            left = -(2 * w_a * n_b + 2 * w_b * n_a + w_a + w_b) / (4 * (2 * n_a + 1) * (2 * n_b + 1))
            right = (2 * n_a + 1) * (2 * n_b + 1) / (w_a * w_b)
            L[sY:sA, sY:sA] += -np.einsum("a, ab, b -> ab", left, d4s, right * ec)
            left1 = -(w_a * n_a * (n_a + 1) * (2 * n_b + 1) + w_b * n_b * (n_b + 1) * (2 * n_a + 1)) / (
                4 * (2 * n_a + 1) * (2 * n_b + 1))
            L[sA:, sY:sA] += -np.einsum("a, ab, b -> ab", left1, d4s, right * ec)
        else:
            chi_plus = (1 + n_a + n_b) * (w_a + w_b) / (2 * w_a * w_b)
            chi_minus = (n_a - n_b) * (w_a - w_b) / (2 * w_a * w_b)
            sp, sm = np.sqrt(0.5 * chi_plus), np.sqrt(-0.5 * chi_minus)
            L[sY:sA, sY:sA] += -np.einsum("a, ab, b -> ab", sm, d4s, sm * ec)
            L[sA:, sA:] += -np.einsum("a, ab, b -> ab", sp, d4s, sp * ec)
            L[sY:sA, sA:] += np.einsum("a, ab, b -> ab", sm, d4s, sp * ec)
            L[sA:, sY:sA] += np.einsum("a, ab, b -> ab", sp, d4s, sm * ec)
    return L
