"""The free-energy Hessian from the static L operator (the reference's tdscha.StaticHessian,
Modules/StaticHessian.py), on the B200 device path.

The state is the vector (G^-1 packed upper, W packed i <= j <= k) of length
n(n+1)/2 + n(n+1)(n+2)/6.  One application of the system matrix (apply_L, :561-623) applies the
static L to the n row vectors (G^-1[i, :], W[i, :, :] packed): here as one batched device apply
of all n rows (tdscha_apply_static_L_device, 64 rows per averages call), with the row vectors
gathered from and scattered back to the packed state by index maps instead of the reference's
n^3 loops.  run (:184-287) is the reference's minimum-residual solve ("cg", "cg-prec") on the
device; run_no_mode_mixing (:403-509) runs the non-degenerate modes' chains together
(run_FT_batched) and takes G(0).  retrieve_hessian returns the supercell matrix (noq=True); the
cellconstructor Phonons object of noq=False is not available in this package.
"""
from __future__ import annotations

import difflib
import json
import os
import sys
import time

import numpy as np

from . import DynamicalLanczos as DL


def _torch():
    return DL._torch()


def _pair_index(n):
    """P[i, j] = packed index of (min, max) in the row-major upper triangle."""
    r, c = np.triu_indices(n)
    P = np.zeros((n, n), dtype=np.int64)
    P[r, c] = np.arange(len(r))
    P[c, r] = P[r, c]
    return P


def _triple_offsets(n):
    """Packed index of (i <= j <= k) in get_vector's order (i outer, then j, then k)."""
    # count of triples with first index < i: sum_{a<i} (n-a)(n-a+1)/2
    a = np.arange(n)
    per_i = (n - a) * (n - a + 1) // 2
    start_i = np.concatenate([[0], np.cumsum(per_i)[:-1]])
    return start_i


def _triple_index(i, j, k, n, start_i):
    """Index of the sorted triple i <= j <= k (arrays) among the packed W entries."""
    # within block i: pairs (j, k) with i <= j <= k, row-major upper triangle of the (n-i) x (n-i) block
    m = n - i
    jj = j - i
    kk = k - i
    return start_i[i] + jj * m - jj * (jj - 1) // 2 + (kk - jj)


def row_maps(n):
    """Index maps between the packed state (G packed upper, W packed i <= j <= k) and the n row
    vectors (G[i, :], W[i] packed upper) of apply_L:
      gather[i, e]                 state index feeding element e of row i
      scatter_row, scatter_elem    (row, element) of every state entry, in get_vector's order
                                   (G[i, j], i <= j: row i element j; W[i, j, k], i <= j <= k:
                                   row i element n + pair(j, k))."""
    n_g = n * (n + 1) // 2
    Pidx = _pair_index(n)
    start_i = _triple_offsets(n)
    r, c = np.triu_indices(n)
    gather = np.empty((n, n + n_g), dtype=np.int64)
    for i in range(n):
        gather[i, :n] = Pidx[i]
        t = np.sort(np.stack([np.full(len(r), i), r, c]), axis=0)
        gather[i, n:] = n_g + _triple_index(t[0], t[1], t[2], n, start_i)
    rows_w, elems_w = [], []
    for i in range(n):
        jj, kk = np.triu_indices(n - i)
        jj, kk = jj + i, kk + i
        rows_w.append(np.full(len(jj), i))
        elems_w.append(n + Pidx[jj, kk])
    return gather, np.concatenate([r] + rows_w), np.concatenate([c] + elems_w)


class StaticHessian(object):
    def __init__(self, ensemble=None, verbose=False, lanczos_input={}):
        """STATIC HESSIAN (Modules/StaticHessian.py:33-68): the object holds a Lanczos (built from
        `ensemble` with `lanczos_input`) and the state vector."""
        self.vector = None
        self.lanczos_input = lanczos_input
        self.lanczos = DL.Lanczos(ensemble, **lanczos_input)
        self.verbose = False
        self.prefix = "hessian_calculation"
        self.preconitioned = True
        self._maps = None
        if ensemble is not None:
            self.init(ensemble, verbose)
        self.__total_attributes__ = [item for item in self.__dict__.keys()]
        self.fixed_attributes = True

    def __setattr__(self, name, value):
        if "fixed_attributes" in self.__dict__:
            if name in self.__total_attributes__:
                super(StaticHessian, self).__setattr__(name, value)
            elif self.fixed_attributes:
                similar_objects = str(difflib.get_close_matches(name, self.__total_attributes__))
                raise AttributeError(f"""
        Error, the attribute '{name}' is not a member of '{type(self).__name__}'.
        Suggested similar attributes: {similar_objects} ?
        """)
        else:
            super(StaticHessian, self).__setattr__(name, value)

    # ---- state ---------------------------------------------------------------------------------
    def _sizes(self):
        n = self.lanczos.n_modes
        return n, (n * (n + 1)) // 2, (n * (n ** 2 + 3 * n + 2)) // 6

    def init(self, ensemble=None, verbose=True):
        """Initial state: G^-1 = the SSCHA matrix (1/w^2, or 1/w when preconditioned), W = 0
        (:133-181)."""
        if ensemble is not None:
            self.lanczos = DL.Lanczos(ensemble, **self.lanczos_input)
            self.lanczos.init()
            n, n_g, n_w = self._sizes()
            self.vector = np.zeros(n_g + n_w, dtype=DL.TYPE_DP)
            counter = 0
            for i in range(n):
                self.vector[counter] = 1 / self.lanczos.w[i] ** 2 if not self.preconitioned else 1 / self.lanczos.w[i]
                counter += n - i
        else:
            if self.lanczos.N == 0:
                raise ValueError("Error, you must specify an ensemble or initialize the system loading a lanczos algorithm.")
        self.verbose = verbose
        if verbose:
            print("Memory of StaticHessian initialized.")
            print("     memory requested: {} Gb of RAM per process".format((self.vector.nbytes) * 3 / 1024 ** 3))
            print("     (excluding memory occupied to store the ensemble)")

    def _index_maps(self):
        """Device copies of row_maps(n), built once per mode count."""
        if self._maps is not None and self._maps[0] == self.lanczos.n_modes:
            return self._maps[1:]
        torch = _torch()
        maps = tuple(torch.as_tensor(m, device="cuda") for m in row_maps(self.lanczos.n_modes))
        self._maps = (self.lanczos.n_modes,) + maps
        return maps

    def get_G_W(self, vector, ignore_W=False):
        """G (n, n) and W (n, n, n) from the state (:625-658)."""
        n, n_g, n_w = self._sizes()
        vector = np.asarray(vector)
        r, c = np.triu_indices(n)
        G = np.zeros((n, n), dtype=np.double)
        G[r, c] = vector[:n_g]
        G[c, r] = vector[:n_g]
        if ignore_W:
            return G
        start_i = _triple_offsets(n)
        I, J, K = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        t = np.sort(np.stack([I.ravel(), J.ravel(), K.ravel()]), axis=0)
        W = vector[n_g + _triple_index(t[0], t[1], t[2], n, start_i)].reshape(n, n, n)
        return G, W

    def get_vector(self, G, W):
        """The state from G and W: upper entries only (:660-690)."""
        n, n_g, n_w = self._sizes()
        vector = np.zeros(n_g + n_w, dtype=np.double)
        r, c = np.triu_indices(n)
        vector[:n_g] = G[r, c]
        counter = n_g
        for i in range(n):
            jj, kk = np.triu_indices(n - i)
            vector[counter:counter + len(jj)] = W[i, jj + i, kk + i]
            counter += len(jj)
        assert counter == n_w + n_g
        return vector

    # ---- the system matrix ---------------------------------------------------------------------
    def _apply_rows(self, rows, preconditioner=False, inverse_preconditioner=False):
        torch = _torch()
        L = self.lanczos
        if not preconditioner and not inverse_preconditioner:
            return L._static_apply_batched(rows, 1.0)
        power = 0.5 if preconditioner else -0.5
        out = torch.empty_like(rows)
        DL._native.apply_L1_static(L.device_ensemble, rows.contiguous(), out, -power)
        return out

    def apply_L_device(self, vect, preconditioner=False, inverse_preconditioner=False):
        """apply_L on a device state vector (a 1-D float64 CUDA tensor)."""
        if preconditioner and inverse_preconditioner:
            raise ValueError("Error, only one between preconditioner and inverse_preconditioner can be True")
        gather, srow, selem = self._index_maps()
        rows = vect[gather].contiguous()                     # (n, n + n_g)
        out = self._apply_rows(rows, preconditioner, inverse_preconditioner)
        return out[srow, selem]

    def apply_L(self, vect, preconditioner=False, inverse_preconditioner=False):
        """Apply the system matrix to the full state (:561-623)."""
        torch = _torch()
        self.lanczos._check_init()
        t1 = time.time()
        v = torch.as_tensor(np.asarray(vect, dtype=np.float64), device="cuda")
        res = self.apply_L_device(v, preconditioner, inverse_preconditioner).cpu().numpy()
        if self.verbose:
            print("Total time to apply the L matrix: {} s".format(time.time() - t1))
            sys.stdout.flush()
        return res

    # ---- solvers -------------------------------------------------------------------------------
    def run(self, n_steps, save_dir=None, threshold=1e-6, algorithm="cg-prec", extra_options={}):
        """RUN THE HESSIAN MATRIX CALCULATION (:184-287): the minimum-residual solve of
        A x = b (b = 1 on the diagonal of G), on the device."""
        torch = _torch()
        if save_dir is not None and not os.path.exists(save_dir):
            os.makedirs(save_dir)
        n, n_g, n_w = self._sizes()
        A = lambda X: torch.stack([self.apply_L_device(x) for x in X])                              # noqa: E731
        M = lambda X: torch.stack([self.apply_L_device(x, preconditioner=True) for x in X])         # noqa: E731

        def callback(x, iters):
            if save_dir is not None:
                np.savetxt(os.path.join(save_dir, "{}_step{:05d}.dat".format(self.prefix, iters)), x[0].cpu().numpy())
            sys.stdout.flush()

        x0 = torch.as_tensor(self.vector.copy(), device="cuda").reshape(1, -1)
        b = torch.zeros_like(x0)
        counter = 0
        for i in range(n):
            b[0, counter] = 1
            counter += n - i
        t1 = time.time()
        alg = algorithm.lower()
        if alg == "cg":
            res = DL.minimum_residual_batched(A, b, x0, max_iters=n_steps, conv_thr=threshold, callback=callback,
                                              verbose=self.verbose)
        elif alg == "cg-prec":
            res = DL.minimum_residual_batched_precond(A, b, M, X0=x0, max_iters=n_steps, conv_thr=threshold,
                                                      callback=callback, verbose=self.verbose)
        else:
            raise NotImplementedError("Error, algorithm '{}' not implemented.".format(algorithm))
        t2 = time.time()
        self.vector[:] = res[0].cpu().numpy()
        if save_dir is not None:
            self.save_status(os.path.join(save_dir, self.prefix))
        if self.verbose:
            print("\nHESSIAN CALCULATION CONVERGED\nTotal time to converge: {:.2f} s\n".format(t2 - t1))

    def run_no_mode_mixing(self, nsteps, save_dir=None, restart_from_file=False, noq=True):
        """RUN THE HESSIAN CALCULATION NEGLECTING MODE MIXING (:403-509): G(w = 0) of the Lanczos
        chain of every mode on the diagonal of G; degenerate modes reuse the previous mode's value.
        The non-degenerate modes' chains advance together (run_FT_batched)."""
        L0 = self.lanczos
        nmodes = L0.n_modes
        Gw = np.zeros((nmodes, nmodes), dtype=np.double)
        if save_dir is not None and not os.path.exists(save_dir):
            os.makedirs(save_dir)
        runs = [i for i in range(nmodes) if not (i > 0 and np.abs(L0.w[i - 1] - L0.w[i]) < 1e-10)]
        chains = {}
        for i in runs:
            c = L0.new_chain()
            c.prepare_mode(i)
            if save_dir is not None and restart_from_file:
                fname = os.path.join(save_dir, self.prefix + "_M{:d}_conv".format(i + 1))
                if os.path.exists(fname + ".npz"):
                    c.load_status(fname + ".npz")
            chains[i] = c
        todo = [c for c in chains.values() if nsteps - len(c.a_coeffs) > 0]
        for k0 in range(0, len(todo), 32):
            batch = todo[k0:k0 + 32]
            steps = max(nsteps - len(c.a_coeffs) for c in batch)
            DL.run_FT_batched(batch, steps)
        last = None
        for i in range(nmodes):
            if i in chains:
                c = chains[i]
                if save_dir is not None:
                    c.save_status(os.path.join(save_dir, self.prefix + "_M{:d}_conv".format(i + 1)))
                last = np.real(c.get_green_function_continued_fraction(np.array([0]), use_terminator=False, smearing=0)[0])
            Gw[i, i] = last
        W = np.zeros((nmodes, nmodes, nmodes), dtype=np.double)
        self.preconitioned = False
        self.vector = self.get_vector(Gw, W)
        return self.retrieve_hessian(noq=noq)

    def retrieve_hessian(self, noq=False):
        """The Hessian (:510-559): G from the state, inverted, back to Cartesian coordinates and
        multiplied by sqrt(m_a m_b).  Only the supercell matrix (noq=True) is available here."""
        if not noq:
            raise NotImplementedError("retrieve_hessian(noq=False) builds a cellconstructor Phonons object, which this "
                                      "package does not provide; call retrieve_hessian(noq=True) for the supercell matrix")
        new_vector = self.vector.copy()
        if self.preconitioned:
            new_vector = self.apply_L(self.vector, preconditioner=True)
        Ginv = self.get_G_W(new_vector, ignore_W=True)
        G = np.linalg.inv(Ginv)
        L = self.lanczos
        dyn = L.pols.dot(G.dot(L.pols.T))
        dyn[:, :] *= np.outer(np.sqrt(L.m), np.sqrt(L.m))
        return dyn

    # ---- files ---------------------------------------------------------------------------------
    def save_status(self, fname):
        """The state as text, the Lanczos status, the other attributes as json (:112-131)."""
        np.savetxt(fname, self.vector)
        self.lanczos.save_status(fname)
        IGNORE = ["lanczos", "vector", "fixed_attributes", "__total_attributes__", "_maps"]
        new_dict = {x: v for x, v in vars(self).items() if x not in IGNORE}
        with open(fname + ".json", "w") as fp:
            json.dump(new_dict, fp)

    def load_status(self, fname):
        """Inverse of save_status (:90-110)."""
        self.lanczos.load_status(fname + ".npz")
        n, n_g, n_w = self._sizes()
        self.vector = np.zeros(n_g + n_w, dtype=DL.TYPE_DP)
        self.vector[:] = np.loadtxt(fname)
        with open(fname + ".json", "r") as fp:
            data = json.load(fp)
            for x in data:
                self.__setattr__(x, data[x])
