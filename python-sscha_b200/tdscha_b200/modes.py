"""Lanczos inputs from an ensemble, computed on the GPU: the step before the hot path.

The reference builds them in the Lanczos constructor (Modules/DynamicalLanczos.py:315-442) and in
prepare_symmetrization (:686-782) with cellconstructor / sscha, which are not vendored with it.
Here the same quantities come from plain arrays:

  * ``ensemble_to_modes``: u (Angstrom) and forces (Ry/Angstrom) of the configurations, the SSCHA
    forces and the (already symmetrised) average force of the unit cell -> X, Y in the
    polarisation basis, exactly the unit handling and subtractions of :376-442;
  * ``symmetries_on_modes``: the symmetry group as image atoms and Cartesian rotations ->
    degenerate blocks of the frequencies and the per-block tables S_b^j = E_b^T P_j E_b.
"""
from __future__ import annotations

import numpy as np

from . import _native

BOHR_TO_ANG = 0.529177210903   # Angstrom per Bohr (the reference converts with sscha's Ensemble.Bohr)


def ensemble_to_modes(u_disps, forces, sscha_forces, masses, pols, f_mean_uc=None, n_cell=1):
    """X, Y (N, n_modes) from displacements u_disps (N, 3 nat) in Angstrom, forces and sscha_forces
    (N, 3 nat) in Ry/Angstrom, masses (3 nat) in Ry units and pols (3 nat, n_modes).  f_mean_uc is
    the symmetrised average force of the unit cell (nat_uc, 3) in Ry/Angstrom (None = zero), tiled
    over the n_cell cells of the supercell (DynamicalLanczos.py:383-425)."""
    u = np.asarray(u_disps, dtype=np.float64).reshape(len(u_disps), -1) / BOHR_TO_ANG
    f = (np.asarray(forces, dtype=np.float64) - np.asarray(sscha_forces, dtype=np.float64)).reshape(u.shape) * BOHR_TO_ANG
    if f_mean_uc is not None:
        fm = np.tile(np.asarray(f_mean_uc, dtype=np.float64), (n_cell, 1)).ravel() * BOHR_TO_ANG
        f = f - fm[None, :]
    return _native.project_ensemble(u, f, masses, pols)


def degenerate_blocks(w, deg_tol=1e-7):
    """Consecutive frequencies (ascending) within a relative tolerance form one block."""
    w = np.asarray(w, dtype=np.float64)
    if np.any(np.diff(w) < 0):
        raise ValueError("frequencies must be sorted in ascending order")
    blocks, start = [], 0
    for m in range(1, len(w) + 1):
        if m == len(w) or abs(w[m] - w[start]) > deg_tol * abs(w[start]):
            blocks.append(np.arange(start, m, dtype=np.intc))
            start = m
    blocks_ids = np.zeros(len(w), dtype=np.intc)
    for b, blk in enumerate(blocks):
        blocks_ids[blk] = b
    return blocks, blocks_ids


def symmetries_on_modes(pols, w, perm, rot, deg_tol=1e-7):
    """(symmetries, degenerate_space, blocks_ids) for the Lanczos: perm (N_sym, nat) gives the image
    of every atom under each operation, rot (N_sym, 3, 3) its Cartesian rotation."""
    blocks, blocks_ids = degenerate_blocks(w, deg_tol)
    return _native.symmetries_on_modes(pols, perm, rot, blocks), blocks, blocks_ids
