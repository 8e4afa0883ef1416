"""
Seeded synthetic rock-salt systems: the inputs of the TD-SCHA linear-response path.

The reference builds X, Y, rho, w, pols and the mode-space symmetry blocks from an
``sscha.Ensemble`` and ``cellconstructor`` (Modules/DynamicalLanczos.py:315-442 for the ensemble
projection, :686-782 for ``prepare_symmetrization`` via ``CC.symmetries.GetSymmetriesOnModesDeg``).
Neither package is vendored with the reference, so this module generates the same objects for a
rock-salt crystal from first principles:

* primitive fcc cell (a = 5.6 A), cation at the origin, anion at a/2 x; L x L x L supercells;
* nearest-neighbour pair potential  V = k2/2 |du|^2 + k3/6 dr^3 + k4/24 dr^4  with du = u_j - u_i
  and dr = r0_hat . du (bond-projected stretch).  The harmonic term is isotropic so that only the
  three uniform translations have zero frequency (a central-force harmonic term leaves whole
  transverse branches at zero frequency, where psi = (1+2n)/(2w) diverges);
* the harmonic dynamical matrix is diagonalised, the three translations removed, and modes of equal
  frequency grouped into degenerate blocks whose frequencies are set to the block mean (so the
  thermal factors commute exactly with every symmetry);
* symmetry operations = O_h (48 signed permutations about the cation) x L^3 lattice translations,
  acting on mass-weighted displacements as atom permutations + rotations; in mode space each block
  gets S_b[j] = E_b^T P_j E_b (the per-block tables consumed by the averages kernel);
* configurations are sampled at temperature T from the harmonic density matrix
  (<q_mu^2> = (1+2n_mu)/(2 w_mu) in the mass-weighted normal coordinates), forces come from the full
  potential, and Y holds the anharmonic residual f - f_harm, mass-rescaled and projected on the
  modes (DynamicalLanczos.py:384-442).  The symmetrised mean force vanishes identically here
  (every atom sits on an O_h site) so the subtraction of DynamicalLanczos.py:388-421 is a no-op.

Units are Rydberg atomic units throughout (Bohr, Ry, mass unit 2 m_e), as in the reference.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

RY_TO_K = 157887.32400374097
RY_TO_EV = 13.605693122994
BOHR_TO_ANG = 0.529177210903
AMU_TO_RY = 911.444243096          # 1 amu in units of 2 m_e
RY_TO_CM = 109737.31568160         # CODATA Rydberg constant in cm^-1

EV_A2_TO_RY_B2 = BOHR_TO_ANG ** 2 / RY_TO_EV
EV_A3_TO_RY_B3 = BOHR_TO_ANG ** 3 / RY_TO_EV
EV_A4_TO_RY_B4 = BOHR_TO_ANG ** 4 / RY_TO_EV


@dataclass
class RockSaltSystem:
    L: int
    T: float
    nat: int
    masses: np.ndarray          # (3 nat,) per Cartesian component, Ry mass units
    positions: np.ndarray       # (nat, 3) Bohr
    bonds: np.ndarray           # (n_bonds, 2) atom indices (i, j)
    bond_dirs: np.ndarray       # (n_bonds, 3) unit vectors r0_j - r0_i
    w: np.ndarray               # (n,) Ry, non-translational
    pols: np.ndarray            # (3 nat, n) orthonormal eigenvectors
    symmetries: list            # per block (N_sym, d, d)
    deg_space: list             # per block mode indices (contiguous)
    blocks_ids: np.ndarray      # (n,)
    n_syms: int
    k2: float
    k3: float
    k4: float
    perm: np.ndarray = field(repr=False, default=None)     # (N_sym, nat) atom maps
    rot: np.ndarray = field(repr=False, default=None)      # (N_sym, 3, 3)
    nat_uc: int = 2
    uc_species: tuple = (0, 1)

    @property
    def n_modes(self):
        return len(self.w)


def _oh_rotations():
    mats = []
    for p in itertools.permutations(range(3)):
        for s in itertools.product((1, -1), repeat=3):
            R = np.zeros((3, 3))
            for r in range(3):
                R[r, p[r]] = s[r]
            mats.append(R)
    return np.array(mats)


def build_system(L, T=300.0, a_ang=5.6, masses_amu=(23.0, 35.45), k2=2.0, k3=-3.0, k4=6.0,
                 deg_tol=1e-7, with_symmetries=True, symmetries_on_gpu=False):
    """Supercell geometry, harmonic modes and mode-space symmetry blocks.  k2/k3/k4 in eV/A^n.
    symmetries_on_gpu: project the symmetry operations onto the modes with the device kernel
    (tdscha_symmetries_on_modes) instead of numpy (large supercells)."""
    a = a_ang / BOHR_TO_ANG
    prim = 0.5 * a * np.array([[0, 1, 1], [1, 0, 1], [1, 1, 0]], dtype=np.float64)
    basis = np.array([[0.0, 0.0, 0.0], [0.5 * a, 0.0, 0.0]])
    species = []
    pos = []
    for n1, n2, n3 in itertools.product(range(L), repeat=3):
        R = n1 * prim[0] + n2 * prim[1] + n3 * prim[2]
        for s in range(2):
            pos.append(R + basis[s])
            species.append(s)
    pos = np.array(pos)
    species = np.array(species)
    nat = len(pos)
    sup = L * prim
    sup_inv = np.linalg.inv(sup)

    def wrap_frac(r):
        f = r @ sup_inv
        return f - np.floor(f + 1e-9)

    frac = wrap_frac(pos)
    key = {tuple(np.round(f * 4 * L).astype(int) % (4 * L)): i for i, f in enumerate(frac)}

    def find(r):
        f = wrap_frac(r)
        k = tuple(np.round(f * 4 * L).astype(int) % (4 * L))
        return key[k]

    # nearest-neighbour bonds: cation i -> anion at r_i + a/2 * (+-x, +-y, +-z)
    bonds, dirs = [], []
    for i in range(nat):
        if species[i] != 0:
            continue
        for d in np.vstack([np.eye(3), -np.eye(3)]):
            j = find(pos[i] + 0.5 * a * d)
            bonds.append((i, j))
            dirs.append(d)
    bonds = np.array(bonds, dtype=np.int64)
    dirs = np.array(dirs)

    m_at = np.array([masses_amu[s] for s in species]) * AMU_TO_RY
    masses = np.repeat(m_at, 3)
    k2r = k2 * EV_A2_TO_RY_B2
    Phi = np.zeros((3 * nat, 3 * nat))
    for (i, j) in bonds:
        for c in range(3):
            Phi[3 * i + c, 3 * i + c] += k2r
            Phi[3 * j + c, 3 * j + c] += k2r
            Phi[3 * i + c, 3 * j + c] -= k2r
            Phi[3 * j + c, 3 * i + c] -= k2r
    sm = np.sqrt(masses)
    Dm = Phi / np.outer(sm, sm)
    ev, vec = np.linalg.eigh(Dm)
    order = np.argsort(ev)
    ev, vec = ev[order], vec[:, order]
    # drop the three uniform translations (the three smallest eigenvalues, all ~0)
    ev, vec = ev[3:], vec[:, 3:]
    if ev.min() <= 0:
        raise RuntimeError("non-positive harmonic frequency after removing translations")
    w = np.sqrt(ev)

    # degenerate blocks: consecutive frequencies within a relative tolerance
    blocks = []
    start = 0
    for m in range(1, len(w) + 1):
        if m == len(w) or abs(w[m] - w[start]) > deg_tol * w[start]:
            blocks.append(list(range(start, m)))
            start = m
    for blk in blocks:
        w[blk] = w[blk].mean()
    blocks_ids = np.zeros(len(w), dtype=np.intc)
    for b, blk in enumerate(blocks):
        blocks_ids[blk] = b

    sys_ = RockSaltSystem(L=L, T=float(T), nat=nat, masses=masses, positions=pos, bonds=bonds,
                          bond_dirs=dirs, w=w, pols=vec, symmetries=[], deg_space=[],
                          blocks_ids=blocks_ids, n_syms=1, k2=k2r, k3=k3 * EV_A3_TO_RY_B3,
                          k4=k4 * EV_A4_TO_RY_B4)
    sys_.deg_space = [np.array(blk, dtype=np.intc) for blk in blocks]
    if not with_symmetries:
        sys_.symmetries = [np.ones((1, 1, 1))] * len(w)
        sys_.deg_space = [np.array([i], dtype=np.intc) for i in range(len(w))]
        sys_.blocks_ids = np.arange(len(w), dtype=np.intc)
        return sys_

    rots = _oh_rotations()
    trans = np.array([n1 * prim[0] + n2 * prim[1] + n3 * prim[2] for n1, n2, n3 in itertools.product(range(L), repeat=3)])
    # image atoms of every (rotation, translation): lattice keys of the images looked up in a table
    q = 4 * L
    lut = np.full(q ** 3, -1, dtype=np.int64)
    for kk, i in key.items():
        lut[(kk[0] * q + kk[1]) * q + kk[2]] = i
    perms, rmats = [], []
    for R in rots:
        img = (pos @ R.T)[None, :, :] + trans[:, None, :]          # (n_trans, nat, 3)
        f = wrap_frac(img.reshape(-1, 3))
        k = np.round(f * q).astype(np.int64) % q
        p = lut[(k[:, 0] * q + k[:, 1]) * q + k[:, 2]].reshape(len(trans), nat)
        if (p < 0).any():
            raise RuntimeError("symmetry image off the lattice")
        perms.extend(p)
        rmats.extend([R] * len(trans))
    perms = np.array(perms, dtype=np.int64)
    rmats = np.array(rmats)
    N_sym = len(perms)
    if symmetries_on_gpu:
        from . import _native
        sym_blocks = _native.symmetries_on_modes(vec, perms, rmats, sys_.deg_space)
    else:
        # P_j acting on (3 nat) mass-weighted displacement: (P v)[pi(a)] = R v[a].  The symmetries
        # are ordered rotation-major, so R E is formed once per rotation; the images of a chunk of
        # translations are stacked and their block products run as one batched matmul (the same
        # per-matrix product as one symmetry at a time, so the tables are identical)
        sym_blocks = [np.zeros((N_sym, len(blk), len(blk))) for blk in blocks]
        E3 = vec.reshape(nat, 3, -1)
        n_tr = len(trans)
        chunk = 32
        for r in range(len(rots)):
            RE = np.einsum("ab,nbm->nam", rmats[r * n_tr], E3)
            for t0 in range(0, n_tr, chunk):
                t1 = min(n_tr, t0 + chunk)
                j0, j1 = r * n_tr + t0, r * n_tr + t1
                PE = np.empty((t1 - t0,) + E3.shape)
                PE[np.arange(t1 - t0)[:, None], perms[j0:j1]] = RE[None]
                PE = PE.reshape(t1 - t0, 3 * nat, -1)
                for b, blk in enumerate(blocks):
                    sym_blocks[b][j0:j1] = np.matmul(vec[:, blk].T[None], PE[:, :, blk])
    sys_.symmetries = sym_blocks
    sys_.n_syms = N_sym
    sys_.perm = perms
    sys_.rot = rmats
    return sys_


def thermal_factors(w, T):
    nb = 1.0 / (np.exp(w * RY_TO_K / T) - 1.0) if T > 0 else np.zeros_like(w)
    ups = 2 * w / (1 + 2 * nb)
    return nb, ups, 1.0 / ups


def anharmonic_forces(sys_: RockSaltSystem, u):
    """Forces of the k3/k4 bond terms for displacements u (N, nat, 3), Ry/Bohr."""
    i, j = sys_.bonds[:, 0], sys_.bonds[:, 1]
    du = u[:, j, :] - u[:, i, :]
    dr = np.einsum("nbc,bc->nb", du, sys_.bond_dirs)
    g = sys_.k3 / 2 * dr ** 2 + sys_.k4 / 6 * dr ** 3       # dV/d(dr)
    fb = -g[:, :, None] * sys_.bond_dirs[None, :, :]          # force on j
    F = np.zeros_like(u)
    np.add.at(F, (slice(None), j), fb)
    np.add.at(F, (slice(None), i), -fb)
    return F


def sample_ensemble(sys_: RockSaltSystem, N, seed=0, chunk=2000):
    """Seeded Gaussian ensemble: returns X, Y (N, n) C order and rho (N,)."""
    rng = np.random.default_rng(seed)
    n = sys_.n_modes
    _, _, psi = thermal_factors(sys_.w, sys_.T)
    sq = np.sqrt(psi)
    sm = np.sqrt(sys_.masses)
    X = np.empty((N, n))
    Y = np.empty((N, n))
    for s in range(0, N, chunk):
        e = min(N, s + chunk)
        Xc = rng.standard_normal((e - s, n)) * sq
        u = (Xc @ sys_.pols.T) / sm                       # Bohr, (N, 3 nat)
        F = anharmonic_forces(sys_, u.reshape(e - s, sys_.nat, 3)).reshape(e - s, -1)
        X[s:e] = Xc
        Y[s:e] = (F / sm) @ sys_.pols
    rho = np.ones(N)
    return np.ascontiguousarray(X), np.ascontiguousarray(Y), rho


def sample_force_components(sys_: RockSaltSystem, N, seed=0):
    """The ensemble of sample_ensemble (same seed, same X) with its forces split by coupling:
    Y = k3 Y3 + k4 Y4 (internal Ry/Bohr units of k3, k4).  Returns X, Y3, Y4, rho."""
    import dataclasses
    X, _, rho = sample_ensemble(sys_, N, seed=seed)
    out = []
    for k3, k4 in ((1.0, 0.0), (0.0, 1.0)):
        part = dataclasses.replace(sys_, k3=k3, k4=k4)
        _, Yk, _ = sample_ensemble(part, N, seed=seed)
        out.append(Yk)
    return X, out[0], out[1], rho


def random_born_charges(nat_uc=2, seed=0):
    """Z*[atom, field, cart] ~ N(0, 1), seeded."""
    return np.random.default_rng(seed).standard_normal((nat_uc, 3, 3))


def random_raman_tensor(nat_uc=2, seed=0):
    """raman_tensor[in, out, 3 nat_uc]: one seeded symmetric 3x3 per (atom, cart)."""
    rng = np.random.default_rng(seed)
    t = rng.standard_normal((3, 3, 3 * nat_uc))
    return 0.5 * (t + t.transpose(1, 0, 2))


def raman_vector(raman_tensor, pol_in, pol_out):
    """Contract the Raman tensor with the light polarisations and impose the acoustic sum rule
    (what the reference obtains from the dynamical matrix's GetRamanVector)."""
    v = np.einsum("a,abc,b->c", pol_in, raman_tensor, pol_out).reshape(-1, 3)
    v -= v.mean(axis=0, keepdims=True)
    return v.ravel()


@dataclass
class SyntheticEnsemble:
    """The arrays the reference's Lanczos constructor extracts from an ``sscha.Ensemble``
    (DynamicalLanczos.py:315-442), plus the mode-space symmetry blocks and the dielectric /
    Raman response tensors that the reference reads from the dynamical matrix."""
    T: float
    nat: int
    m: np.ndarray
    w: np.ndarray
    pols: np.ndarray
    N: int
    rho: np.ndarray
    X: np.ndarray
    Y: np.ndarray
    symmetries: list
    deg_space: list
    blocks_ids: np.ndarray
    supercell: tuple
    nat_uc: int = 2
    effective_charges: np.ndarray = None
    raman_tensor: np.ndarray = None
    system: RockSaltSystem = None


def make_ensemble(L, N, T=300.0, seed=0, k2=2.0, k3=-3.0, k4=6.0, with_symmetries=True, system=None):
    """Seeded rock-salt ensemble (the synthetic stand-in for an sscha ensemble)."""
    s = system if system is not None else build_system(L, T=T, k2=k2, k3=k3, k4=k4, with_symmetries=with_symmetries)
    X, Y, rho = sample_ensemble(s, N, seed=seed)
    return SyntheticEnsemble(T=s.T, nat=s.nat, m=s.masses, w=s.w, pols=s.pols, N=N, rho=rho, X=X, Y=Y,
                             symmetries=s.symmetries, deg_space=s.deg_space, blocks_ids=s.blocks_ids,
                             supercell=(L, L, L), nat_uc=2, effective_charges=random_born_charges(seed=seed),
                             raman_tensor=random_raman_tensor(seed=seed), system=s)


# ------------------------------------------------------------------------------------------------
# The seeded chain of the precision check: one bi-conjugate chain from a seeded random unit vector
# on R^(1), G(w) on 500 points 0-400 cm^-1 with 5 cm^-1 smearing and no terminator.
# ------------------------------------------------------------------------------------------------
CHAIN_SEED = 11
RY_TO_CM = 109737.31568160


def gf_grid():
    """(omega in Ry, smearing in Ry) of the precision check."""
    return np.linspace(0.0, 400.0, 500) / RY_TO_CM, 5.0 / RY_TO_CM


def seeded_chain(system, X, Y, rho, device_ensemble, precision, steps, seed=CHAIN_SEED):
    """Run `steps` bi-conjugate steps of the seeded chain on `device_ensemble` in `precision`;
    returns the Lanczos object (a/b/c coefficients filled)."""
    from .DynamicalLanczos import Lanczos, run_FT_batched
    s = system
    eo = SyntheticEnsemble(T=s.T, nat=s.nat, m=s.masses, w=s.w, pols=s.pols, N=X.shape[0], rho=rho, X=X, Y=Y,
                           symmetries=s.symmetries, deg_space=s.deg_space, blocks_ids=s.blocks_ids,
                           supercell=(round((s.nat // 2) ** (1 / 3)),) * 3)
    lanc = Lanczos(eo, precision=precision)
    lanc.symmetries, lanc.degenerate_space, lanc.sym_block_id = s.symmetries, s.deg_space, s.blocks_ids
    lanc.N_degeneracy = np.array([len(d) for d in s.deg_space], dtype=np.intc)
    lanc.n_syms, lanc.initialized, lanc.device_ensemble = s.n_syms, True, device_ensemble
    lanc.prepare_random(seed=seed, sector="R")
    run_FT_batched([lanc], steps, precision=precision, verbose=False)
    return lanc


def ensemble_checksum(X, Y, rho):
    """Order-sensitive float summary of the sampled ensemble (identifies the inputs of a stored chain)."""
    k = np.arange(1, X.shape[0] + 1, dtype=np.float64)[:, None]
    return np.array([float((X * k).sum()), float((Y * k).sum()), float(rho.sum())])
