"""Configuration-sharded apply_full_L over several GPUs (one process per GPU, torch.distributed/NCCL).

The reference distributes the configurations of the ensemble over MPI ranks
(CModules/LanczosFunctions.c:2123-2136: contiguous slices, the first N % size ranks get one extra),
broadcasts the perturbation (:2120, 2334, 2647) and sums the partial averages with MPI_Allreduce
(:2237, 2417, 2731) before normalising by N_eff * N_sym of the whole ensemble.  Here every rank keeps
its slice resident on its GPU; one apply is
    prologue (local) -> averages of the slice (local, normalised by the slice's N_eff)
    -> rescale by N_eff_slice / N_eff_total -> one all-reduce(SUM) of (f_av, d2v_av), n + n^2 FP64
       per vector -> epilogue (local)
so the only exchange is the reduction the reference does.  Every rank must call with the same
vectors (they are replicated, as the reference's Bcast makes them).
"""
from __future__ import annotations

import numpy as np


def config_slice(N, rank, size):
    """[start, stop) of the configurations owned by `rank` (LanczosFunctions.c:2123-2136)."""
    count, rem = divmod(N, size)
    if rank < rem:
        start = rank * (count + 1)
        return start, start + count + 1
    start = rank * count + rem
    return start, start + count


def reduce_partial_averages(f_local, d_local, neff_local, neff_total, all_reduce):
    """Rescale slice-normalised averages to the whole ensemble and sum them over ranks in place.
    `all_reduce(buf)` sums a flat buffer over the group (torch.distributed.all_reduce on GPU)."""
    scale = neff_local / neff_total
    f_local.mul_(scale)
    d_local.mul_(scale)
    nb = f_local.shape[0]
    flat = __import__("torch").cat([f_local.reshape(nb, -1), d_local.reshape(nb, -1)], dim=1).contiguous()
    all_reduce(flat)
    n = f_local.shape[1]
    f_local.copy_(flat[:, :n])
    d_local.copy_(flat[:, n:].reshape(d_local.shape))


class ShardedEnsemble:
    """This rank's slice of the ensemble on its GPU, reduced over `group` at every apply."""

    def __init__(self, X, Y, w, rho, T, symmetries, deg_space, blocks_ids, group=None):
        import torch.distributed as dist
        from . import _native
        self.dist = dist
        self.group = group
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        size = dist.get_world_size(group) if dist.is_initialized() else 1
        N = X.shape[0]
        a, b = config_slice(N, rank, size)
        if b <= a:
            raise ValueError(f"rank {rank} owns no configuration (N={N} < world size {size})")
        self.slice = (a, b)
        self.neff_total = float(np.sum(rho))
        self.neff_local = float(np.sum(rho[a:b]))
        self.n = X.shape[1]
        self.local = _native.DeviceEnsemble(X[a:b], Y[a:b], w, rho[a:b], T, symmetries, deg_space, blocks_ids)

    def apply_full_L(self, psi, out, transpose, opts, precision="fp64"):
        import torch
        nb = psi.shape[0]
        n = self.n
        R = torch.empty((nb, n), dtype=torch.float64, device=psi.device)
        Ys = torch.empty((nb, n, n), dtype=torch.float64, device=psi.device)
        f = torch.zeros((nb, n), dtype=torch.float64, device=psi.device)
        d = torch.zeros((nb, n, n), dtype=torch.float64, device=psi.device)
        if not opts.ignore_v3:
            self.local.apply_prologue(psi, R, Ys, transpose, opts)
            self.local.perturb_average_device(R, Ys, f, d, 0 if opts.ignore_v4 else 1, precision)
            reduce_partial_averages(f, d, self.neff_local, self.neff_total,
                                    lambda buf: self.dist.all_reduce(buf, group=self.group))
        self.local.apply_epilogue(psi, f, d, out, transpose, opts)
