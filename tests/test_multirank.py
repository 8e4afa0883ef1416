"""Configuration-sharded averages across ranks (gloo, world size 2, CPU): the slices' averages,
rescaled by N_eff and all-reduced, equal the average over the whole ensemble -- the reference's
MPI_Allreduce semantics (CModules/LanczosFunctions.c:2123-2136, 2237, 2417, 2731)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import GOLDEN, load_golden


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    from conftest import REPO
    sys.path.insert(0, os.path.join(REPO, "python-sscha_b200"))
    from oracle import lanczos_oracle as LO
    from tdscha_b200.parallel import config_slice, reduce_partial_averages
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    d = load_golden("rocksalt_L2.npz")
    a, b = config_slice(len(d["rho"]), rank, world)
    # local average over the slice, normalised by the slice's own N_eff (what one GPU computes)
    f, dv = LO.perturb_average_sym(d["X"][a:b], d["Y"][a:b], d["w"], d["rho"][a:b], d["case0_R1"], d["case0_Y1"], d["T"],
                                   1, d["syms"], d["n_deg"], d["blocks"], d["blocks_ids"], n_threads=1)
    ft = torch.as_tensor(f).reshape(1, -1).clone()
    dt = torch.as_tensor(dv).reshape(1, *dv.shape).clone()
    reduce_partial_averages(ft, dt, float(d["rho"][a:b].sum()), float(d["rho"].sum()), lambda buf: dist.all_reduce(buf))
    if rank == 0:
        np.savez(out_path, f=ft[0].numpy(), d=dt[0].numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_config_slices_cover_the_ensemble():
    from tdscha_b200.parallel import config_slice
    for N in (1, 7, 10, 11):
        for size in (1, 2, 3, 4):
            sl = [config_slice(N, r, size) for r in range(size)]
            assert sl[0][0] == 0 and sl[-1][1] == N
            assert all(sl[i][1] == sl[i + 1][0] for i in range(size - 1))
            assert max(b - a for a, b in sl) - min(b - a for a, b in sl) <= 1


def test_two_rank_sharded_average_equals_full(tmp_path):
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    d = load_golden("rocksalt_L2.npz")
    gf, gd = d["case0_f"], d["case0_d2v"]
    assert np.abs(r["f"] - gf).max() <= 1e-12 * np.abs(gf).max()
    assert np.abs(r["d"] - gd).max() <= 1e-12 * np.abs(gd).max()
