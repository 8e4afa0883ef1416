"""Configuration-sharded apply_full_L (tdscha_b200.parallel.ShardedEnsemble) run as two processes.

Each rank keeps its contiguous slice of the configurations on the device, computes its averages,
rescales them by N_eff of its slice and all-reduces (f_av, d2v_av) -- the reference's MPI partition
and MPI_Allreduce (CModules/LanczosFunctions.c:2123-2136, 2237, 2417, 2731).  Both ranks share the one
GPU of this machine and reduce over gloo on the host, so no kernel of one rank waits on the other's.
The sharded apply (direct and transposed, FP64 and bf16x3) must equal the apply of the whole ensemble
on one device."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, data_path, out_dir):
    import sys
    from datetime import timedelta
    from conftest import REPO
    sys.path.insert(0, os.path.join(REPO, "python-sscha_b200"))
    import torch
    import torch.distributed as dist
    from tdscha_b200 import _native
    from tdscha_b200.parallel import ShardedEnsemble
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    d = np.load(data_path)
    nb_ = int(d["n_blocks"])
    syms = [d[f"sym{i}"] for i in range(nb_)]
    blocks = [d[f"block{i}"] for i in range(nb_)]
    sh = ShardedEnsemble(d["X"], d["Y"], d["w"], d["rho"], float(d["T"]), syms, blocks, d["blocks_ids"])
    psi = torch.as_tensor(d["psi"], device="cuda")
    tr = [0, 1]
    opts = _native.ApplyOpts(0, 0, 0, 0, 0, 0.0)
    res = {}
    for prec in ("fp64", "bf16x3"):
        out = torch.empty_like(psi)
        sh.apply_full_L(psi, out, tr, opts, prec)
        torch.cuda.synchronize()
        res[f"sharded_{prec}"] = out.cpu().numpy()
        if rank == 0:
            full = _native.DeviceEnsemble(d["X"], d["Y"], d["w"], d["rho"], float(d["T"]), syms, blocks, d["blocks_ids"])
            ref = torch.empty_like(psi)
            full.apply_full_L(psi, ref, tr, opts, prec)
            torch.cuda.synchronize()
            res[f"full_{prec}"] = ref.cpu().numpy()
            full.close()
    res["slice"] = np.array(sh.slice)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **res)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_apply_equals_single_device(cuda, tmp_path):
    from tdscha_b200 import rocksalt as RS
    ens = RS.make_ensemble(2, 50, seed=9)
    n = len(ens.w)
    rng = np.random.default_rng(4)
    psi = rng.standard_normal((2, n + n * (n + 1))) * 1e-2
    data = dict(X=ens.X, Y=ens.Y, w=ens.w, rho=ens.rho, T=ens.T, blocks_ids=ens.blocks_ids,
                n_blocks=len(ens.symmetries), psi=psi)
    for i, (s, b) in enumerate(zip(ens.symmetries, ens.deg_space)):
        data[f"sym{i}"] = s
        data[f"block{i}"] = b
    path = str(tmp_path / "ens.npz")
    np.savez(path, **data)
    mp.start_processes(_worker, args=(2, _free_port(), path, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = np.load(str(tmp_path / "rank0.npz")), np.load(str(tmp_path / "rank1.npz"))
    assert tuple(r0["slice"]) == (0, 25) and tuple(r1["slice"]) == (25, 50)
    for prec, tol in (("fp64", 1e-12), ("bf16x3", 1e-4)):
        ref = r0[f"full_{prec}"]
        for r in (r0, r1):
            err = np.abs(r[f"sharded_{prec}"] - ref).max() / np.abs(ref).max()
            print(f"sharded {prec}: rel err {err:.2e}")
            assert err < tol, (prec, err)
