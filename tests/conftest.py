import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (REPO, os.path.join(REPO, "python-sscha_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def _ensure_oracle_built():
    lib = os.path.join(REPO, "oracle", "_build", "libtdscha_oracle.so")
    src = os.path.join(REPO, "oracle", "tdscha_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "all"], check=True)


_ensure_oracle_built()


def load_golden(name):
    """Golden fixture as a dict with the symmetry blocks regrouped into lists."""
    d = dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))
    nb = int(d["n_blocks"])
    d["syms"] = [d[f"sym{i}"] for i in range(nb)]
    d["blocks"] = [d[f"block{i}"] for i in range(nb)]
    d["n_deg"] = np.array([len(b) for b in d["blocks"]], dtype=np.intc)
    d["T"] = float(d["T"])
    return d


@pytest.fixture(scope="session")
def mode10():
    return load_golden("mode10.npz")


@pytest.fixture(scope="session")
def rocksalt_l2():
    return load_golden("rocksalt_L2.npz")


def gpu_available():
    try:
        import torch
        if not torch.cuda.is_available():
            return False
        return torch.cuda.get_device_capability(0)[0] == 10
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no sm_100 GPU")
    import torch
    return torch
