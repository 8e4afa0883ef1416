"""The benchmark's reference arm (the reference's CPU implementation of the averages on the host
cores) prints the contract's JSON line; its timing falls back to the C port when the reference
kernel is not built.  CPU only, tiny workload."""
import json
import os
import subprocess
import sys

import numpy as np

from conftest import REPO


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--L", "2", "--N", "20",
                          "--steps", "1", "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["reference_kind"] == line["cpu_baseline"]["kind"]     # which CPU code ran, at the top level
    # the same step as the repo arm: one batched apply of 2 x chains vectors
    assert line["applies_per_step"] == 16
    assert abs(line["ms_per_step"] - 16 * line["ms_per_apply"]) <= 1e-9 * line["ms_per_step"]
    assert abs(line["ms_per_apply"] * line["value"] - 1e3) <= 1e-9 * 1e3


def test_cpu_timing_with_the_port_backend():
    sys.path.insert(0, REPO)
    import bench
    from tdscha_b200 import rocksalt as RS
    s = RS.build_system(2)
    X, Y, rho = RS.sample_ensemble(s, 4, seed=0)
    v, cores, sample, kind = bench.cpu_reference_timing(s, X, Y, rho, seconds_target=0.5, max_procs=8, backend="port")
    assert kind == "port" and v > 0 and np.isfinite(v)
    assert cores == 4            # never more processes than configurations
    assert "C port" in sample
