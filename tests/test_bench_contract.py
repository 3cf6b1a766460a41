"""bench.py's reference arm (the oracle port on the host cores; no GPU) prints one JSON
line with the contract's keys; the batched and served workload generators draw the shapes
their configurations name."""
import json
import os
import subprocess
import sys

import numpy as np

from conftest import REPO


def test_reference_arm_json_line():
    """Every step of the reference arm is measured: steps x ms_per_step fits inside the
    process's own wall time, and the config dict is the workload only."""
    import time
    t0 = time.time()
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--workload", "c1",
                          "--steps", "3", "--warmup", "1", "--ref-bandwidth-steps", "2"], capture_output=True,
                         text=True, timeout=600, cwd=REPO)
    wall = time.time() - t0
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["steps"] == 3 and line["warmup"] == 1
    assert line["steps"] * line["ms_per_step"] / 1000.0 < wall
    # value = grid points x bandwidth steps per second of the timed steps
    assert abs(line["value"] - 1024 * 2 * 3 / (3 * line["ms_per_step"] / 1000.0)) <= 1e-6 * line["value"]
    assert set(line["config"]) == {"workload", "grid_points", "bandwidths", "bootstraps", "samples", "l2",
                                   "parallelism"}
    assert line["config"]["grid_points"] == 1024 and line["config"]["bandwidths"] == 251
    assert line["cpu_baseline"]["serial"]["cores"] == 1 and line["cpu_baseline"]["serial"]["value"] > 0


def test_workload_generators():
    from pkde_b200 import workloads as W
    mix = W.batched_mix(count=40, seed=3, n_range=(1e3, 2e3))
    assert len(mix) == 40 and {len(m["dims"]) for m in mix} <= {1, 2, 3}
    for m in mix:
        d = m["dims"]
        assert m["data"].shape[0] == len(d) and 1e3 <= m["data"].shape[1] <= 2e3
        if len(d) == 1:
            assert 256 <= d[0] <= 4096
        elif len(d) == 2:
            assert 128 <= d[0] <= 512 and d[0] == d[1]
        else:
            assert 32 <= d[0] <= 96
    served = W.served_mix(count=40, seed=4, n_range=(1e3, 2e3))
    assert {len(m["dims"]) for m in served} == {1, 2, 3, 4}
    assert max(np.prod(m["dims"]) for m in served if len(m["dims"]) == 4) <= 48 ** 4
    assert max(np.prod(m["dims"]) for m in served if len(m["dims"]) == 3) <= 128 ** 3
