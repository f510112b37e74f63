"""The bench's reference arm on CPU: one JSON line with the contract's keys from rank 0, the
same config as the GPU arm's, nothing from the other ranks (they exit 0 without work), and
the product's CUDA library never mapped into the arm's process."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--chunk", "4000", "--variants", "1",
        "--points", "300000"]
# runs bench.py as __main__, then prints the shared objects mapped into the process
PROBE = ("import runpy, sys; sys.argv = ['bench.py'] + sys.argv[1:]; runpy.run_path('bench.py', run_name='__main__'); "
         "print('MAPS', sorted({l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')}))")


def _run(extra_env):
    env = dict(os.environ, **extra_env)
    cmd = [sys.executable, "-c", PROBE] + ARGS
    return subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


def test_reference_arm_line():
    from oracle import available_reference
    if not available_reference():
        pytest.skip("the reference was not built here (oracle/_ref)")
    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
    assert d["config"]["workload"].startswith("terrain 300000 points")
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.workload_config("terrain", 300000, bench.WORKLOADS["terrain"][2][:1], 1)
    maps = [ln for ln in r.stdout.splitlines() if ln.startswith("MAPS")]
    assert maps and "libxnyz_ref.so" in maps[0] and "libxnyz.so" not in maps[0].replace("libxnyz_ref.so", "")


def test_reference_arm_other_ranks_print_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
