"""bench.py's reference arm on the CPU: the C/OpenMP restatement of the reference kernels on a
sample of the schedule, loading no library of this package, printing the contract's keys."""
import json
import os
import subprocess
import sys

from tests.conftest import REPO

PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--n", "18", "--depth", "8", "--nl", "12", "--steps", "2",
            "--warmup", "1", "--ref-units", "6"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED", int("libqsim_b200" in maps), int("libqsim_oracle" in maps))
"""


def test_reference_arm_runs_the_oracle_only():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=REPO, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    loaded = [l for l in lines if l.startswith("LOADED")][0].split()
    assert loaded[1] == "0" and loaded[2] == "1"  # the package's library is never mapped
    line = json.loads([l for l in lines if l.startswith("{")][0])
    for key in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["parallelism"] == "single GPU"
    assert set(line["config"]) == {"workload", "n", "depth", "nL", "tile_mode", "l2", "parallelism"}
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
