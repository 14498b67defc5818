"""bench.py's reference arm on the CPU: it prints one JSON line with the bench contract's keys, its
inputs are built on the host, and the only shared objects of this repository it maps are the
oracle's (the timed packet loop is the oracle, never the device library)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "cartesian_oligo",
           "--steps", "1", "--warmup", "0", "--packets", "1e5", "--cpu-seconds", "0.3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "packets/s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["setup"]["grid"].startswith("host")
    assert line["config"]["name"] == "cartesian_oligo" and line["config"]["cells"] == 500000
    libs = line["native_so_loaded"]
    assert libs and all(p.startswith("oracle" + os.sep) for p in libs), libs
