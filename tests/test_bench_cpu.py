"""The benchmark's CPU side: its command line, the traffic figure it reads
from the committed profiles, and the reference arm's JSON line (the CPU
restatement of the reference's BA iteration, run here on a small size)."""
import importlib.util
import json
import os
import subprocess
import sys

from conftest import REPO

BENCH = os.path.join(REPO, "bench.py")


def _bench_module():
    spec = importlib.util.spec_from_file_location("bench_under_test", BENCH)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_help_lists_the_modes():
    r = subprocess.run([sys.executable, BENCH, "--help"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    for mode in ("bench", "kernels", "ttb", "batch", "adjoint", "precision", "gen"):
        assert mode in r.stdout


def test_profile_traffic_of_the_top_kernel():
    b = _bench_module()
    t = b.profile_traffic("k_mma_ba", 24, 12)
    # hx, Lt, Pw at 4.2e6 representatives: between the written-back minimum and 2x the algorithmic bytes
    assert t is not None and 5e7 < t < 3.4e8
    assert b.profile_traffic("k_mma_ba", 99, 1) is None


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--n", "10", "--k", "5", "--steps", "2",
                        "--warmup", "3", "--cpu-sample", "2000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
