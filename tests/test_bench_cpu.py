"""bench.py on the CPU: the reference arm's JSON line and the size-independent
checksums the table-wide operations are verified with.

The reference arm (``--impl reference``) times the CPU port of the
reference algorithm, so it runs without a GPU; its line must carry the same
metric, unit and direction as the library's arm, a ``cpu_baseline`` that
describes the run, and an ``e2e`` with no host/device copies."""
import json
import os
import subprocess
import sys

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_wrapping_sum_is_unsigned_modulo_2_64():
    # int64 tensors hold u64 keys: -1 is 2^64 - 1, and sums wrap
    assert bench._wrapping_sum(torch.tensor([-1, 1], dtype=torch.int64)) == 0
    assert bench._wrapping_sum(torch.tensor([-1], dtype=torch.int64)) == (1 << 64) - 1
    # int32 tensors hold u32 keys: summed as unsigned 32-bit words
    assert bench._wrapping_sum(torch.tensor([-1, -1], dtype=torch.int32)) == 2 * 0xFFFFFFFF
    assert bench._wrapping_sum(torch.tensor([5, 7], dtype=torch.int32)) == 12


def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "insert+retrieve Gops/s (keys processed per second, whole job)"
    assert d["unit"] == "Gops/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("SingleValueHashTable<u64,u64>")
