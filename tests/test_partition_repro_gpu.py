"""The partition count kernel's miscount, reduced to a minimal program
(tests/cpp/partition_count_repro.cu): one shared-memory atomicAdd on
hist[partition_owner(...)] against the range-checked local form the library
uses.  The library's form must count right in every case; the direct form's
outcome is reported (nvcc 12.9, sm_100a, -O3 counted every key in bin 0)."""
import json
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_partition_count_forms():
    src = os.path.join(HERE, "cpp", "partition_count_repro.cu")
    out = os.path.join(HERE, "cpp", "_build", "partition_count_repro")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    subprocess.run([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-o", out, src], check=True, capture_output=True)
    r = subprocess.run([out], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    cases = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(cases) == 20
    assert all(c["local_bad_bins"] == 0 for c in cases)
    direct_wrong = sum(c["direct_bad_bins"] > 0 for c in cases)
    print("direct form wrong in %d of %d cases" % (direct_wrong, len(cases)))
