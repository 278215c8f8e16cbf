"""Compiles tests/cpp/dropin_test.cu against the C++ drop-in headers and the
in-tree libwarpcore_b200.so into tests/cpp/_build/dropin_test."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(HERE, "dropin_test.cu")
OUT = os.path.join(HERE, "_build", "dropin_test")


def build(force=False):
    deps = [SRC, os.path.join(ROOT, "warpcore_b200", "libwarpcore_b200.so")]
    for dirpath, _, files in os.walk(os.path.join(ROOT, "include")):
        deps += [os.path.join(dirpath, f) for f in files]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    subprocess.run([nvcc, "-std=c++17", "--expt-extended-lambda", "--expt-relaxed-constexpr", "-O2",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-I" + os.path.join(ROOT, "include"),
                    SRC, "-L" + os.path.join(ROOT, "warpcore_b200"), "-lwarpcore_b200",
                    "-Xlinker", "-rpath," + os.path.join(ROOT, "warpcore_b200"),
                    "-o", OUT], check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
