"""Builds libwarpcore_b200.so in-tree with nvcc for sm_100a.

    python -m warpcore_b200.build [--jobs N] [--force]

Steps: generate the capacity prime table (csrc/gen_primes.c), compile every
csrc/*.cu translation unit in parallel, link one shared library with the
static CUDA runtime.  Objects go to warpcore_b200/_build/, the library next
to this file.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwarpcore_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O2", "-Xptxas", "-warn-spills",
    "-I" + os.path.join(ROOT, "include"), "-I" + BUILD, "-I" + CSRC,
]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(jobs=None, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    primes = os.path.join(BUILD, "wc_primes.inc")
    gen = os.path.join(BUILD, "gen_primes")
    gen_src = os.path.join(CSRC, "gen_primes.c")
    if force or not _newer(primes, [gen_src]):
        cc = os.environ.get("CC", "gcc")
        _run([cc, "-O2", "-o", gen, gen_src])
        _run([gen, primes])
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(ROOT, "include", "**", "*.cuh"), recursive=True) \
        + glob.glob(os.path.join(ROOT, "include", "*.h")) + [primes]
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    nvcc = _nvcc()
    objs = []
    todo = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or not _newer(obj, [src] + headers):
            todo.append((src, obj))
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
            futs = [ex.submit(_run, [nvcc] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", s, "-o", o])
                    for s, o in todo]
            for f in futs:
                logs.append(f.result())
    if force or todo or not _newer(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs)
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    print(build(args.jobs, args.force, args.verbose))
