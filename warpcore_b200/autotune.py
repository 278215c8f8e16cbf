"""Autotuner: launch geometry of the table kernels and the shape of the
served tables.

Two groups of choices are measured on the current GPU and written to a JSON
file that the library loads (wc_tune_load, called by the Python binding and
by the C++ headers):

- entries: threads per block and resident blocks per SM of the bulk table
  kernels, per (key width, operation, load-factor bucket, batch-size
  bucket).  Candidates are timed with CUDA events, median of `reps`
  repetitions; a candidate replaces the default (256 threads, occupancy
  limit) only if it is faster by more than `threshold`.  Batches under 2^14
  keys are launch-bound (a launch costs more than the work), so they keep
  the default and are not measured.
- serving: the window width (cooperative-group size) of the tables the
  serving layer creates itself, and the largest chunk of the persistent
  kernel, measured on a reduced served mix through the persistent kernel
  (aggregate Gops/s at a saturating arrival rate).  A caller's own tables
  keep the cg_size the caller asks for: it fixes capacity and slot
  placement, as in the reference.

    python -m warpcore_b200.autotune [--out FILE] [--quick] [--no-serving]
"""
import argparse
import json
import os
import statistics
import subprocess

import warpcore_b200 as wc

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_FILE = os.path.join(HERE, "tuning_b200.json")

CANDIDATES = [(256, 0), (128, 0), (64, 0), (256, 2)]
LOADS = [0.4, 0.6, 0.8, 0.9]          # one per load bucket (<.5, <.7, <.85, >=.85)
OPS = {"insert": 0, "retrieve": 2}
MIN_TUNED_BUCKET = 4                  # 2^15 keys: smaller batches keep the default


def size_for_bucket(b):
    return 1 << (7 + 2 * b)           # bucket b covers 2^(6+2b) .. 2^(8+2b)


def load(path=DEFAULT_FILE):
    """load a tuning file into the library; returns the number of entries"""
    import ctypes
    n = ctypes.c_uint64(0)
    wc._check(wc.lib().wc_tune_load(path.encode(), ctypes.byref(n)))
    return n.value


def _events_ms(fn):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b)


def tune_launch(key_widths=(4, 8), max_bucket=7, reps=9, threshold=0.05, quick=False):
    """measure the launch candidates; returns (entries, report)"""
    import torch
    from . import datagen
    lib = wc.lib()
    lib.wc_tune_reset()
    entries, report = [], []
    buckets = range(MIN_TUNED_BUCKET, max_bucket + 1, 2 if quick else 1)
    for kb in key_widths:
        for lb, lf in enumerate(LOADS):
            for sb in buckets:
                n = size_for_bucket(sb)
                cap = max(16 * n, 1 << 21)   # the batch adds at most 1/16 of capacity
                base = int(lf * cap)
                gen = torch.Generator(device="cuda")
                gen.manual_seed(7)
                keys = datagen.unique_keys(kb, 0, base + 2 * n, 11 + sb)
                vals = datagen.uniform_values(base + n, kb, gen)
                bk, bv = keys[:base], vals[:base]
                nk, nv = keys[base:base + n], vals[base:base + n]
                q = torch.cat([keys[:n // 2], keys[base + n:base + n + n - n // 2]])
                out = torch.empty(n, dtype=vals.dtype, device="cuda")
                t = wc.SingleValueHashTable(cap, key_bytes=kb)
                ms = {}
                for op_name, op in OPS.items():
                    for block, bps in CANDIDATES:
                        lib.wc_tune_set(kb, op, lb, sb, block, bps)
                        samples = []
                        if op_name == "retrieve":
                            t.init()
                            t.insert(bk, bv)
                        for _ in range(reps):
                            if op_name == "insert":
                                t.init()
                                t.insert(bk, bv)
                                torch.cuda.synchronize()
                                samples.append(_events_ms(lambda: t.insert(nk, nv)))
                            else:
                                samples.append(_events_ms(lambda: t.retrieve(q, out)))
                        ms["%s/%d/%d" % (op_name, block, bps)] = statistics.median(samples)
                    lib.wc_tune_set(kb, op, lb, sb, 0, 0)
                for op_name, op in OPS.items():
                    cand = {(b, p): ms["%s/%d/%d" % (op_name, b, p)] for b, p in CANDIDATES}
                    best = min(cand, key=cand.get)
                    if cand[best] > (1.0 - threshold) * cand[(256, 0)]:
                        best = (256, 0)
                    if best != (256, 0):
                        entries.append([kb, op, lb, sb, best[0], best[1]])
                        if op == 0:   # counting inserts follow the insert choice
                            entries.append([kb, 1, lb, sb, best[0], best[1]])
                report.append({"key_bytes": kb, "load": lf, "n": n,
                               "median_ms": {k: round(v, 5) for k, v in ms.items()}})
                del t, keys, vals, bk, bv, nk, nv, q, out
                torch.cuda.empty_cache()
    return entries, report


def tune_serving(cg_sizes=(4, 8, 16), chunks=(256, 1024, 4096), num_tables=512,
                 num_requests=4096, rate=1e6, reps=2):
    """window width of the served tables and the persistent kernel's largest
    chunk, by aggregate Gops/s of the reduced served mix at a saturating
    rate; returns (choice, report)"""
    import torch
    from .serve import ServedWorkload, run
    report = []
    for cg in cg_sizes:
        w = ServedWorkload(num_tables=num_tables, num_requests=num_requests, rate=rate, seed=5,
                           cg_size=cg)
        w.admit()
        for chunk in chunks:
            g, p99 = [], []
            for _ in range(reps + 1):
                w.reset()
                torch.cuda.synchronize()
                r = run(w, "persistent", max_batch_keys=chunk)
                if not w.verify():
                    raise RuntimeError("served answers differ (cg %d, chunk %d)" % (cg, chunk))
                g.append(r["gops"])
                p99.append(r["p99_us"])
            report.append({"cg_size": cg, "chunk_keys": chunk,
                           "gops": round(statistics.median(g[1:]), 4),
                           "p99_us": round(statistics.median(p99[1:]), 1)})
        del w
        torch.cuda.empty_cache()
    best = max(report, key=lambda m: m["gops"])
    return {"cg_size": best["cg_size"], "chunk_keys": best["chunk_keys"]}, report


def _git_head():
    try:
        return subprocess.run(["git", "-C", HERE, "rev-parse", "--short", "HEAD"],
                              capture_output=True, text=True).stdout.strip() or None
    except OSError:
        return None


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_FILE)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--reps", type=int, default=9)
    args = ap.parse_args()
    entries, report = tune_launch(reps=args.reps, quick=args.quick)
    data = {"device": torch.cuda.get_device_name(0),
            "commit": _git_head(),
            "note": "entries: launch geometry per (key_bytes, op, load bucket, size bucket) "
                    "[key_bytes, op, load_bucket, size_bucket, block_threads, blocks_per_sm]; "
                    "op 0 insert, 1 counting insert, 2 retrieve; only cells where a candidate "
                    "beat 256 threads at the occupancy limit by more than 5 %% (median of %d "
                    "CUDA-event timings) are listed; batches under 2^14 keys are not tuned"
                    % args.reps,
            "entries": entries, "measurements": report}
    if not args.no_serving:
        choice, sreport = tune_serving()
        data["serving"] = dict(choice, measurements=sreport)
    with open(args.out, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote %d entries to %s" % (len(entries), args.out))


if __name__ == "__main__":
    main()
