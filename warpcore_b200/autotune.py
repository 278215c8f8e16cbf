"""Launch-geometry autotuner for the table kernels.

The probe-window width is the table's cooperative-group size, a template knob
of the reference that fixes capacity and slot placement; the lanes per
window follow from it (window bytes / 16). What remains free is the launch
geometry: threads per block and resident blocks per SM. Small batches want
small blocks spread over many SMs. Large batches want full occupancy.

This module measures candidates for each (key width, operation, load-factor
bucket, batch-size bucket) on the current GPU. It stores the winners in a
JSON file and loads them into the library with wc_tune_set.
`warpcore_b200/tuning_b200.json` holds the table measured on B200, and the
Python binding loads it when the library is first used.

    python -m warpcore_b200.autotune [--out FILE] [--quick]
"""
import argparse
import json
import os

import warpcore_b200 as wc

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_FILE = os.path.join(HERE, "tuning_b200.json")

CANDIDATES = [(256, 0), (128, 0), (64, 0), (32, 0)]
LOADS = [0.4, 0.6, 0.8, 0.9]          # one per load bucket (<.5, <.7, <.85, >=.85)
OPS = {"insert": 0, "retrieve": 2}


def size_for_bucket(b):
    return 1 << (7 + 2 * b)           # bucket b covers 2^(6+2b) .. 2^(8+2b)


def apply(entries):
    lib = wc.lib()
    for kb, op, lb, sb, block, bps in entries:
        wc._check(lib.wc_tune_set(kb, op, lb, sb, block, bps))


def load(path=DEFAULT_FILE):
    """load a tuning file into the library; returns the number of entries"""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        data = json.load(f)
    apply(data["entries"])
    return len(data["entries"])


def _time(fn, reps):
    import torch
    best = None
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    return best


def entries_from_measurements(report, threshold=0.05):
    """pick per (key width, op, load, size) the fastest geometry, but keep the
    default (256 threads) unless a candidate beats it by more than
    `threshold`: differences below that are run-to-run noise"""
    entries = []
    for m in report:
        kb = m["key_bytes"]
        lb = LOADS.index(m["load"])
        sb = [b for b in range(16) if size_for_bucket(b) == m["n"]][0]
        for op_name, op in OPS.items():
            times = {int(k.split("/")[1]): v for k, v in m["ms"].items() if k.startswith(op_name)}
            block = min(times, key=times.get)
            if times[block] > (1.0 - threshold) * times[256]:
                block = 256
            entries.append([kb, op, lb, sb, block, 0])
    entries += [[kb, 1, lb, sb, b, p] for kb, op, lb, sb, b, p in entries if op == 0]
    return entries


def tune(key_widths=(4, 8), max_bucket=8, reps=3, quick=False):
    import torch
    from . import datagen
    lib = wc.lib()
    lib.wc_tune_reset()
    entries, report = [], []
    buckets = range(0, max_bucket + 1, 2 if quick else 1)
    for kb in key_widths:
        for lb, lf in enumerate(LOADS):
            for sb in buckets:
                n = size_for_bucket(sb)
                cap = max(16 * n, 1 << 21)  # the batch adds at most 1/16 of capacity
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
                timings = {}
                for op_name, op in OPS.items():
                    best = None
                    for block, bps in CANDIDATES:
                        lib.wc_tune_set(kb, op, lb, sb, block, bps)

                        def fill():
                            t.init()
                            t.insert(bk, bv)
                            torch.cuda.synchronize()

                        if op_name == "insert":
                            ms = []
                            for _ in range(reps):
                                fill()
                                ms.append(_time(lambda: t.insert(nk, nv), 1))
                            ms = min(ms)
                        else:
                            fill()
                            ms = _time(lambda: t.retrieve(q, out), reps)
                        timings[(op_name, block)] = ms
                        if best is None or ms < best[0]:
                            best = (ms, block, bps)
                    entries.append([kb, op, lb, sb, best[1], best[2]])
                    lib.wc_tune_set(kb, op, lb, sb, best[1], best[2])
                report.append({"key_bytes": kb, "load": lf, "n": n,
                               "ms": {f"{k[0]}/{k[1]}": round(v, 4) for k, v in timings.items()}})
                del t
    # counting inserts follow the insert choice
    entries += [[kb, 1, lb, sb, b, p] for kb, op, lb, sb, b, p in entries if op == 0]
    return entries, report


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_FILE)
    ap.add_argument("--quick", action="store_true")
    args = ap.parse_args()
    _, report = tune(quick=args.quick)
    entries = entries_from_measurements(report)
    data = {"device": torch.cuda.get_device_name(0),
            "note": "launch geometry per (key_bytes, op, load bucket, size bucket); "
                    "op 0 insert, 1 counting insert, 2 retrieve; default 256 threads "
                    "unless a candidate is more than 5% faster",
            "entries": entries, "measurements": report}
    with open(args.out, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote %d entries to %s" % (len(entries), args.out))


if __name__ == "__main__":
    main()
