#!/usr/bin/env python3
"""Benchmark of the B200-native warpcore hot path.

Default workload (one step): SingleValueHashTable<uint64,uint64>, CG 8, at
load factor 0.9 (reference capacity 149,963,432 slots): init the table,
insert 2^27 unique uniform keys with uniform values, retrieve 2^27 queries
(50 % hits) in uniform random order.  Metric: Gops/s = keys processed
(inserts + queries) per second, whole job.  Inputs (1 GiB per array) are
larger than L2, so no flush is needed between iterations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload svht64|svht32|hashset64|counting32|bloom64]
                  [--log2n L] [--load F]

--impl reference times the reference algorithm's CPU port (the oracle's
multi-threaded open-addressing table: same MurmurHash, DoubleHashing and
lane order) on the host cores; it is the one other place this script runs
oracle code besides the cpu_baseline leg.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

MASK64 = (1 << 64) - 1
KEY_NOT_FOUND = 1 << 5  # Status::key_not_found (status.cuh:44-68)


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "of measured"
    except Exception:
        return 6650.0, "of fallback"


def measure_l2_copy_gbs(device, mib=32, reps=200):
    """Copy bandwidth between two buffers that L2 holds together (2 x `mib`
    MiB, read + write bytes), CUDA events: the roofline denominator of a
    table that stays in L2."""
    import torch
    n = (mib << 20) // 8
    a = torch.ones(n, dtype=torch.int64, device=device)
    b = torch.empty_like(a)
    for _ in range(10):
        b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        b.copy_(a)
    e1.record()
    torch.cuda.synchronize()
    return 2 * (mib << 20) * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9


def measure_random_atomic_gops(device, array_bytes, n, reps=3):
    """Random 64-bit atomic adds per second (G/s) into an array of
    `array_bytes`, n per launch with indices streamed from memory
    (torch index_add_, one atomicAdd per element), median of `reps` CUDA-event
    timings: an insert claims at least one random slot by an atomic, so this
    rate bounds inserts into a table of that size whatever their bytes."""
    import statistics as st
    import torch
    m = max(int(array_bytes) // 8, 1 << 20)
    g = torch.Generator(device=device)
    g.manual_seed(5)
    buf = torch.zeros(m, dtype=torch.int64, device=device)
    idx = torch.randint(0, m, (n,), device=device, generator=g)
    ones = torch.ones(n, dtype=torch.int64, device=device)
    buf.index_add_(0, idx, ones)
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        buf.index_add_(0, idx, ones)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    del buf, idx, ones
    torch.cuda.empty_cache()
    return n / (st.median(ms) * 1e-3) / 1e9


def profile_traffic(name):
    """dram bytes per launch recorded by the ncu capture summarised under
    profiles/ (line 'dram_bytes_per_launch <kernel-tag> <bytes>')."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 3 and f[0] == "dram_bytes_per_launch" and f[1] == name:
            return float(f[2])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region"""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# synthetic data on the device: warpcore_b200.datagen (int tensors hold the
# unsigned bit patterns)
from warpcore_b200.datagen import (unique_keys32, unique_keys64,  # noqa: E402
                                   uniform_values, zipf_ranks as zipf_ranks_t)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

class Workload:
    """one step = init + insert(n) + retrieve(q) on resident inputs"""

    def __init__(self, kind, log2n, load, rank, device, world=1, shard=False, bucket=2,
                 fill=False, store="aos"):
        import torch
        import warpcore_b200 as wc
        self.kind = kind
        # single-value tables: {key, value} slots ("aos") or a key array and a
        # value array ("soa", SoAStore)
        self.store = store if kind in ("svht32", "svht64") and not shard else "aos"
        self.n = 1 << log2n
        # the table of min capacity 2^L / load under the capacity rule; with
        # `fill` it is filled to a real load of `load` (n = load x capacity)
        # instead of holding 2^L keys
        self.table_min_cap = int(self.n / load)
        if fill and kind in ("svht32", "svht64", "hashset64") and not shard:
            cg = 16 if kind == "hashset64" else 8
            self.n = int(load * wc.valid_capacity(self.table_min_cap, cg))
        # svht32 is the small configuration: every inserted key queried once
        # plus as many absent keys; the others query n keys, half of them hits
        self.q = 2 * self.n if kind == "svht32" else self.n
        self.load = load
        self.device = device
        gen = torch.Generator(device=device)
        gen.manual_seed(1000 + rank)
        seed = 17 + 101 * rank
        kb = 4 if kind in ("svht32", "counting32") else 8
        self.kb = kb
        n, q = self.n, self.q
        if kind in ("svht32", "svht64", "hashset64"):
            mk = unique_keys32 if kb == 4 else unique_keys64
            # ranks draw disjoint index ranges of the same bijection
            keys = mk(rank * (n + q), n + q // 2, 17, device)
            self.keys = keys[:n].contiguous()
            absent = keys[n:n + q // 2]
            self.values = uniform_values(n, kb, gen, device)
            hit_idx = torch.randperm(n, device=device, generator=gen)[: q - q // 2]
            queries = torch.cat([self.keys[hit_idx], absent])
            exp = torch.cat([self.values[hit_idx],
                             torch.zeros(q // 2, dtype=self.values.dtype, device=device)])
            hit = torch.cat([torch.ones(q - q // 2, dtype=torch.bool, device=device),
                             torch.zeros(q // 2, dtype=torch.bool, device=device)])
            perm = torch.randperm(q, device=device, generator=gen)
            self.queries = queries[perm].contiguous()
            self.expected = exp[perm].contiguous()
            self.hit = hit[perm].contiguous()
            if kind == "hashset64":
                self.table = wc.HashSet(self.table_min_cap, key_bytes=8)
                self.out = torch.empty(q, dtype=torch.uint8, device=device)
                self.bytes_insert, self.bytes_retrieve = 8 + 32 + 32, 8 + 1 + 32
            elif shard and kind != "hashset64":
                # sharded over the ranks: keys are routed to their owner
                # (partition kernel + NCCL all-to-all) inside every step
                from warpcore_b200.distributed import DistributedSingleValueHashTable
                self.table = DistributedSingleValueHashTable(int(world * n / load), key_bytes=kb)
                self.out = torch.empty(q, dtype=self.values.dtype, device=device)
                # the table kernel's algorithmic bytes; the timed op also
                # holds the routing (partition + all-to-all)
                self.bytes_insert = kb + kb + 32 + 32
                self.bytes_retrieve = kb + kb + 1 + 32
            else:
                self.table = wc.SingleValueHashTable(self.table_min_cap, key_bytes=kb,
                                                     store=self.store)
                self.out = torch.empty(q, dtype=self.values.dtype, device=device)
                self.bytes_insert = kb + kb + 32 + 32
                self.bytes_retrieve = kb + kb + 1 + 32
        elif kind == "counting32":
            distinct = n >> 4
            self.distinct = distinct
            keys = unique_keys32(0, distinct + (distinct >> 2), seed, device)
            self.dkeys = keys[:distinct]
            ranks = zipf_ranks_t(distinct, 1.1, n, gen, device)
            self.ranks = ranks
            self.keys = self.dkeys[ranks].contiguous()
            self.values = None
            self.queries = keys.contiguous()
            self.q = self.queries.numel()
            self.hist = torch.bincount(ranks, minlength=distinct)
            self.table = wc.CountingHashTable(int(distinct / load), key_bytes=4)
            self.out = torch.empty(self.q, dtype=torch.int32, device=device)
            self.bytes_insert, self.bytes_retrieve = 4 + 32 + 32, 4 + 4 + 1 + 32
        elif kind == "mv32":
            # 2^(L-2) distinct keys with 4 values each, inserted as 2^L pairs
            # in one shuffled batch; retrieve every key plus as many absent
            distinct = n >> 2
            self.distinct = distinct
            keys = unique_keys32(0, 2 * distinct, seed, device)
            idx = (torch.arange(n, device=device) % distinct)[
                torch.randperm(n, device=device, generator=gen)]
            self.keys = keys[:distinct][idx].contiguous()
            self.values = uniform_values(n, 4, gen, device)
            self.queries = keys.contiguous()
            self.q = 2 * distinct
            # per-key checksums of the values: sum and sum of squares (wrapping)
            v64 = self.values.to(torch.int64) & 0xFFFFFFFF
            self.exp_sum = torch.zeros(distinct, dtype=torch.int64, device=device).index_add_(0, idx, v64)
            self.exp_sq = torch.zeros(distinct, dtype=torch.int64, device=device).index_add_(0, idx, v64 * v64)
            self.table = wc.MultiValueHashTable(int(n / load), key_bytes=4)
            self.begin = torch.empty(self.q, dtype=torch.int64, device=device)
            self.end = torch.empty(self.q, dtype=torch.int64, device=device)
            self.out = torch.empty(n, dtype=torch.int32, device=device)
            # insert: pair in + one window sector read + written; retrieve:
            # key in, offsets out, two window sectors (count and values
            # passes), 2 values per query out on average
            self.bytes_insert, self.bytes_retrieve = 4 + 4 + 32 + 32, 4 + 16 + 32 + 32 + 8
        elif kind == "mb32":
            # the reference's multi_bucket benchmark: 2^L values, key of input
            # i = i mod 2^(L-3) + 1 (8 values per key, copies 2^(L-3) apart);
            # queries 1 .. 2^L (one in 8 present); table capacity for key
            # load 0.8 of a B-bucket table; values uniform and non-zero
            distinct = n >> 3
            self.distinct = distinct
            self.per_key = 8
            idx = torch.arange(n, device=device) % distinct
            self.keys = (idx + 1).to(torch.int32).contiguous()
            self.values = uniform_values(n, 4, gen, device)
            self.values[self.values == 0] = 1
            self.queries = (torch.arange(n, device=device) + 1).to(torch.int32).contiguous()
            self.q = n
            v64 = self.values.to(torch.int64) & 0xFFFFFFFF
            self.exp_sum = torch.zeros(distinct, dtype=torch.int64, device=device).index_add_(0, idx, v64)
            self.exp_sq = torch.zeros(distinct, dtype=torch.int64, device=device).index_add_(0, idx, v64 * v64)
            b = bucket
            self.bucket = b
            cap = int(n * (4 + 4) / (4 + 4 * b) / load)
            self.table = wc.MultiBucketHashTable(cap, key_bytes=4, value_bytes=4, bucket_size=b)
            self.min_cap = cap
            self.begin = torch.empty(self.q, dtype=torch.int64, device=device)
            self.end = torch.empty(self.q, dtype=torch.int64, device=device)
            self.out = torch.empty(n, dtype=torch.int32, device=device)
            # insert: pair in + the key window's sector read and written +
            # the bucket's sector written; retrieve: key in, offsets out,
            # the window sector in the count and value passes, one value out
            # per query on average
            self.bytes_insert, self.bytes_retrieve = 4 + 4 + 32 + 32, 4 + 16 + 32 + 32 + 4
        elif kind == "bl32":
            # the reference's bucket_list benchmark: 2^L values, key of input
            # i = i mod 2^(L-3) + 1 (8 values per key); key table for load 0.9
            # of the distinct keys, value pool for load 0.5 of the values;
            # store bits 29 / 18 / 15, grow factor 1.1, first bucket 1
            distinct = n >> 3
            self.distinct = distinct
            self.per_key = 8
            idx = torch.arange(n, device=device) % distinct
            self.keys = (idx + 1).to(torch.int32).contiguous()
            self.values = uniform_values(n, 4, gen, device)
            self.queries = (torch.arange(n, device=device) + 1).to(torch.int32).contiguous()
            self.q = n
            v64 = self.values.to(torch.int64) & 0xFFFFFFFF
            self.exp_sum = torch.zeros(distinct, dtype=torch.int64, device=device).index_add_(0, idx, v64)
            self.exp_sq = torch.zeros(distinct, dtype=torch.int64, device=device).index_add_(0, idx, v64 * v64)
            self.key_cap, self.value_cap = int(distinct / 0.9), int(n / 0.5)
            self.table = wc.BucketListHashTable(self.key_cap, self.value_cap, key_bytes=4,
                                                value_bytes=4, grow_factor=1.1, min_bucket_size=1,
                                                bits=(29, 18, 15))
            self.begin = torch.empty(self.q, dtype=torch.int64, device=device)
            self.end = torch.empty(self.q, dtype=torch.int64, device=device)
            self.out = torch.empty(n, dtype=torch.int32, device=device)
            # insert: pair in + the key window's sector + the handle's sector
            # + the pool sector written; retrieve: key in, offsets out, key
            # window and handle sectors in the count and value passes, one
            # value out per query on average
            self.bytes_insert, self.bytes_retrieve = 4 + 4 + 32 + 32 + 32, 4 + 16 + 4 * 32 + 4
        elif kind == "bloom64":
            keys = unique_keys64(0, 2 * n, seed, device)
            self.keys = keys[:n].contiguous()
            self.queries = torch.cat([keys[n:], keys[:n]]).contiguous()
            self.q = 2 * n
            self.values = None
            # 16 bits per key, 512-bit blocks, 8 bits per key
            self.table = wc.BloomFilter(16 * n, 8, key_bytes=8, slot_bytes=8, cg_size=8)
            self.out = torch.empty(self.q, dtype=torch.uint8, device=device)
            self.bytes_insert, self.bytes_retrieve = 8 + 64 + 64, 8 + 1 + 64
        else:
            raise ValueError(kind)
        torch.cuda.synchronize()

    # -- one step's operations --
    def init(self, stream):
        if self.sharded:
            self.table.init()
        else:
            self.table.init(stream=stream)

    def insert(self, stream):
        if self.sharded:
            self.table.insert(self.keys, self.values)
        elif self.kind in ("svht32", "svht64", "mv32", "mb32", "bl32"):
            self.table.insert(self.keys, self.values, stream=stream)
        else:
            self.table.insert(self.keys, stream=stream)

    def retrieve(self, stream):
        if self.sharded:
            self.table.retrieve(self.queries, self.out)
        elif self.kind in ("mv32", "mb32", "bl32"):
            self.table.retrieve(self.queries, self.begin, self.end, self.out, stream=stream)
        else:
            self.table.retrieve(self.queries, self.out, stream=stream)

    @property
    def sharded(self):
        return type(self.table).__name__ == "DistributedSingleValueHashTable"

    def answers_ok(self, out):
        """the retrieve output `out` (written by any implementation after an
        insert of this workload) holds the right answers"""
        import torch
        if self.kind in ("svht32", "svht64"):
            return (bool(torch.equal(out[self.hit], self.expected[self.hit]))
                    and bool((out[~self.hit] == -1).all()))
        if self.kind == "hashset64":
            return bool((out == self.hit.to(torch.uint8)).all())
        if self.kind == "counting32":
            got = out[: self.distinct].to(torch.int64)
            return (bool(torch.equal(got, self.hist))
                    and bool((out[self.distinct:] == 0).all()))
        if self.kind == "bloom64":
            return bool((out[self.n:] == 1).all())
        if self.kind in ("mv32", "mb32", "bl32"):
            return self.mv_ok(self.begin, self.end, out)
        return False

    def mv_ok(self, begin, end, values):
        """every key has its values (per-key count, sum and sum of
        squares), absent keys none"""
        import torch
        d = self.distinct
        per = getattr(self, "per_key", 4)
        cnt = end - begin
        if not (bool((cnt[:d] == per).all()) and bool((cnt[d:] == 0).all())):
            return False
        v64 = values[: per * d].to(torch.int64) & 0xFFFFFFFF
        seg = torch.repeat_interleave(torch.arange(self.q, device=v64.device), cnt)
        s1 = torch.zeros(d, dtype=torch.int64, device=v64.device).index_add_(0, seg, v64)
        s2 = torch.zeros(d, dtype=torch.int64, device=v64.device).index_add_(0, seg, v64 * v64)
        return bool(torch.equal(s1, self.exp_sum)) and bool(torch.equal(s2, self.exp_sq))

    def verify(self):
        """size-independent properties of one fresh step; the step's answers
        stay in self.answers for the exact comparison with the reference
        build (reference_gpu)"""
        import torch
        s = torch.cuda.current_stream()
        self.init(s)
        self.insert(s)
        self.answers = {}
        if self.kind in ("svht32", "svht64"):
            self.out.fill_(-1)
            if self.sharded:
                self.retrieve(s)
            else:
                st = torch.zeros(self.q, dtype=torch.int32, device=self.out.device)
                self.table.retrieve(self.queries, self.out, stream=s, status_out=st)
                self.answers["status"] = st
                if not bool(torch.equal(st != 0, ~self.hit)):
                    return False
                if not bool((st[~self.hit] == KEY_NOT_FOUND).all()):
                    return False
            torch.cuda.synchronize()
            self.answers["out"] = self.out.clone()
            ok_hits = bool(torch.equal(self.out[self.hit], self.expected[self.hit]))
            ok_miss = bool((self.out[~self.hit] == -1).all())
            ok_size = self.table.size() == self.n * (self.table.world if self.sharded else 1)
            return ok_hits and ok_miss and ok_size
        if self.kind == "hashset64":
            self.out.fill_(7)
            self.retrieve(s)
            torch.cuda.synchronize()
            self.answers["out"] = self.out.clone()
            return bool((self.out == self.hit.to(torch.uint8)).all()) and self.table.size() == self.n
        if self.kind == "counting32":
            self.out.fill_(0)
            st = torch.zeros(self.q, dtype=torch.int32, device=self.out.device)
            self.table.retrieve(self.queries, self.out, stream=s, status_out=st)
            torch.cuda.synchronize()
            self.answers["out"] = self.out.clone()
            self.answers["status"] = st
            got = self.out[: self.distinct].to(torch.int64)
            present = self.hist > 0
            # the device histogram of the stream against its CPU histogram
            # (np.bincount over all ranks), then the table against it
            cpu_hist = np.bincount(self.ranks.cpu().numpy(), minlength=self.distinct)
            self.cpu_hist_ok = bool(np.array_equal(cpu_hist, self.hist.cpu().numpy()))
            ok = self.cpu_hist_ok and bool(torch.equal(got[present], self.hist[present]))
            # keys never drawn and the absent keys: untouched, key_not_found
            ok = ok and bool((self.out[self.distinct:] == 0).all()) and bool((got[~present] == 0).all())
            miss = torch.cat([~present, torch.ones(self.q - self.distinct, dtype=torch.bool,
                                                   device=st.device)])
            ok = ok and bool(torch.equal(st != 0, miss)) and bool((st[miss] == KEY_NOT_FOUND).all())
            self.distinct_drawn = int(present.sum())
            return ok and self.table.size() == self.distinct_drawn
        if self.kind == "bloom64":
            self.out.fill_(7)
            self.retrieve(s)
            torch.cuda.synchronize()
            self.answers["out"] = self.out.clone()
            self.answers["words"] = self.table.words_tensor().clone()
            # measured false-positive rate: the absent half of the queries
            self.fpr_measured = float(self.out[: self.n].double().mean())
            return bool((self.out[self.n:] == 1).all()) and bool((self.out <= 1).all())
        if self.kind in ("mv32", "mb32", "bl32"):
            self.retrieve(s)
            torch.cuda.synchronize()
            size = self.table.num_values() if self.kind == "bl32" else self.table.size()
            return (self.mv_ok(self.begin, self.end, self.out) and size == self.n
                    and self.table.num_keys() == self.distinct)
        return False


def reference_gpu(wl, reps=5):
    """Time the reference warpcore compiled for sm_100a
    (baseline/_ref/libwarpcore_ref_bench.so, built by
    baseline/build_ref_gpu.sh) on the same resident inputs, with the
    reference's own bulk methods: min over `reps`, table re-initialised
    untimed before each insert (benchmark_common.cuh:116-199)."""
    import ctypes
    import torch
    path = os.path.join(ROOT, "baseline", "_ref", "libwarpcore_ref_bench.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    f32 = ctypes.c_float
    ti, tr, cap = f32(), f32(), ctypes.c_uint64(0)
    u64 = ctypes.c_uint64
    vp = ctypes.c_void_p
    torch.cuda.synchronize()
    out = torch.empty_like(wl.out)
    min_cap = wl.table_min_cap if wl.kind != "counting32" else int(wl.distinct / wl.load)
    rb = re_ = None
    st = words = None
    nslots = ctypes.c_uint64(0)
    if wl.kind in ("svht64", "svht32"):
        # misses must stay untouched: the same fill as our verification run
        out.fill_(-1)
        st = torch.zeros(wl.q, dtype=torch.int32, device=out.device)
        if wl.store == "soa":
            fn = lib.ref_svht64_soa_run if wl.kind == "svht64" else lib.ref_svht32_soa_run
        else:
            fn = lib.ref_svht64_run if wl.kind == "svht64" else lib.ref_svht32_run
        rc = fn(vp(wl.keys.data_ptr()), vp(wl.values.data_ptr()), u64(wl.n),
                vp(wl.queries.data_ptr()), u64(wl.q), vp(out.data_ptr()), u64(min_cap),
                ctypes.c_int(reps), ctypes.byref(ti), ctypes.byref(tr), ctypes.byref(cap),
                vp(st.data_ptr()))
    elif wl.kind == "hashset64":
        out.fill_(7)
        rc = lib.ref_hashset64_run(vp(wl.keys.data_ptr()), u64(wl.n), vp(wl.queries.data_ptr()),
                                   u64(wl.q), vp(out.data_ptr()), u64(min_cap), ctypes.c_int(reps),
                                   ctypes.byref(ti), ctypes.byref(tr), ctypes.byref(cap))
    elif wl.kind == "counting32":
        out.zero_()
        st = torch.zeros(wl.q, dtype=torch.int32, device=out.device)
        rc = lib.ref_counting32_run(vp(wl.keys.data_ptr()), u64(wl.n), vp(wl.queries.data_ptr()),
                                    u64(wl.q), vp(out.data_ptr()), u64(min_cap), ctypes.c_int(reps),
                                    ctypes.byref(ti), ctypes.byref(tr), ctypes.byref(cap),
                                    vp(st.data_ptr()))
    elif wl.kind == "mv32":
        rb, re_ = torch.empty_like(wl.begin), torch.empty_like(wl.end)
        num = ctypes.c_uint64(0)
        rc = lib.ref_mv32_run(vp(wl.keys.data_ptr()), vp(wl.values.data_ptr()), u64(wl.n),
                              vp(wl.queries.data_ptr()), u64(wl.q), vp(rb.data_ptr()),
                              vp(re_.data_ptr()), vp(out.data_ptr()), ctypes.byref(num),
                              u64(min_cap), ctypes.c_int(reps), ctypes.byref(ti), ctypes.byref(tr),
                              ctypes.byref(cap))
    elif wl.kind == "mb32":
        rb, re_ = torch.empty_like(wl.begin), torch.empty_like(wl.end)
        num = ctypes.c_uint64(0)
        rc = lib.ref_mb32_run(vp(wl.keys.data_ptr()), vp(wl.values.data_ptr()), u64(wl.n),
                              vp(wl.queries.data_ptr()), u64(wl.q), vp(rb.data_ptr()),
                              vp(re_.data_ptr()), vp(out.data_ptr()), ctypes.byref(num),
                              u64(wl.min_cap), ctypes.c_uint32(wl.bucket), ctypes.c_int(reps),
                              ctypes.byref(ti), ctypes.byref(tr), ctypes.byref(cap))
    elif wl.kind == "bl32":
        rb, re_ = torch.empty_like(wl.begin), torch.empty_like(wl.end)
        num = ctypes.c_uint64(0)
        rc = lib.ref_bl32_run(vp(wl.keys.data_ptr()), vp(wl.values.data_ptr()), u64(wl.n),
                              vp(wl.queries.data_ptr()), u64(wl.q), vp(rb.data_ptr()),
                              vp(re_.data_ptr()), vp(out.data_ptr()), ctypes.byref(num),
                              u64(wl.key_cap), u64(wl.value_cap), ctypes.c_int(reps),
                              ctypes.byref(ti), ctypes.byref(tr), ctypes.byref(cap))
    elif wl.kind == "bloom64":
        out.fill_(7)
        words = torch.full((wl.table.num_slots(),), -1, dtype=torch.int64, device=out.device)
        rc = lib.ref_bloom64_run(vp(wl.keys.data_ptr()), u64(wl.n), vp(wl.queries.data_ptr()),
                                 u64(wl.q), vp(out.data_ptr()), u64(16 * wl.n), u64(8),
                                 ctypes.c_int(reps), ctypes.byref(ti), ctypes.byref(tr),
                                 vp(words.data_ptr()), ctypes.byref(nslots))
    else:
        return None
    torch.cuda.synchronize()
    if rc != 0:
        return {"error": "CUDA error %d" % rc}
    # the reference's answers on the same inputs must equal ours
    compared = {}
    if wl.kind in ("mv32", "mb32", "bl32"):
        same = wl.mv_ok(rb, re_, out)
    else:
        ans = getattr(wl, "answers", {})
        same = wl.answers_ok(out)
        if "out" in ans:
            # every output element, misses included (same fill before the call)
            compared["outputs"] = bool(torch.equal(out, ans["out"]))
        if st is not None and "status" in ans:
            compared["statuses"] = bool(torch.equal(st, ans["status"]))
        if words is not None:
            ours = wl.table.words_tensor()
            compared["filter_words"] = int(nslots.value)
            compared["words_equal"] = (int(nslots.value) == ours.numel()
                                       and bool(torch.equal(words, ours)))
        same = same and all(v for k, v in compared.items() if k != "filter_words")
    ins_g = wl.n / (ti.value * 1e-3) / 1e9
    ret_g = wl.q / (tr.value * 1e-3) / 1e9
    r = {"insert_gops": round(ins_g, 4), "retrieve_gops": round(ret_g, 4),
         "value": round((wl.n + wl.q) / ((ti.value + tr.value) * 1e-3) / 1e9, 4),
         "insert_ms": round(ti.value, 4), "retrieve_ms": round(tr.value, 4),
         "capacity": int(cap.value) if cap.value else None, "reps": reps,
         "timing": "cudaEvent min of %d on the reference's own bulk methods" % reps,
         "same_answers": same}
    if compared:
        r["compared"] = compared
    return r


WORKLOAD_NAMES = {
    "svht64": "SingleValueHashTable<u64,u64> CG8 LF{LF}: insert 2^{L} + retrieve 2^{L} (50% hit)",
    "svht32": "SingleValueHashTable<u32,u32> CG8 LF{LF}: insert 2^{L} + retrieve 2^{L1} "
              "(every inserted key + 2^{L} absent)",
    "hashset64": "HashSet<u64> CG16 LF{LF}: insert 2^{L} + contains 2^{L} (50% hit)",
    "counting32": "CountingHashTable<u32,u32> CG4 LF0.85: insert 2^{L} Zipf(1.1) + retrieve distinct+absent",
    "bloom64": "BloomFilter<u64,Murmur64,u64,CG8> 16 bits/key k=8: insert 2^{L} + query 2^{L1}",
    "mv32": "MultiValueHashTable<u32,u32> CG8 LF{LF}: insert 2^{L} pairs (4 values per key, "
            "one shuffled batch) + retrieve every key and as many absent keys",
    "mb32": "MultiBucketHashTable<u32,u32> CG8 bucket {B}, key LF{LF}: insert 2^{L} values "
            "(key i mod 2^{L3} + 1, 8 per key) + retrieve keys 1..2^{L} (two-phase, offsets)",
    "bl32": "BucketListHashTable<u32,u32> CG8 BucketListStore<29,18,15> grow 1.1: insert 2^{L} "
            "values (key i mod 2^{L3} + 1, 8 per key; key LF 0.9, pool LF 0.5) + retrieve keys "
            "1..2^{L} (two-phase, offsets)",
    "gen": "on-device generators: unique + uniform u64 keys, Zipf(1.1) ranks",
    "served": "4096 SingleValueHashTable<u32,u32> (caps log-uniform 2^10..2^22, LF 0.85), "
              "Poisson requests (batch 2^6..2^18, 30% insert, 80% hit): persistent kernel and "
              "continuous batching vs plain launches",
}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != world and world > 1:
        log("warning: --gpus %d but WORLD_SIZE %d" % (args.gpus, world))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=device)
    elif args.shard:
        import datetime
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                                world_size=1, timeout=datetime.timedelta(seconds=120),
                                device_id=device)

    import warpcore_b200  # noqa: F401
    warpcore_b200.lib()

    wl = Workload(args.workload, args.log2n, args.load, rank, device, world, bucket=args.bucket,
                  shard=args.shard or world > 1, fill=args.fill, store=args.store)
    stream = torch.cuda.Stream(device=device)
    torch.cuda.synchronize()
    verified = wl.verify()

    # warm-up
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            wl.init(stream)
            wl.insert(stream)
            wl.retrieve(stream)
    torch.cuda.synchronize()

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    launches0 = warpcore_b200.launch_count()
    wall0 = time.perf_counter()
    t0.record(stream)
    with torch.cuda.stream(stream):  # the sharded table runs on the current stream
        for k in range(args.steps):
            ev[k][0].record(stream)
            wl.init(stream)
            ev[k][1].record(stream)
            wl.insert(stream)
            ev[k][2].record(stream)
            wl.retrieve(stream)
            ev[k][3].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    launches = warpcore_b200.launch_count() - launches0
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = t0.elapsed_time(t1)
    init_ms = [e[0].elapsed_time(e[1]) for e in ev]
    ins_ms = [e[1].elapsed_time(e[2]) for e in ev]
    ret_ms = [e[2].elapsed_time(e[3]) for e in ev]
    if world > 1:
        tt = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    ops_step = wl.n + wl.q
    value = world * ops_step * args.steps / (total_ms * 1e-3) / 1e9

    # end to end through the public API with host buffers
    table_ops = table_wide_ops(wl, stream) if (world == 1 and not wl.sharded) else None
    e2e = run_e2e(wl, stream, args, world) if not args.no_e2e else None
    ref_gpu = reference_gpu(wl) if (rank == 0 and not args.no_ref_gpu) else None

    if world > 1:
        dist.barrier()
    if rank == 0:
        peak, peak_src = measured_peak()
        ins_avg = statistics.mean(ins_ms)
        ret_avg = statistics.mean(ret_ms)
        if ins_avg >= ret_avg:
            dom, dom_ms, dom_bytes, dom_ops = "insert", ins_avg, wl.bytes_insert, wl.n
        else:
            dom, dom_ms, dom_bytes, dom_ops = "retrieve", ret_avg, wl.bytes_retrieve, wl.q
        achieved = dom_bytes * dom_ops / (dom_ms * 1e-3) / 1e9
        tag = "%s_%s_2p%d" % (args.workload, dom, args.log2n)
        traffic = profile_traffic(tag)
        # a table that L2 holds is bounded by L2, not HBM: its denominator is
        # an L2-resident copy measured now
        table_bytes = getattr(wl.table, "info", None) and _table_bytes(wl.table)
        l2_resident = bool(table_bytes) and table_bytes <= torch.cuda.get_device_properties(device).L2_cache_size
        hbm_peak = peak
        if l2_resident:
            peak, peak_src = round(measure_l2_copy_gbs(device), 1), "measured L2-resident copy (2 x 32 MiB)"
        # the host baseline is timed on rank 0 of a one-GPU run only
        cpu = cpu_baseline(args) if not args.no_cpu and world == 1 else None
        # inserts: the rate of random atomics into an array of the table's
        # size (in DRAM, or in L2 for a table that L2 holds) bounds them too
        # (one claim per key); at least 2^24 atomics, so that the rate is the
        # throughput and not the ramp of a short launch
        atomic = None
        if (dom == "insert" and table_bytes
                and args.workload in ("svht32", "svht64", "hashset64")):
            n_atomic = max(dom_ops, 1 << 24)
            rate = measure_random_atomic_gops(device, table_bytes, n_atomic)
            ins_rate = dom_ops / (dom_ms * 1e-3) / 1e9
            atomic = {"random_atomic_gops": round(rate, 3),
                      "insert_gops": round(ins_rate, 3),
                      "frac": round(ins_rate / rate, 4),
                      "measured": "torch index_add_ of %d int64 ones at random indices into "
                                  "%d bytes%s (one atomicAdd each), median of 3"
                                  % (n_atomic, table_bytes, " (L2-resident)" if l2_resident else "")}
        line = {
            "metric": "insert+retrieve Gops/s (keys processed per second, whole job)",
            "value": round(value, 4),
            "unit": "Gops/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u64" if wl.kb == 8 else "u32",
            "data": "synthetic (seeded uniform unique keys, uniform values; inputs resident in HBM)",
            "config": {
                "workload": WORKLOAD_NAMES[args.workload].format(L=args.log2n, L1=args.log2n + 1, L3=args.log2n - 3,
                                                         LF=args.load, B=args.bucket)
                            + ("; filled: %d keys (load x capacity) instead of 2^%d" % (wl.n, args.log2n)
                               if wl.n != (1 << args.log2n) and args.fill else "")
                            + ("; SoAStore (key array + value array) on both sides"
                               if wl.store == "soa" else ""),
                "store": wl.store,
                "capacity": int(wl.table.capacity) if hasattr(wl.table, "capacity") else None,
                "keys_inserted": wl.n,
                "real_load": (round(wl.n / wl.table.capacity, 4)
                              if args.workload in ("svht32", "svht64", "hashset64")
                              and hasattr(wl.table, "capacity") else None),
                "filled": bool(args.fill),
                "ops_per_step": ops_step,
                "l2": "inputs larger than L2 (no flush)" if args.log2n >= 24 else "inputs may be L2-resident",
                "parallelism": ("table sharded over %d GPU(s): keys routed to owners by "
                                "partition kernel + NCCL all-to-all in every step" % world)
                               if wl.sharded else "single GPU",
            },
            "insert_gops": round(wl.n / (statistics.mean(ins_ms) * 1e-3) / 1e9, 4),
            "retrieve_gops": round(wl.q / (statistics.mean(ret_ms) * 1e-3) / 1e9, 4),
            "init_ms": round(statistics.mean(init_ms), 4),
            "insert_ms": round(statistics.mean(ins_ms), 4),
            "retrieve_ms": round(statistics.mean(ret_ms), 4),
            "verified": verified,
            "roofline": {
                "bound": "l2" if l2_resident else "hbm",
                "kernel": dom,
                "achieved": round(achieved, 2),
                "peak": peak,
                "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "peak_source": peak_src,
                "algorithmic_bytes_per_op": dom_bytes,
                "traffic": traffic,
                "frac_of_hbm": round(achieved / hbm_peak, 4),
                "table_bytes": table_bytes or None,
                "atomic_ceiling": atomic,
            },
            "cpu_baseline": cpu,
            "reference_gpu_build": ref_gpu,
            "table_wide_ops": table_ops,
            "e2e": e2e,
            # this library's kernels launched inside the timed region, as the
            # library counts them (wc_launch_count)
            "gpu_launches": launches,
            "clocks": clocks,
            "wall_s": round(wall, 3),
        }
        if wl.kind == "bloom64":
            line["fpr"] = bloom_fpr_report(wl)
        if wl.kind == "counting32":
            line["config"]["distinct_keys"] = wl.distinct
            line["config"]["distinct_drawn"] = getattr(wl, "distinct_drawn", None)
            line["cpu_histogram_equal"] = getattr(wl, "cpu_hist_ok", None)
        print(json.dumps(line), flush=True)
    if world > 1 or args.shard:
        dist.barrier()
        dist.destroy_process_group()


def _wrapping_sum(x):
    """sum of a key or value tensor as unsigned 64-bit words, modulo 2^64"""
    import torch
    if x.dtype == torch.int32:
        x = x.to(torch.int64) & 0xFFFFFFFF
    return int(x.sum().item()) & ((1 << 64) - 1)


def multi_value_keys_op(wl, stream, reps=3):
    """retrieve_all_keys of a multi-value table after the timed steps
    (multi_value_hash_table.cuh:561-598; bucket_list_hash_table.cuh and
    multi_bucket_hash_table.cuh through gpu_engine.cuh:51-93): each stored
    key once, CUDA events around the blocking call, best of `reps`.  The
    keys must be the distinct inserted keys (count and sum modulo 2^64)."""
    import torch
    t = wl.table
    nk = int(t.num_keys())
    kout = torch.empty(nk, dtype=wl.keys.dtype, device=wl.keys.device)
    expect = _wrapping_sum(torch.unique(wl.keys))
    ms, ok = [], nk == wl.distinct
    for _ in range(reps):
        kout.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        got = t.retrieve_all_keys(kout, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
        ok = ok and got == nk and _wrapping_sum(kout) == expect
    return {"retrieve_all_keys_ms": round(min(ms), 4), "keys": nk,
            "retrieve_all_keys_gkeys": round(nk / (min(ms) * 1e-3) / 1e9, 4),
            "retrieve_all_keys_verified": ok,
            "timing": "CUDA events around the blocking call, best of %d" % reps}


def table_wide_ops(wl, stream, reps=3):
    """Table-wide operations on the workload's table after its insert
    (single_value_hash_table.cuh:426-496, 535-592, 606-651): retrieve_all of
    every stored pair and the erase of every inserted key (CUDA events on
    the launching stream, table re-filled untimed before each repetition,
    best of `reps`), and the time of size() (the maintained count) against
    size_scan() (a scan of the slot array) on the full table.  The dump must
    hold as many entries as the table and, for the single-value tables and
    the set, the inserted keys and values (equal sums modulo 2^64; the
    counting table: counts summing to the keys inserted).  After the erase
    both sizes must be 0."""
    import torch
    if wl.kind in ("mv32", "mb32", "bl32"):
        return multi_value_keys_op(wl, stream, reps)
    if wl.kind not in ("svht32", "svht64", "hashset64", "counting32"):
        return None
    t = wl.table
    best, sizes_ok = None, True
    size_ms, scan_ms, dump_ms = [], [], []
    dump_ok = True
    kdt = torch.int64 if t.key_bytes == 8 else torch.int32
    has_val = wl.kind != "hashset64"
    vdt = wl.values.dtype if wl.values is not None else torch.int32
    for _ in range(reps):
        wl.init(stream)
        wl.insert(stream)
        torch.cuda.synchronize()
        for fn, acc in ((t.size, size_ms), (t.size_scan, scan_ms)):
            t0 = time.perf_counter()
            fn()
            acc.append((time.perf_counter() - t0) * 1e3)
        live = int(t.size())
        kout = torch.empty(live, dtype=kdt, device=wl.keys.device)
        vout = torch.empty(live, dtype=vdt, device=wl.keys.device) if has_val else None
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        got = t.retrieve_all(kout, vout, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        dump_ms.append(a.elapsed_time(b))
        ok = got == live
        if wl.kind == "counting32":
            ok = ok and _wrapping_sum(vout) == wl.keys.numel()
        else:
            ok = ok and got == wl.keys.numel() and _wrapping_sum(kout) == _wrapping_sum(wl.keys)
            if has_val:
                ok = ok and _wrapping_sum(vout) == _wrapping_sum(wl.values)
        dump_ok = dump_ok and ok
        del kout, vout
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        t.erase(wl.keys, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
        sizes_ok = sizes_ok and t.size() == 0 and t.size_scan() == 0
    return {"retrieve_all_ms": round(min(dump_ms), 4), "retrieved_all": int(got),
            "retrieve_all_gops": round(got / (min(dump_ms) * 1e-3) / 1e9, 4),
            "retrieve_all_verified": dump_ok,
            "retrieve_all_timing": "CUDA events around the blocking call, best of %d" % reps,
            "erase_gops": round(wl.keys.numel() / (best * 1e-3) / 1e9, 4),
            "erase_ms": round(best, 4), "erased_keys": int(wl.keys.numel()),
            "size_ms": round(min(size_ms), 4), "size_scan_ms": round(min(scan_ms), 4),
            "size_timing": "host wall clock of the blocking call, best of %d" % reps,
            "sizes_zero_after_erase": sizes_ok}


def bloom_fpr_report(wl):
    """False-positive rate of the filter after the step's inserts: measured
    on the absent half of the queries, beside the reference's estimator
    (bloom_filter.cuh:342-408).  The library's fpr() follows the reference
    literally and overflows to NaN at this size (its binomial coefficient is
    a product of n factors); the same sum is evaluated here with log-space
    binomial probabilities."""
    from scipy.stats import binom
    nb = int(wl.table.num_blocks())
    m = int(wl.table.num_bits()) // nb          # bits per block
    k = int(wl.table.k())
    n = wl.n
    i = np.arange(0, 5 * n // nb)
    base = (1.0 - np.power(1.0 - 1.0 / m, i * k)) ** k
    est = float(np.sum(binom.pmf(i, n, 1.0 / nb) * base))
    lib_fpr = wl.table.fpr(n)
    return {"measured": getattr(wl, "fpr_measured", None),
            "absent_queries": wl.n,
            "estimate": est,
            "estimate_how": "the reference's pattern-blocked estimator, log-space binomials",
            "library_fpr_call": None if math.isnan(lib_fpr) else lib_fpr}


def _table_bytes(table):
    """device bytes of a table's slot array (or a filter's words)"""
    try:
        inf = table.info()
    except Exception:
        return 0
    if hasattr(inf, "capacity") and hasattr(inf, "slot_bytes"):
        return int(inf.capacity) * int(inf.slot_bytes)
    if hasattr(inf, "local_blocks"):
        return int(inf.local_blocks) * int(inf.cg_size) * int(inf.slot_bytes)
    return 0


def run_e2e(wl, stream, args, world):
    """Same workload through the public API with pinned host buffers: every
    step copies its inputs host->device, runs init + insert + retrieve and
    copies the results back."""
    import torch
    hk = wl.keys.cpu().pin_memory()
    hv = wl.values.cpu().pin_memory() if wl.values is not None else None
    hq = wl.queries.cpu().pin_memory()
    ho = torch.empty(wl.out.shape, dtype=wl.out.dtype).pin_memory()
    dk = torch.empty_like(wl.keys)
    dv = torch.empty_like(wl.values) if wl.values is not None else None
    dq = torch.empty_like(wl.queries)
    h2d = hk.numel() * hk.element_size() + hq.numel() * hq.element_size()
    if hv is not None:
        h2d += hv.numel() * hv.element_size()
    d2h = ho.numel() * ho.element_size()
    keys0, vals0, q0 = wl.keys, wl.values, wl.queries
    steps = max(1, min(args.steps, 3))
    piped = hasattr(wl.table, "insert_from_host") and not wl.sharded and wl.kind not in ("mv32", "mb32", "bl32")
    if piped:
        # host buffers straight into the C ABI: chunks of 2^22 keys, copy-in
        # / kernel / copy-out overlapped; a miss gets the fill value the
        # device-side verification uses (-1, or 0 for counts)
        import warpcore_b200 as wc
        pipe = wc.HostPipe(1 << 22, 3)
        fill = 0 if wl.kind == "counting32" else -1
        hvals = hv if wl.kind in ("svht32", "svht64") else None

        def step():
            wl.init(stream)
            wl.table.insert_from_host(pipe, hk, hvals, stream=stream)
            wl.table.retrieve_to_host(pipe, hq, ho, miss_fill=fill if wl.kind != "hashset64" else None,
                                      stream=stream)
    else:
        def step():
            dk.copy_(hk, non_blocking=True)
            if dv is not None:
                dv.copy_(hv, non_blocking=True)
            dq.copy_(hq, non_blocking=True)
            wl.keys, wl.values, wl.queries = dk, dv, dq
            wl.init(stream)
            wl.insert(stream)
            wl.retrieve(stream)
            ho.copy_(wl.out, non_blocking=True)

    with torch.cuda.stream(stream):
        step()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            step()
        b.record(stream)
        torch.cuda.synchronize()
    wl.keys, wl.values, wl.queries = keys0, vals0, q0
    ms = a.elapsed_time(b)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=wl.keys.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)  # slowest rank
        ms = float(t.item())
    ops = (wl.n + wl.q) * steps * world
    verified = None
    if piped and wl.kind in ("svht32", "svht64"):
        # the host output of the last step: hits hold their values, misses -1
        exp, hit = wl.expected.cpu(), wl.hit.cpu()
        verified = bool(torch.equal(ho[hit], exp[hit])) and bool((ho[~hit] == -1).all())
    if piped:
        if wl.kind not in ("svht32", "svht64") and hv is not None:
            h2d -= hv.numel() * hv.element_size()
        api = ("wc_table_insert_host + wc_table_retrieve_host (C ABI, pinned host buffers, "
               "2^22-key chunks, copies overlapping the kernels)")
    else:
        api = "warpcore_b200 Python binding over the C ABI (copies, then device calls)"
    return {"value": round(ops / (ms * 1e-3) / 1e9, 4), "unit": "Gops/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "steps": steps, "api": api, "verified": verified}


# ---------------------------------------------------------------------------
# CPU legs (oracle port of the reference algorithm)
# ---------------------------------------------------------------------------

def cpu_sample(args, threads, reps):
    """bounded sample of the workload on the host cores: insert + retrieve
    2^log2s keys through the oracle's multi-threaded port"""
    import numpy as np
    from oracle import oracle as o
    kb = 4 if args.workload in ("svht32", "counting32") else 8
    log2s = args.cpu_log2n
    n = 1 << log2s
    keys = o.gen_unique_keys(kb, n + n // 2, 31)
    ins = keys[:n]
    vals = o.gen_uniform(kb, n, 32)
    rng = np.random.default_rng(5)
    q = np.concatenate([ins[rng.permutation(n)[: n - n // 2]], keys[n:]])
    q = q[rng.permutation(n)]
    cap = o.valid_capacity(int(n / args.load), 8)
    t = o.MTTable(kb, cap, 8)
    out = np.zeros(n, dtype=keys.dtype)
    found = np.zeros(n, dtype=np.uint8)
    best = None
    for _ in range(reps):
        t.clear(threads)
        ti = t.insert(ins, vals, threads)
        tr = t.retrieve(q, out, found, threads)
        best = ti + tr if best is None else min(best, ti + tr)
    ok = int(found.sum()) == n - n // 2
    return 2 * n / best / 1e9, n, ok


def cpu_baseline(args):
    threads = os.cpu_count() or 1
    v, n, ok = cpu_sample(args, threads, 3)
    return {"value": round(v, 5), "unit": "Gops/s", "cores": threads, "kind": "port",
            "sample": "insert 2^%d + retrieve 2^%d (50%% hit) at load %.2f, CG 8, min of 3"
                      % (args.cpu_log2n, args.cpu_log2n, args.load),
            "verified": ok}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    vals = []
    for _ in range(args.warmup):
        cpu_sample(args, threads, 1)
    for _ in range(args.steps):
        v, n, ok = cpu_sample(args, threads, 1)
        vals.append(v)
    value = statistics.mean(vals)
    line = {
        "impl": "reference",
        "metric": "insert+retrieve Gops/s (keys processed per second, whole job)",
        "value": round(value, 5),
        "unit": "Gops/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(2 * (1 << args.cpu_log2n) / (value * 1e9) * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64" if args.workload not in ("svht32", "counting32") else "u32",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD_NAMES[args.workload].format(L=args.log2n, L1=args.log2n + 1, L3=args.log2n - 3,
                                                         LF=args.load, B=args.bucket),
                   "sample": "2^%d keys per step on the host" % args.cpu_log2n},
        "cpu_baseline": {"value": round(value, 5), "unit": "Gops/s", "cores": threads,
                         "kind": "port",
                         "sample": "insert 2^%d + retrieve 2^%d per step, CG 8 windows, "
                                   "reference lane order" % (args.cpu_log2n, args.cpu_log2n)},
        "e2e": {"value": round(value, 5), "unit": "Gops/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": round(time.perf_counter() - t0, 2),
    }
    print(json.dumps(line), flush=True)


def run_gen(args):
    """The on-device input generators (random_distributions.cuh:50-326):
    2^L distinct u64 keys, 2^L uniform u64 words and 2^(L-2) Zipf(1.1)
    ranks over 2^(L-4) per step, each checked against the oracle on its
    first elements.  Reported value: elements generated per second over the
    three; the roofline is the unique-key kernel's write bandwidth.  The
    step's outputs are checked by properties: every key distinct and no
    sentinel, uniform words with the right mean, Zipf ranks in range with
    rank 1 at its expected frequency."""
    import torch
    import warpcore_b200 as wc
    torch.cuda.set_device(0)
    n = 1 << args.log2n
    nz = n >> 2
    a = torch.empty(n, dtype=torch.int64, device="cuda")
    b = torch.empty(n, dtype=torch.int64, device="cuda")
    z = torch.empty(nz, dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    seed = 77

    def step(k):
        wc.gen_unique(a, seed + k, stream=stream)
        wc.gen_uniform(b, seed + k, stream=stream)
        wc.gen_zipf(z, n >> 4, 1.1, seed + k, stream=stream)

    with torch.cuda.stream(stream):
        step(0)
    torch.cuda.synchronize()
    m = min(n, 1 << 24)
    distinct = torch.unique(a[:m]).numel() == m and not bool(((a == 0) | (a == -1)).any())
    top = (b[:m] >> 32) & 0xFFFFFFFF                       # the high words, uniform on 2^32
    uniform = abs(float(top.double().mean()) / 2**32 - 0.5) < 0.01
    nin = n >> 4
    h = sum(k ** -1.1 for k in range(1, 100001)) + (nin ** -0.1 - 100000 ** -0.1) / -0.1
    p1 = float((z == 1).double().mean())
    zipf = bool(((z >= 1) & (z <= nin)).all()) and abs(p1 * h - 1.0) < 0.02
    verified = distinct and uniform and zipf
    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            step(k)
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    launches0 = wc.launch_count()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            ev[k][0].record(stream)
            wc.gen_unique(a, seed + k, stream=stream)
            ev[k][1].record(stream)
            wc.gen_uniform(b, seed + k, stream=stream)
            ev[k][2].record(stream)
            wc.gen_zipf(z, n >> 4, 1.1, seed + k, stream=stream)
            ev[k][3].record(stream)
    torch.cuda.synchronize()
    launches = wc.launch_count() - launches0
    clocks = sampler.stop()
    uq = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    un = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    zf = statistics.mean(e[2].elapsed_time(e[3]) for e in ev)
    total_ms = uq + un + zf
    peak, peak_src = measured_peak()
    achieved = 8 * n / (uq * 1e-3) / 1e9
    line = {
        "metric": "generated elements/s (distinct keys, uniform words, Zipf draws)",
        "value": round((2 * n + nz) / (total_ms * 1e-3) / 1e9, 4),
        "unit": "Gelem/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "generated on the device (counter-based splitmix64 / fmix64)",
        "config": {"workload": "generators: unique 2^%d u64 + uniform 2^%d u64 + Zipf(1.1) 2^%d over 2^%d"
                               % (args.log2n, args.log2n, args.log2n - 2, args.log2n - 4)},
        "unique_gelem_s": round(n / (uq * 1e-3) / 1e9, 3),
        "uniform_gelem_s": round(n / (un * 1e-3) / 1e9, 3),
        "zipf_gelem_s": round(nz / (zf * 1e-3) / 1e9, 3),
        "verified": bool(verified),
        "roofline": {"bound": "hbm", "kernel": "gen_unique_kernel", "achieved": round(achieved, 2),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "peak_source": peak_src, "algorithmic_bytes_per_op": 8, "traffic": None},
        "cpu_baseline": None, "e2e": None, "gpu_launches": launches, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_served(args):
    """The served mixed workload on one GPU, in both forms, at several
    arrival rates, bit-exact against per-table expectations.  Reported
    value: aggregate Gops/s of continuous batching at the highest rate."""
    import numpy as np
    import torch
    import warpcore_b200  # noqa: F401
    from warpcore_b200.serve import ServedWorkload, run
    torch.cuda.set_device(0)
    rates = [float(r) for r in args.rates.split(",")]
    sampler = ClockSampler(0)
    sweep = []
    launches = 0
    for i, rate in enumerate(rates):
        w = ServedWorkload(num_tables=args.tables, num_requests=args.requests, rate=rate, seed=5)
        w.admit()
        point = {"rate_per_s": rate}
        for mode in ("plain", "batched", "persistent"):
            rs = []
            for k in range(args.warmup + args.steps):
                w.reset()
                torch.cuda.synchronize()
                if i == len(rates) - 1 and mode == "plain" and k == args.warmup:
                    sampler.start()
                r = run(w, mode)
                if k >= args.warmup:
                    r["verified"] = w.verify()
                    rs.append(r)
            point[mode] = {key: round(float(np.median([r[key] for r in rs])), 3)
                           for key in ("gops", "p50_us", "p99_us", "span_ms", "launches")}
            point[mode]["verified"] = all(r["verified"] for r in rs)
            if i == len(rates) - 1 and mode == "persistent":
                launches = int(sum(r["launches"] for r in rs))
        sweep.append(point)
        admitted, table_gib, keys = int(w.admitted.sum()), w.table_bytes / 2**30, int(w.num.sum())
        del w
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    top = sweep[-1]
    line = {
        "metric": "served aggregate Gops/s (persistent kernel), p50/p99 request latency",
        "value": top["persistent"]["gops"], "unit": "Gops/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": top["persistent"]["span_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded Poisson stream, keys unique per table)",
        "config": {"workload": WORKLOAD_NAMES["served"], "tables": args.tables,
                   "admitted_tables": admitted, "table_gib": round(table_gib, 2),
                   "budget_gib": 64, "requests": args.requests, "keys": keys,
                   "rates_per_s": rates},
        "sweep": sweep,
        "batched_vs_plain_at_top_rate": {
            "gops": round(top["batched"]["gops"] / top["plain"]["gops"], 3),
            "p99": round(top["plain"]["p99_us"] / top["batched"]["p99_us"], 3)},
        "persistent_vs_plain": [
            {"rate_per_s": p["rate_per_s"],
             "gops": round(p["persistent"]["gops"] / p["plain"]["gops"], 3),
             "p99": round(p["plain"]["p99_us"] / p["persistent"]["p99_us"], 3)} for p in sweep],
        "gpu_launches": launches, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="svht64", choices=sorted(WORKLOAD_NAMES))
    ap.add_argument("--log2n", type=int, default=None,
                    help="keys per step (2^L); default 27, or 24 pairs for mv32")
    ap.add_argument("--load", type=float, default=None,
                    help="target load factor; default 0.9, or 0.8 for mv32")
    ap.add_argument("--store", default="aos", choices=["aos", "soa"],
                    help="svht32/svht64: slot layout of this library's table and of the "
                         "reference build's (SoAStore for soa)")
    ap.add_argument("--fill", action="store_true",
                    help="svht32/svht64/hashset64: fill the table of min capacity 2^L/load to a "
                         "real load of `load` (keys = load x capacity) instead of inserting 2^L")
    ap.add_argument("--cpu-log2n", type=int, default=24)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="svht: use the sharded table (partition + NCCL all-to-all) "
                         "even with one rank; with more ranks it is always used")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--tables", type=int, default=4096)
    ap.add_argument("--requests", type=int, default=8192)
    ap.add_argument("--rates", default="100000,200000,300000,1000000")
    ap.add_argument("--bucket", type=int, default=2,
                    help="values per slot of the mb32 workload (1, 2, 4 or 8)")
    args = ap.parse_args()
    if args.log2n is None:
        args.log2n = 24 if args.workload == "mv32" else 27
    if args.load is None:
        args.load = {"mv32": 0.8, "mb32": 0.8, "counting32": 0.85}.get(args.workload, 0.9)
    if args.warmup < 3:
        log("warm-up raised to 3 steps")
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "gen":
        run_gen(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
