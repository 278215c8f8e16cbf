"""Served mixed workload: many resident tables, a Poisson request stream,
continuous batching (wc_serve_run) and per-table bit-exact verification.

The workload follows the served configuration:
- T independent SingleValueHashTable<u32,u32> tables;
- nominal capacities log-uniform in [cap_lo, cap_hi], filled to at most
  `load` of the nominal capacity;
- Poisson arrivals at `rate` requests/s;
- batch sizes log-uniform in [batch_lo, batch_hi];
- 30 % inserts and 70 % retrieves, 80 % of retrieved keys being hits.

Keys are unique per table: key(t, j) = fmix32(j ^ salt_t), a bijection of
the per-table index j, so the indices [0, budget) used by inserts and
[2^31, 2^32) used by absent keys never collide. Hits draw only keys that
earlier requests of the same table inserted, so every request's answer is
fixed by arrival order. The expected outputs are computed from the indices,
without the tables.

Admission, two policies:
- static (admit()): tables are created, resident for the whole run, in
  table order while the sum of their device bytes stays within
  `budget_bytes`; requests for a table that was not admitted are rejected
  before the run and counted;
- dynamic (admit(dynamic=True), persistent form only): every table is
  registered in a table pool (wc_table_pool) with the budget and none is
  resident; a table is placed in device memory when its first request
  runs, and when the budget (resident tables plus the buffers of requests
  in flight) has no room, the least recently used idle tables are copied
  out to host memory and restored when a request needs them again.
"""
import ctypes
import math

import numpy as np

from . import (OP_INSERT, OP_RETRIEVE, SERVE_BATCHED, SERVE_PERSISTENT, SERVE_PLAIN, ServeOptions,
               ServeRequest, ServeStats, SingleValueHashTable, _check, lib,
               set_l2_persistence, valid_capacity, DEFAULT_PROBING_LENGTH)

MASK32 = 0xFFFFFFFF
_C1, _C2 = 0x85EBCA6B, 0xC2B2AE35


def fmix32_np(x):
    x = x.astype(np.uint64) & MASK32
    x ^= x >> 16
    x = (x * _C1) & MASK32
    x ^= x >> 13
    x = (x * _C2) & MASK32
    x ^= x >> 16
    return x


def _inv32(a):
    return pow(a, -1, 1 << 32)


def fmix32_inverse(y):
    """the index whose fmix32 is y (fmix32 is a bijection of u32)"""
    y &= MASK32
    y ^= y >> 16
    y = (y * _inv32(_C2)) & MASK32
    y ^= (y >> 13) ^ (y >> 26)
    y = (y * _inv32(_C1)) & MASK32
    y ^= y >> 16
    return y


def fmix32_torch(j):
    import torch
    x = j & MASK32
    x = x ^ (x >> 16)
    x = (x * _C1) & MASK32
    x = x ^ (x >> 13)
    x = (x * _C2) & MASK32
    x = x ^ (x >> 16)
    return x


def _as_i32(x):
    """int64 tensor of u32 values -> int32 tensor with the same bits"""
    import torch
    return (x - ((x >= (1 << 31)).to(torch.int64) << 32)).to(torch.int32)


class ServedWorkload:
    """Seeded request stream for the served configuration, resident on the
    device."""

    ABSENT_BASE = 1 << 31

    def __init__(self, num_tables=4096, cap_lo=1 << 10, cap_hi=1 << 22, load=0.85,
                 num_requests=8192, batch_lo=1 << 6, batch_hi=1 << 18, insert_frac=0.3,
                 hit_frac=0.8, rate=100000.0, seed=5, budget_bytes=64 << 30, device="cuda",
                 cg_size=None):
        import torch
        # the window width of the tables this layer creates itself: the
        # autotuner's choice (tuning_b200.json, "serving"), else 8
        self.cg_size = int(cg_size or serving_tuning().get("cg_size", 8))
        rng = np.random.default_rng(seed)
        self.num_tables = num_tables
        self.caps = np.exp(rng.uniform(math.log(cap_lo), math.log(cap_hi), num_tables)).astype(np.int64)
        self.budget = np.floor(load * self.caps).astype(np.int64)
        bad0 = fmix32_inverse(0)
        bad1 = fmix32_inverse(MASK32)
        salts = []
        for _ in range(num_tables):
            while True:
                s = int(rng.integers(1 << 23, 1 << 30))
                # keep both sentinel preimages out of the insert and absent ranges
                if all(not ((b ^ s) < (1 << 23) or (b ^ s) >= self.ABSENT_BASE) for b in (bad0, bad1)):
                    salts.append(s)
                    break
        self.salts = np.array(salts, dtype=np.int64)

        gaps = rng.exponential(1.0 / rate, num_requests)
        self.arrival_us = np.cumsum(gaps) * 1e6
        self.table = rng.integers(0, num_tables, num_requests)
        want_insert = rng.random(num_requests) < insert_frac
        size = np.exp(rng.uniform(math.log(batch_lo), math.log(batch_hi), num_requests)).astype(np.int64)
        inserted = np.zeros(num_tables, dtype=np.int64)
        self.op = np.empty(num_requests, dtype=np.int64)
        self.num = np.empty(num_requests, dtype=np.int64)
        self.ins_start = np.zeros(num_requests, dtype=np.int64)
        self.hits_from = np.zeros(num_requests, dtype=np.int64)  # inserted count at arrival
        for r in range(num_requests):
            t = self.table[r]
            room = self.budget[t] - inserted[t]
            if want_insert[r] and room > 0:
                n = int(min(size[r], room))
                self.op[r] = OP_INSERT
                self.ins_start[r] = inserted[t]
                inserted[t] += n
            else:
                n = int(size[r])
                self.op[r] = OP_RETRIEVE
                self.hits_from[r] = inserted[t]
            self.num[r] = n
        self.offsets = np.concatenate([[0], np.cumsum(self.num)])
        self.total_keys = int(self.offsets[-1])

        # per-key index j and table salt, on the host, vectorised per kind
        j = np.empty(self.total_keys, dtype=np.int64)
        is_hit = np.zeros(self.total_keys, dtype=bool)
        absent_next = self.ABSENT_BASE
        for r in range(num_requests):
            a, b = self.offsets[r], self.offsets[r + 1]
            n = b - a
            if self.op[r] == OP_INSERT:
                j[a:b] = np.arange(self.ins_start[r], self.ins_start[r] + n)
            else:
                avail = self.hits_from[r]
                hit = (rng.random(n) < hit_frac) if avail > 0 else np.zeros(n, dtype=bool)
                nh = int(hit.sum())
                jj = np.empty(n, dtype=np.int64)
                jj[hit] = rng.integers(0, max(avail, 1), nh)
                jj[~hit] = np.arange(absent_next, absent_next + (n - nh))
                absent_next += n - nh
                j[a:b] = jj
                is_hit[a:b] = hit
        salt_per_key = np.repeat(self.salts[self.table], self.num)
        jt = torch.from_numpy(j).to(device)
        st = torch.from_numpy(salt_per_key).to(device)
        keyidx = jt ^ st
        self.keys = _as_i32(fmix32_torch(keyidx)).contiguous()
        self.values = _as_i32(fmix32_torch(keyidx ^ 0x9E3779B9)).contiguous()
        self.is_hit = torch.from_numpy(is_hit).to(device)
        self.is_retrieve = torch.from_numpy(np.repeat(self.op == OP_RETRIEVE, self.num)).to(device)
        self.out = torch.empty_like(self.keys)
        assert not bool(((self.keys == 0) | (self.keys == -1)).any())
        self.budget_bytes = budget_bytes
        self.tables = [None] * num_tables
        self.admitted = np.zeros(num_tables, dtype=bool)
        self.table_bytes = 0
        self.rejected = 0
        self.pool = None      # table pool handle (dynamic admission)
        self.dynamic = False

    def admission_plan(self):
        """tables admitted in table order while their device bytes (the
        reference capacity rule, 8-byte slots) fit in the budget"""
        used = 0
        plan = np.zeros(self.num_tables, dtype=bool)
        for t in range(self.num_tables):
            need = valid_capacity(int(self.caps[t]), self.cg_size) * 8 + 256
            if used + need <= self.budget_bytes:
                plan[t] = True
                used += need
        return plan, used

    def admit(self, dynamic=False, budget_bytes=None):
        """create the admitted tables; they stay resident for the run.
        dynamic=True instead registers every table in a table pool with the
        budget (`budget_bytes`, default the workload's) and creates none.
        When the resident tables together exceed L2, none gets an L2
        persistence window: windows on the first few tables would only
        take L2 away from the many others (measured: -7 % aggregate at
        1M requests/s on 41 GiB of tables)."""
        import torch
        if dynamic:
            self.dynamic = True
            self.pool_budget = int(self.budget_bytes if budget_bytes is None else budget_bytes)
            self._new_pool()
            self.admitted = np.ones(self.num_tables, dtype=bool)
            self.rejected = 0
            return
        plan, used = self.admission_plan()
        windows = used <= torch.cuda.get_device_properties(0).L2_cache_size
        prev = set_l2_persistence(windows)
        try:
            for t in np.nonzero(plan)[0]:
                self.tables[t] = SingleValueHashTable(int(self.caps[t]), key_bytes=4,
                                                      cg_size=self.cg_size)
        finally:
            set_l2_persistence(prev)
        self.admitted = plan
        self.table_bytes = used
        self.rejected = int((~plan[self.table]).sum())

    def _new_pool(self):
        from . import TableConfig, lib as _lib, wc_svht_default_config_py
        if self.pool is not None:
            _lib().wc_table_pool_destroy(self.pool)
            self.pool = None
        h = ctypes.c_void_p()
        _check(_lib().wc_table_pool_create(self.pool_budget, ctypes.byref(h)))
        self.pool = h
        cfg = wc_svht_default_config_py(4, 4)
        cfg.cg_size = self.cg_size
        tid = ctypes.c_uint64()
        for t in range(self.num_tables):
            _check(_lib().wc_table_pool_add(h, ctypes.byref(cfg), int(self.caps[t]),
                                            0x5AD0DED, ctypes.byref(tid)))
            assert tid.value == t
        self.table_bytes = 0

    def pool_stats(self):
        from . import TablePoolStats
        st = TablePoolStats()
        _check(lib().wc_table_pool_get_stats(self.pool, ctypes.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in st._fields_}

    def close(self):
        if self.pool is not None:
            lib().wc_table_pool_destroy(self.pool)
            self.pool = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        """every table empty again (dynamic: a fresh pool, nothing resident)"""
        if self.dynamic:
            self._new_pool()
        for t in self.tables:
            if t is not None:
                t.init()
        self.out.fill_(-1)

    def requests(self):
        import torch
        keep = np.nonzero(self.admitted[self.table])[0]
        arr = (ServeRequest * len(keep))()
        kp = self.keys.data_ptr()
        vp = self.values.data_ptr()
        op = self.out.data_ptr()
        for i, r in enumerate(keep):
            q = arr[i]
            q.arrival_us = float(self.arrival_us[r])
            q.table = None if self.dynamic else self.tables[self.table[r]]._h.value
            q.table_id = int(self.table[r])
            q.op = int(self.op[r])
            off = int(self.offsets[r]) * 4
            q.keys = kp + off
            if self.op[r] == OP_INSERT:
                q.values = vp + off
            else:
                q.values_out = op + off
            q.num = int(self.num[r])
        return arr, keep

    def verify(self):
        """every retrieved key: value on a hit, untouched output on a miss"""
        import torch
        admitted_key = torch.from_numpy(np.repeat(self.admitted[self.table], self.num)).to(self.keys.device)
        ret = self.is_retrieve & admitted_key
        hits = ret & self.is_hit
        miss = ret & ~self.is_hit
        ok_hits = bool(torch.equal(self.out[hits], self.values[hits]))
        ok_miss = bool((self.out[miss] == -1).all())
        return ok_hits and ok_miss


def serving_tuning():
    """the "serving" section of the tuning file (cg_size, chunk_keys), or {}"""
    import json
    import os
    path = os.environ.get("WARPCORE_B200_TUNING") or os.path.join(
        os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json")
    try:
        with open(path) as f:
            return json.load(f).get("serving", {}) or {}
    except (OSError, ValueError):
        return {}


def run(workload, mode, streams=4, depth=2, max_batch_requests=4096, max_batch_keys=None,
        blocks_per_sm=0):
    """Replays the workload in `mode` ("plain", "batched" or "persistent");
    returns a dict with throughput, latency percentiles and launch counts.
    For "persistent", max_batch_keys is the largest chunk (default: the
    autotuner's chunk_keys, else 1024 keys); for "batched" the keys per batch
    (default no limit)."""
    if max_batch_keys is None:
        max_batch_keys = int(serving_tuning().get("chunk_keys", 0)) if mode == "persistent" else 0
    reqs, keep = workload.requests()
    n = len(keep)
    opt = ServeOptions()
    opt.mode = {"plain": SERVE_PLAIN, "batched": SERVE_BATCHED,
                "persistent": SERVE_PERSISTENT}[mode]
    opt.streams = streams
    opt.depth = depth
    opt.max_batch_requests = max_batch_requests
    opt.max_batch_keys = max_batch_keys
    opt.blocks_per_sm = blocks_per_sm
    opt.probing_length = DEFAULT_PROBING_LENGTH
    if workload.dynamic:
        if mode != "persistent":
            raise ValueError("dynamic admission runs with the persistent form")
        opt.pool = workload.pool.value
    issue = (ctypes.c_double * n)()
    done = (ctypes.c_double * n)()
    stats = ServeStats()
    _check(lib().wc_serve_run(reqs, n, ctypes.byref(opt), issue, done, ctypes.byref(stats)))
    arrival = np.array([reqs[i].arrival_us for i in range(n)])
    complete = np.frombuffer(done, dtype=np.float64, count=n).copy()
    lat = complete - arrival
    keys = int(workload.num[keep].sum())
    span_us = complete.max() - arrival.min()
    return {
        "mode": mode,
        "requests": n,
        "keys": keys,
        "gops": keys / (span_us * 1e-6) / 1e9,
        "p50_us": float(np.percentile(lat, 50)),
        "p99_us": float(np.percentile(lat, 99)),
        "mean_us": float(lat.mean()),
        "span_ms": span_us / 1e3,
        "launches": int(stats.launches),
        "batches": int(stats.batches),
        "max_keys_in_batch": int(stats.max_keys_in_batch),
        "gpu_batch_us_mean": float(stats.gpu_batch_us) / max(1, int(stats.batches)),
        "host_launch_us_mean": float(stats.host_launch_us) / max(1, int(stats.batches)),
    }
