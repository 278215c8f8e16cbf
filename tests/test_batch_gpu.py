"""Batches (wc_batch_run) and the serving loop (wc_serve_run) on the GPU:
requests on many tables in one launch give the per-table oracle's answers,
and both served forms reproduce every request's answer alone and in the mix."""
import numpy as np
import pytest

import warpcore_b200 as wc
from oracle import oracle as o
from tests.wc_helpers import dev, empty_dev, host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kb", [4, 8])
def test_batch_many_tables_matches_oracle(kb):
    rng = np.random.default_rng(1)
    caps = [1000, 50000, 200000, 3000, 777777, 64, 90000, 12345]
    gpu = [wc.SingleValueHashTable(c, key_bytes=kb) for c in caps]
    ref = [o.Table(o.SVHT, kb, kb, c) for c in caps]
    b = wc.Batch(max_requests=64)
    keys, vals, absent = [], [], []
    for i, c in enumerate(caps):
        n = int(c * 0.7)
        k = o.gen_unique_keys(kb, n + 500, 100 + i)
        keys.append(k[:n])
        absent.append(k[n:])
        vals.append(o.gen_uniform(kb, n, 200 + i))
    # one batch of inserts: two requests per table (distinct keys commute)
    reqs, st_bufs = [], []
    for i in range(len(caps)):
        h = len(keys[i]) // 2
        for part in (slice(0, h), slice(h, None)):
            kk, vv = keys[i][part], vals[i][part]
            st = empty_dev(kk.size, 4)
            st_bufs.append((i, part, st))
            reqs.append({"table": gpu[i], "op": "insert", "keys": dev(kk), "buffer": dev(vv),
                         "status_out": st})
    keep = b.run(reqs)
    for i in range(len(caps)):
        ref[i].insert(keys[i], vals[i])
    for i, part, st in st_bufs:
        assert (host(st) == 0).all()
    for i in range(len(caps)):
        assert gpu[i].size() == ref[i].size()
    # one batch of retrieves over all tables, hits and misses interleaved
    reqs, outs = [], []
    for i in range(len(caps)):
        q = np.concatenate([keys[i][rng.permutation(len(keys[i]))[:300]], absent[i][:300]])
        rng.shuffle(q)
        out = empty_dev(q.size, kb, 0xA5A5A5A5)
        st = empty_dev(q.size, 4)
        reqs.append({"table": gpu[i], "op": "retrieve", "keys": dev(q), "buffer": out,
                     "status_out": st})
        outs.append((i, q, out, st))
    keep2 = b.run(reqs)
    for i, q, out, st in outs:
        r_out = np.full(q.size, 0xA5A5A5A5, dtype=keys[i].dtype)
        r_out, r_st = ref[i].retrieve(q, r_out, want_status=True)
        assert np.array_equal(host(out), r_out)
        assert np.array_equal(host(st), r_st)
    for g, r in zip(gpu, ref):
        assert g.pop_status() == r.pop_status()
    del keep, keep2


def test_batch_rejects_mixed_layouts():
    a = wc.SingleValueHashTable(1000, key_bytes=4)
    c = wc.SingleValueHashTable(1000, key_bytes=8)
    b = wc.Batch(max_requests=4)
    k4, k8 = empty_dev(10, 4, 5), empty_dev(10, 8, 5)
    with pytest.raises(wc.WarpcoreError):
        b.run([(a, "insert", k4, k4), (c, "insert", k8, k8)])


def test_batch_graph_reuse_many_runs():
    # many runs through the same staging slots and cached graphs
    t = wc.SingleValueHashTable(100000, key_bytes=4)
    b = wc.Batch(max_requests=8, depth=2)
    allk = o.gen_unique_keys(4, 60000, 9)
    vals = o.gen_uniform(4, 60000, 10)
    keep = []
    for s in range(0, 60000, 1000):
        keep.append(b.run([(t, "insert", dev(allk[s:s + 500]), dev(vals[s:s + 500])),
                           (t, "insert", dev(allk[s + 500:s + 1000]), dev(vals[s + 500:s + 1000]))]))
    out = empty_dev(60000, 4)
    t.retrieve(dev(allk), out)
    assert np.array_equal(host(out), vals)


@pytest.mark.parametrize("mode", ["plain", "batched", "persistent"])
def test_served_small_workload(mode):
    from warpcore_b200.serve import ServedWorkload, run
    w = ServedWorkload(num_tables=48, cap_lo=1 << 10, cap_hi=1 << 15, num_requests=600,
                       batch_lo=1 << 4, batch_hi=1 << 12, rate=2e4, seed=11)
    w.admit()
    w.reset()
    res = run(w, mode)
    assert w.verify()
    assert res["requests"] == 600
    assert res["p50_us"] > 0 and res["p99_us"] >= res["p50_us"]
    if mode == "batched":
        assert res["batches"] <= 600


def test_served_same_answers_alone_and_in_the_mix():
    # each request replayed alone (its own plain launch, in arrival order)
    # equals its answer inside continuous batches
    from warpcore_b200.serve import ServedWorkload, run
    w = ServedWorkload(num_tables=16, cap_lo=1 << 10, cap_hi=1 << 13, num_requests=300,
                       batch_lo=1 << 4, batch_hi=1 << 10, rate=1e6, seed=12)
    w.admit()
    w.reset()
    run(w, "plain", streams=1)
    alone = w.out.clone()
    w.reset()
    res = run(w, "batched")
    assert res["batches"] < 300  # requests really shared launches
    import torch
    assert torch.equal(alone, w.out)
    assert w.verify()
    # and inside the persistent kernel, with small chunks so that requests
    # share the resident warps chunk by chunk
    w.reset()
    res = run(w, "persistent", max_batch_keys=64)
    assert res["launches"] == 1
    assert torch.equal(alone, w.out)
    assert w.verify()


def _pserver(key_bytes=4, cg=8, idle_us=2000000, chunk=0):
    import ctypes
    import torch
    opt = wc.PServerOptions()
    opt.key_bytes, opt.cg_size, opt.idle_timeout_us, opt.chunk_keys = key_bytes, cg, idle_us, chunk
    opt.probing_length = wc.DEFAULT_PROBING_LENGTH
    stream = torch.cuda.Stream()
    h = ctypes.c_void_p()
    rc = wc.lib().wc_pserver_start(ctypes.byref(opt), stream.cuda_stream, ctypes.byref(h))
    assert rc == 0, wc.lib().wc_last_error()
    return h, stream


def _wait(h, ticket, limit_s=10.0):
    import ctypes
    import time
    done, cu = ctypes.c_int(0), ctypes.c_double(0)
    t0 = time.time()
    while not done.value:
        assert wc.lib().wc_pserver_poll(h, ticket, ctypes.byref(done), ctypes.byref(cu)) == 0
        assert time.time() - t0 < limit_s
    return cu.value


@pytest.mark.parametrize("kb", [4, 8])
def test_persistent_server_requests(kb):
    """insert, then retrieve (hits and misses), through the resident kernel;
    answers equal the oracle's and size() counts the inserts"""
    import ctypes
    n = 5000
    t = wc.SingleValueHashTable(2 * n, key_bytes=kb)
    r = o.Table(o.SVHT, kb, kb, 2 * n)
    allk = o.gen_unique_keys(kb, 2 * n, 61)
    keys, absent = allk[:n], allk[n:]
    vals = o.gen_uniform(kb, n, 62)
    r.insert(keys, vals)
    dk, dv = dev(keys), dev(vals)
    q = np.concatenate([keys[::2], absent[:1000]])
    dq = dev(q)
    out = empty_dev(q.size, kb, 7)
    h, _ = _pserver(key_bytes=kb, chunk=256)
    tk = ctypes.c_uint64()
    try:
        assert wc.lib().wc_pserver_submit(h, t._h, wc.OP_INSERT, dk.data_ptr(), dv.data_ptr(),
                                          None, n, ctypes.byref(tk)) == 0
        c1 = _wait(h, tk.value)
        assert wc.lib().wc_pserver_submit(h, t._h, wc.OP_RETRIEVE, dq.data_ptr(), None,
                                          out.data_ptr(), q.size, ctypes.byref(tk)) == 0
        c2 = _wait(h, tk.value)
        assert c2 >= c1 > 0
    finally:
        rc = wc.lib().wc_pserver_stop(h)
    assert rc == 0, wc.lib().wc_last_error()
    r_out = np.full(q.size, 7, dtype=keys.dtype)
    r_out = r.retrieve(q, r_out)
    assert np.array_equal(host(out), r_out)
    assert t.size() == n


def test_persistent_server_idle_limit_ends_the_kernel():
    """a server that gets no request ends on its idle limit (a bounded wait
    that runs out), reports WC_ERR_TIMEOUT at the stop, and the context
    stays usable"""
    import time
    h, _ = _pserver(idle_us=20000)
    time.sleep(0.3)
    rc = wc.lib().wc_pserver_stop(h)
    assert rc == wc.ERR_TIMEOUT
    assert b"idle" in wc.lib().wc_last_error()
    t = wc.SingleValueHashTable(1000, key_bytes=4)
    k = o.gen_unique_keys(4, 100, 3)
    t.insert(dev(k), dev(k))
    assert t.size() == 100


def test_served_dynamic_admission_evicts_and_restores():
    """Tables admitted against a budget of about a third of their bytes:
    each is placed in device memory when its first request runs, evicted to
    host memory when the budget needs room and restored when a request needs
    it again, all while the persistent kernel runs; every answer equals the
    run with every table resident, and the budget is never exceeded."""
    import torch
    from warpcore_b200.serve import ServedWorkload, run
    # (every table takes about 8 MB under the capacity rule; at 2000
    # requests/s a table is often idle and evicted before its next request)
    w = ServedWorkload(num_tables=24, cap_lo=1 << 12, cap_hi=1 << 16, num_requests=300,
                       batch_lo=1 << 4, batch_hi=1 << 11, rate=2e3, seed=13)
    w.admit()
    w.reset()
    run(w, "plain", streams=1)
    alone = w.out.clone()
    assert w.verify()
    budget = w.table_bytes // 3
    w.admit(dynamic=True, budget_bytes=budget)
    w.reset()
    res = run(w, "persistent", max_batch_keys=64)
    st = w.pool_stats()
    assert res["requests"] == 300
    assert torch.equal(alone, w.out)
    assert w.verify()
    assert st["admissions"] > 24 and st["evictions"] > 0 and st["restores"] > 0
    assert st["peak_bytes"] <= budget
    w.close()
