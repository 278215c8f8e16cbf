"""Parity of the CUDA tables with the CPU oracle, called through the C ABI.

Same seeded inputs on both sides; bit-exact comparison of retrieved values,
membership flags, per-key statuses, sizes, table Status words and the table
contents as multisets (slot placement differs by design: the CUDA tables
probe bucket-aligned windows)."""
import numpy as np
import pytest

import warpcore_b200 as wc
from oracle import oracle as o
from tests.wc_helpers import dev, empty_dev, host, sorted_pairs

pytestmark = pytest.mark.gpu

SENT = {4: 0xA5A5A5A5, 8: 0xA5A5A5A5A5A5A5A5}
HANDLER_STATUS = wc.HANDLER_STATUS

ORACLE_PROBE = {wc.PROBING_DOUBLE: o.PROBE_DOUBLE, wc.PROBING_LINEAR: o.PROBE_LINEAR,
                wc.PROBING_QUADRATIC: o.PROBE_QUADRATIC}


def make_pair(kind, kb, n_cap, cg, probing=wc.PROBING_DOUBLE, h1=wc.HASH_MURMUR,
              h2=wc.HASH_MURMUR, seed=wc.DEFAULT_SEED, max_count=None, empty=0, tomb=None,
              vb=None, store="aos"):
    if tomb is None:
        tomb = (1 << (8 * kb)) - 1
    vb = kb if vb is None else vb
    kw = dict(key_bytes=kb, cg_size=cg, probing=probing, hasher1=h1, hasher2=h2,
              empty_key=empty, tombstone_key=tomb)
    if kind == o.SVHT:
        g = wc.SingleValueHashTable(n_cap, seed=seed, value_bytes=vb, store=store, **kw)
    elif kind == o.HASHSET:
        g = wc.HashSet(n_cap, seed=seed, **kw)
    else:
        g = wc.CountingHashTable(n_cap, seed=seed, max_count=max_count, value_bytes=vb, **kw)
    r = o.Table(kind, kb, 0 if kind == o.HASHSET else vb, n_cap, seed=seed, cg=cg,
                scheme=ORACLE_PROBE[probing], h1=h1, h2=h2, empty_key=empty,
                tombstone_key=tomb, max_count=max_count)
    assert g.capacity == r.capacity
    return g, r


def svht_round_trip(kb, cg, probing=wc.PROBING_DOUBLE, h1=wc.HASH_MURMUR,
                    h2=wc.HASH_MURMUR, n=20000, load=0.8, seed=7, vb=None, store="aos"):
    vb = kb if vb is None else vb
    n_cap = int(n / load)
    g, r = make_pair(o.SVHT, kb, n_cap, cg, probing, h1, h2, vb=vb, store=store)
    allk = o.gen_unique_keys(kb, 2 * n, seed)
    keys, absent = allk[:n], allk[n:]
    vals = o.gen_uniform(vb, n, seed + 1)
    st = empty_dev(n, 4)
    g.insert(dev(keys), dev(vals), status_out=st)
    r_st = r.insert(keys, vals, want_status=True)
    assert np.array_equal(host(st), r_st)
    assert g.size() == r.size() == n
    assert g.pop_status() == r.pop_status()

    # duplicates with new values, plus both sentinels
    nd = n // 8
    k2 = np.concatenate([keys[:nd], np.array([0, (1 << (8 * kb)) - 1], dtype=keys.dtype)])
    v2 = o.gen_uniform(vb, nd + 2, seed + 2)
    st2 = empty_dev(nd + 2, 4)
    g.insert(dev(k2), dev(v2), status_out=st2)
    assert np.array_equal(host(st2), r.insert(k2, v2, want_status=True))
    assert g.pop_status() == r.pop_status()

    q = np.empty(2 * n, dtype=keys.dtype)
    q[0::2] = keys
    q[1::2] = absent
    out = empty_dev(2 * n, vb, SENT[vb])
    st3 = empty_dev(2 * n, 4)
    g.retrieve(dev(q), out, status_out=st3)
    r_out = np.full(2 * n, SENT[vb], dtype=vals.dtype)
    r_out, r_st3 = r.retrieve(q, r_out, want_status=True)
    assert np.array_equal(host(out), r_out)
    assert np.array_equal(host(st3), r_st3)
    assert g.pop_status() == r.pop_status()

    er = np.concatenate([keys[::5], absent[:16]])
    st4 = empty_dev(er.size, 4)
    g.erase(dev(er), status_out=st4)
    assert np.array_equal(host(st4), r.erase(er, want_status=True))
    assert g.size() == r.size()
    assert g.pop_status() == r.pop_status()

    out = empty_dev(2 * n, vb, SENT[vb])
    st5 = empty_dev(2 * n, 4)
    g.retrieve(dev(q), out, status_out=st5)
    r_out = np.full(2 * n, SENT[vb], dtype=vals.dtype)
    r_out, r_st5 = r.retrieve(q, r_out, want_status=True)
    assert np.array_equal(host(out), r_out)
    assert np.array_equal(host(st5), r_st5)

    # contents as a multiset
    ko = empty_dev(g.capacity, kb)
    vo = empty_dev(g.capacity, vb)
    m = g.retrieve_all(ko, vo)
    rk, rv = r.retrieve_all()
    assert m == rk.size
    a = sorted_pairs(host(ko)[:m], host(vo)[:m])
    b = sorted_pairs(rk, rv)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("cg", [1, 2, 4, 8, 16, 32])
def test_svht_double_hashing(kb, cg):
    svht_round_trip(kb, cg)


@pytest.mark.parametrize("probing", [wc.PROBING_LINEAR, wc.PROBING_QUADRATIC])
@pytest.mark.parametrize("kb", [4, 8])
def test_svht_other_probing(kb, probing):
    svht_round_trip(kb, 8, probing=probing)


@pytest.mark.parametrize("h1,h2", [(wc.HASH_NVIDIA, wc.HASH_MUELLER),
                                   (wc.HASH_MUELLER, wc.HASH_MURMUR),
                                   (wc.HASH_IDENTITY32, wc.HASH_MURMUR)])
def test_svht_hashers_u32(h1, h2):
    svht_round_trip(4, 8, h1=h1, h2=h2)


def test_svht_identity64():
    svht_round_trip(8, 8, h1=wc.HASH_IDENTITY64, h2=wc.HASH_IDENTITY64)


@pytest.mark.parametrize("load", [0.5, 0.9, 0.97])
def test_svht_high_load(load):
    # capacity is 131101*cg at minimum, so fill it to the requested load
    cap = wc.valid_capacity(1, 8)
    svht_round_trip(4, 8, n=int(cap * load), load=load)


def test_svht_custom_sentinels():
    kb, n = 4, 5000
    g, r = make_pair(o.SVHT, kb, 8000, 8, empty=7, tomb=9)
    keys = o.gen_unique_keys(kb, n, 3)
    keys = keys[(keys != 7) & (keys != 9)]
    keys = np.concatenate([keys, np.array([0, 0xFFFFFFFF, 7, 9], dtype=np.uint32)])
    vals = o.gen_uniform(kb, keys.size, 4)
    st = empty_dev(keys.size, 4)
    g.insert(dev(keys), dev(vals), status_out=st)
    assert np.array_equal(host(st), r.insert(keys, vals, want_status=True))
    out = empty_dev(keys.size, kb, SENT[kb])
    g.retrieve(dev(keys), out)
    r_out = r.retrieve(keys, np.full(keys.size, SENT[kb], dtype=np.uint32))
    assert np.array_equal(host(out), r_out)
    assert g.peek_status() == r.peek_status()


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("cg", [4, 8, 16, 32])
def test_hashset(kb, cg):
    n = 20000
    g, r = make_pair(o.HASHSET, kb, 25000, cg)
    allk = o.gen_unique_keys(kb, 2 * n, 11)
    keys = allk[:n]
    st = empty_dev(n, 4)
    g.insert(dev(keys), status_out=st)
    assert np.array_equal(host(st), r.insert(keys, want_status=True))
    k2 = np.concatenate([keys[: n // 8], np.array([0], dtype=keys.dtype)])
    st2 = empty_dev(k2.size, 4)
    g.insert(dev(k2), status_out=st2)
    assert np.array_equal(host(st2), r.insert(k2, want_status=True))
    assert g.pop_status() == r.pop_status()
    q = np.empty(2 * n, dtype=keys.dtype)
    q[0::2] = keys
    q[1::2] = allk[n:]
    flags = empty_dev(2 * n, 1, 7)
    st3 = empty_dev(2 * n, 4)
    g.retrieve(dev(q), flags, status_out=st3)
    rf = np.full(2 * n, 7, dtype=np.uint8)
    rf, r_st3 = r.retrieve(q, rf, want_status=True)
    assert np.array_equal(host(flags), rf)
    assert np.array_equal(host(st3), r_st3)
    er = keys[::5]
    st4 = empty_dev(er.size, 4)
    g.erase(dev(er), status_out=st4)
    assert np.array_equal(host(st4), r.erase(er, want_status=True))
    assert g.size() == r.size()
    flags = empty_dev(2 * n, 1, 7)
    g.retrieve(dev(q), flags)
    rf = r.retrieve(q, np.full(2 * n, 7, dtype=np.uint8))
    assert np.array_equal(host(flags), rf)
    assert g.pop_status() == r.pop_status()
    ko = empty_dev(g.capacity, kb)
    m = g.retrieve_all(ko)
    assert np.array_equal(np.sort(host(ko)[:m]), np.sort(r.retrieve_all()))


@pytest.mark.parametrize("kb,vb", [(4, 8), (8, 4)])
@pytest.mark.parametrize("cg", [1, 8, 32])
@pytest.mark.parametrize("policy", ["never", "always"])
def test_svht_mixed_widths(kb, vb, cg, policy):
    """u32 keys with u64 values and u64 keys with u32 values (16-byte slots),
    on the window and the fingerprint kernels"""
    old = wc.set_fingerprint_policy(policy)
    try:
        svht_round_trip(kb, cg, vb=vb, load=0.9)
    finally:
        wc.set_fingerprint_policy(old)


def test_svht_mixed_widths_rebuild_route():
    """a large insert into a table with fingerprints larger than half of
    L2 takes the window kernel and the fingerprint rebuild; every pair reads
    back and the size is exact"""
    import torch
    n = 1 << 26
    t = wc.SingleValueHashTable(int(n / 0.9), key_bytes=4, value_bytes=8)
    assert t.info().fingerprints
    keys = wc.gen_unique(torch.empty(n, dtype=torch.int32, device="cuda"), 5)
    vals = wc.gen_uniform(torch.empty(n, dtype=torch.int64, device="cuda"), 6)
    t.insert(keys, vals)
    assert t.size() == n
    out = torch.zeros(n, dtype=torch.int64, device="cuda")
    st = torch.empty(n, dtype=torch.int32, device="cuda")
    t.retrieve(keys, out, status_out=st)
    assert bool((st == 0).all())
    assert torch.equal(out, vals)


@pytest.mark.parametrize("kb,vb", [(4, 4), (8, 8), (4, 8), (8, 4)])
@pytest.mark.parametrize("max_count", [None, 10])
def test_counting_zipf(kb, vb, max_count):
    distinct, occ = 5000, 200000
    g, r = make_pair(o.COUNTING, kb, 6000, 4, max_count=max_count, vb=vb)
    allk = o.gen_unique_keys(kb, distinct + distinct // 4, 51)
    ranks = o.gen_zipf_ranks(distinct, 1.1, occ, 54)
    keys = allk[(ranks - 1).astype(np.int64)]
    st = empty_dev(occ, 4)
    g.insert(dev(keys), status_out=st)
    r_st = r.insert(keys, want_status=True)
    g_st = host(st)
    # which occurrence of a key claims the slot is schedule-dependent; the
    # number of claims and of duplicates is not
    assert np.array_equal(np.sort(g_st), np.sort(r_st))
    assert g.pop_status() == r.pop_status()
    out = empty_dev(allk.size, vb, SENT[vb])
    st2 = empty_dev(allk.size, 4)
    g.retrieve(dev(allk), out, status_out=st2)
    r_out = np.full(allk.size, SENT[vb], dtype=np.uint32 if vb == 4 else np.uint64)
    r_out, r_st2 = r.retrieve(allk, r_out, want_status=True)
    assert np.array_equal(host(out), r_out)
    assert np.array_equal(host(st2), r_st2)
    # against a plain histogram as well
    hist = np.bincount(ranks.astype(np.int64) - 1, minlength=distinct)
    exp = hist if max_count is None else np.minimum(hist, max_count)
    got = host(out)[:distinct].astype(np.int64)
    present = hist > 0
    assert np.array_equal(got[present], exp[present])
    assert g.size() == r.size() == int(present.sum())


def test_status_handlers_boolean():
    n = 4000
    g, r = make_pair(o.SVHT, 4, 8000, 8)
    keys = o.gen_unique_keys(4, 2 * n, 5)
    vals = o.gen_uniform(4, n, 6)
    g.insert(dev(keys[:n]), dev(vals))
    r.insert(keys[:n], vals)
    q = np.concatenate([keys, np.array([0, 0xFFFFFFFF], dtype=np.uint32)])
    for ignore in (0, wc.Status.key_not_found().base(),
                   wc.Status.key_not_found().base() | wc.Status.invalid_key().base()):
        b = empty_dev(q.size, 1, 9)
        out = empty_dev(q.size, 4)
        g.retrieve(dev(q), out, status_out=b, status_handler=wc.HANDLER_BOOLEAN, ignore=ignore)
        _, r_st = r.retrieve(q, want_status=True)
        exp = np.array([o.status_to_bool(int(s), ignore) for s in r_st], dtype=np.uint8)
        assert np.array_equal(host(b), exp)


def test_probing_length_one_window():
    # probing_length = cg: exactly one window per key
    kb, cg = 4, 8
    cap = wc.valid_capacity(1, cg)
    g = wc.SingleValueHashTable(1, key_bytes=kb, cg_size=cg)
    keys = o.gen_unique_keys(kb, int(cap * 0.95), 9)
    vals = o.gen_uniform(kb, keys.size, 10)
    st = empty_dev(keys.size, 4)
    g.insert(dev(keys), dev(vals), probing_length=cg, status_out=st)
    s = host(st)
    assert set(np.unique(s).tolist()) <= {0, wc.Status.probing_length_exceeded().base()}
    ok = s == 0
    assert ok.sum() == g.size()
    out = empty_dev(keys.size, kb, SENT[kb])
    g.retrieve(dev(keys), out)
    assert np.array_equal(host(out)[ok], vals[ok])


def test_full_table_reports_probing_length_exceeded():
    # a completely full table: inserts and misses end after every bucket was
    # visited instead of spinning
    kb, cg = 4, 32
    g = wc.SingleValueHashTable(1, key_bytes=kb, cg_size=cg, probing=wc.PROBING_LINEAR)
    cap = g.capacity
    keys = o.gen_unique_keys(kb, cap + 64, 12)
    vals = o.gen_uniform(kb, keys.size, 13)
    st = empty_dev(cap, 4)
    g.insert(dev(keys[:cap]), dev(vals[:cap]), status_out=st)
    assert (host(st) == 0).all()
    assert g.size() == cap
    st2 = empty_dev(64, 4)
    g.insert(dev(keys[cap:]), dev(vals[cap:]), status_out=st2)
    assert (host(st2) == wc.Status.probing_length_exceeded().base()).all()
    out = empty_dev(64, kb)
    st3 = empty_dev(64, 4)
    g.retrieve(dev(keys[cap:]), out, status_out=st3)
    assert (host(st3) == wc.Status.probing_length_exceeded().base()).all()
    assert g.pop_status().has_probing_length_exceeded()


def test_empty_and_ragged_batches():
    g = wc.SingleValueHashTable(1000, key_bytes=8)
    k = empty_dev(0, 8)
    g.insert(k, k)
    g.retrieve(k, k)
    g.erase(k)
    for n in (1, 31, 33, 257, 1000):
        keys = o.gen_unique_keys(8, n, n)
        vals = o.gen_uniform(8, n, n + 1)
        g.init()
        g.insert(dev(keys), dev(vals))
        out = empty_dev(n, 8)
        g.retrieve(dev(keys), out)
        assert np.array_equal(host(out), vals)
        assert g.size() == n


def test_intra_batch_duplicates_keep_one_slot():
    # equal keys inside one batch: exactly one claim, the rest duplicates,
    # and the stored value is one of the inserted values
    g = wc.SingleValueHashTable(100000, key_bytes=4)
    base = o.gen_unique_keys(4, 1000, 21)
    keys = np.repeat(base, 7)
    rng = np.random.default_rng(0)
    rng.shuffle(keys)
    vals = o.gen_uniform(4, keys.size, 22)
    st = empty_dev(keys.size, 4)
    g.insert(dev(keys), dev(vals), status_out=st)
    s = host(st)
    assert (s == 0).sum() == base.size
    assert (s == wc.Status.duplicate_key().base()).sum() == keys.size - base.size
    assert g.size() == base.size
    out = empty_dev(base.size, 4)
    g.retrieve(dev(base), out)
    got = host(out)
    for kk, vv in zip(base[:50], got[:50]):
        assert vv in set(vals[keys == kk].tolist())


@pytest.mark.parametrize("block", [32, 64, 128, 256])
def test_results_do_not_depend_on_launch_geometry(block):
    # force one launch geometry for every tuning bucket of the u32 and u64
    # tables, run a full round trip, then restore the shipped tuning
    lib = wc.lib()
    try:
        for kb in (4, 8):
            for op in range(4):
                for lb in range(4):
                    for sb in range(12):
                        assert lib.wc_tune_set(kb, op, lb, sb, block, 1 if block == 32 else 0) == 0
        svht_round_trip(4, 8, n=5000)
        svht_round_trip(8, 8, n=5000)
    finally:
        lib.wc_tune_reset()
        wc._load_tuning(lib)


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("skew", ["zipf", "uniform"])
def test_counting_block_cache_path(kb, skew):
    # no per-key statuses: counts go through the per-block shared-memory
    # cache; counts and the table Status word must still match the oracle
    distinct = 20000
    occ = 300000
    g, r = make_pair(o.COUNTING, kb, 3 * distinct, 4)
    allk = o.gen_unique_keys(kb, distinct + 1000, 61)
    if skew == "zipf":
        ranks = o.gen_zipf_ranks(distinct, 1.1, occ, 62).astype(np.int64) - 1
    else:
        ranks = np.random.default_rng(63).integers(0, distinct, occ)
    keys = allk[ranks]
    # two calls: keys of the second are partly present already
    for part in (keys[: occ // 2], keys[occ // 2:]):
        g.insert(dev(part))
        r.insert(part)
        assert g.pop_status() == r.pop_status()
    out = empty_dev(allk.size, kb, SENT[kb])
    g.retrieve(dev(allk), out)
    r_out = r.retrieve(allk, np.full(allk.size, SENT[kb], dtype=allk.dtype))
    assert np.array_equal(host(out), r_out)
    assert g.size() == r.size()


@pytest.mark.parametrize("kb", [4, 8])
def test_counting_cache_and_direct_claims_agree(kb):
    """A counting insert without statuses adds through a per-block cache and
    straight into the table in the same launch (each block sees more keys
    than its cache holds). Both paths must claim a window's free slots in
    the same order, or one key can take two slots and split its count.
    Every key here appears 4 times; each of them must hold one slot with
    count 4, on several fresh tables."""
    import torch
    distinct = 1 << 19
    keys = o.gen_unique_keys(kb, distinct, 81)
    occ = np.repeat(keys, 4)
    for rep in range(3):
        perm = np.random.default_rng(90 + rep).permutation(occ.size)
        t = wc.CountingHashTable(int(distinct / 0.8), key_bytes=kb, cg_size=4)
        t.insert(dev(occ[perm]))
        assert t.size() == distinct, rep
        out = empty_dev(distinct, kb, 0)
        t.retrieve(dev(keys), out)
        assert bool((out == 4).all()), rep
        assert int(t.peek_status()) == o.ST_DUPLICATE_KEY


def test_launch_count_counts_this_librarys_kernels():
    # init is one fill kernel; a bulk call on a table without fingerprints
    # is one kernel; a retrieve on a fingerprint table is one kernel too
    t = wc.SingleValueHashTable(10000, key_bytes=4)
    keys = o.gen_unique_keys(4, 5000, 3)
    vals = o.gen_uniform(4, 5000, 4)
    dk, dv = dev(keys), dev(vals)
    out = empty_dev(5000, 4)
    c0 = wc.launch_count()
    t.init()
    t.insert(dk, dv)
    t.retrieve(dk, out)
    assert wc.launch_count() - c0 == 3
    assert np.array_equal(host(out), vals)


@pytest.mark.parametrize("kind,kb,vb,cg", [
    (o.SVHT, 4, 4, 8), (o.SVHT, 8, 8, 8), (o.SVHT, 4, 8, 4), (o.SVHT, 8, 4, 2),
    (o.HASHSET, 4, 0, 16), (o.HASHSET, 8, 0, 1), (o.COUNTING, 4, 4, 4), (o.COUNTING, 8, 8, 32)])
@pytest.mark.parametrize("policy", ["never", "always"])
def test_size_counter_matches_scan(kind, kb, vb, cg, policy):
    """size() reads the count that claims and erases maintain; after batches
    with in-batch duplicates (inserts and erases), re-inserts of erased keys
    and counting increments it equals the scan of the slot array and the
    oracle's size"""
    prev = wc.set_fingerprint_policy(policy)
    try:
        g, r = make_pair(kind, kb, 60000, cg, vb=None if kind == o.HASHSET else vb)
    finally:
        wc.set_fingerprint_policy(prev)
    assert g.has_fingerprints == (policy == "always")
    rng = np.random.default_rng(11)
    keys = o.gen_unique_keys(kb, 40000, 21)

    def ins(k):
        if kind == o.SVHT:
            v = o.gen_uniform(vb, k.size, int(k.size))
            g.insert(dev(k), dev(v))
            r.insert(k, v)
        else:
            g.insert(dev(k))
            r.insert(k)

    def check():
        assert g.size() == g.size_scan() == r.size()

    batch = np.concatenate([keys[:20000], keys[rng.integers(0, 20000, 5000)]])
    ins(batch[rng.permutation(batch.size)])
    check()
    er = np.concatenate([keys[:8000:2], keys[:8000:2], keys[30000:30100]])  # dups + absent
    er = er[rng.permutation(er.size)]
    g.erase(dev(er))
    r.erase(er)
    check()
    ins(np.concatenate([keys[:8000:4], keys[20000:40000]]))
    check()
    g.erase(dev(keys[::3]))
    r.erase(keys[::3])
    check()
    g.init()
    assert g.size() == g.size_scan() == 0
    ins(keys[:100])
    assert g.size() == 100
