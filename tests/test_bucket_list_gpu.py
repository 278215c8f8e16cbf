"""BucketListHashTable through the C ABI against the reference's own outputs
(tests/golden/ref_gpu, bl_* fixtures) and the oracle: per-key statuses,
list lengths, offsets, every key's values in list order (newest bucket
first), bucket growth (grow factor, minimum and maximum bucket sizes, the
handle bit widths), max_values_per_key, pool use and exhaustion, dry runs
and all keys.  Batches that hold a key more than once append its values in
a schedule-dependent order (as in the reference), so they are compared as
per-key multisets."""
import numpy as np
import pytest
import torch

import warpcore_b200 as wc
from oracle import oracle as o
from tests import golden_scenarios as gs
from tests.golden_io import fixtures
from tests.wc_helpers import dev, empty_dev, host

pytestmark = pytest.mark.gpu

F = fixtures("ref_gpu")


class GpuBL:
    """the oracle.BLTable interface over wc.BucketListHashTable"""

    def __init__(self, kb, vb, key_cap, value_cap, **kw):
        self.kb, self.vb = kb, vb
        self.t = wc.BucketListHashTable(key_cap, value_cap, key_bytes=kb, value_bytes=vb, **kw)

    @property
    def key_capacity(self):
        return self.t.key_capacity

    def insert(self, keys, values, want_status=False, status_fill=0):
        st = empty_dev(len(keys), 4, fill=status_fill) if want_status else None
        self.t.insert(dev(keys), dev(values), status_out=st)
        return host(st) if want_status else None

    def num_keys(self):
        return self.t.num_keys()

    def total_values(self):
        return self.t.num_values()

    def next_free(self):
        return self.t.pool_used()

    def pop_status(self):
        return int(self.t.pop_status())

    def retrieve(self, keys, dry_run=False, fill=0):
        n = len(keys)
        b = torch.zeros(n, dtype=torch.int64, device="cuda")
        e = torch.zeros(n, dtype=torch.int64, device="cuda")
        st = empty_dev(n, 4)
        dk = dev(keys)
        if dry_run:
            self.t.retrieve(dk, b, e, None, status_out=st)
            return None, host(e), None, host(st)
        total = self.t.num_values(dk)
        v = empty_dev(max(total, 1), self.vb, fill=fill)
        num = self.t.retrieve(dk, b, e, v, status_out=st)
        assert num == total
        return host(b), host(e), host(v)[:num], host(st)

    def all_keys(self):
        n = self.t.retrieve_all_keys()
        out = empty_dev(max(n, 1), self.kb)
        m = self.t.retrieve_all_keys(out)
        return host(out)[:m]


def _gpu(kb, vb):
    def make(key_cap, value_cap, grow, min_b, max_b, mx, bits):
        return GpuBL(kb, vb, key_cap, value_cap, grow_factor=grow, min_bucket_size=min_b,
                     max_bucket_size=max_b, max_values_per_key=mx, bits=bits)
    return make


@pytest.mark.parametrize("tag,kb,vb", gs.BL_CASES)
def test_bucket_list_golden(tag, kb, vb):
    gs.bl_scenario(F, tag, kb, vb, _gpu(kb, vb))


CONFIGS = [
    dict(grow_factor=1.1, min_bucket_size=1, max_bucket_size=1023, bits=(32, 20, 10)),
    dict(grow_factor=2.0, min_bucket_size=3, max_bucket_size=16, bits=(32, 20, 10)),
    dict(grow_factor=1.0, min_bucket_size=2, max_bucket_size=2, bits=(29, 18, 15)),
    dict(grow_factor=1.5, min_bucket_size=1, max_bucket_size=7, bits=(24, 5, 3), max_values_per_key=9),
]


@pytest.mark.parametrize("kb,vb", [(4, 4), (4, 8), (8, 4), (8, 8)])
@pytest.mark.parametrize("ci", range(len(CONFIGS)))
@pytest.mark.parametrize("cg", [8, 16])
def test_bucket_list_vs_oracle(kb, vb, ci, cg):
    # rounds of unique keys: every key's list is built in a fixed order, so
    # statuses, list order, counts and pool use are exact
    cfg = dict(CONFIGS[ci])
    n = 2048
    keys = o.gen_unique_keys(kb, n + 256, 501 + ci + cg)
    g = GpuBL(kb, vb, 2 * n, 40 * n, cg_size=cg, **cfg)
    r = o.BLTable(kb, vb, 2 * n, 40 * n, cg=cg, **cfg)
    assert g.key_capacity == r.key_capacity
    for rnd in range(12):
        m = n - rnd * 160
        v = o.gen_uniform(vb, m, 600 + rnd)
        assert np.array_equal(g.insert(keys[:m], v, want_status=True),
                              r.insert(keys[:m], v, want_status=True)), rnd
    assert g.num_keys() == r.num_keys()
    assert g.total_values() == r.total_values()
    assert g.next_free() == r.next_free()
    q = np.concatenate([keys, keys[:50]])
    gb, ge, gv, gst = g.retrieve(q)
    rb, re, rv, rst = r.retrieve(q)
    assert np.array_equal(gb, rb) and np.array_equal(ge, re)
    assert np.array_equal(gv, rv)
    assert np.array_equal(gst, rst)
    assert g.pop_status() == r.pop_status()
    assert np.array_equal(np.sort(g.all_keys()), np.sort(r.all_keys()))


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_bucket_list_in_batch_duplicates(ci):
    # every key 7 times in one shuffled batch, and copies far apart in a
    # large batch (as the reference's benchmark): list lengths, pool use and
    # per-key status multisets equal the oracle's; each list holds the
    # key's own values (all of them when nothing is capped)
    cfg = dict(CONFIGS[ci])
    kb = vb = 4
    keys = o.gen_unique_keys(kb, 3000, 31 + ci)
    rep = np.repeat(keys, 7)
    vals = np.arange(1, rep.size + 1, dtype=np.uint32)
    perm = np.random.default_rng(ci).permutation(rep.size)
    rep, vals = rep[perm], vals[perm]
    g = GpuBL(kb, vb, 4000, 30 * 3000, **cfg)
    r = o.BLTable(kb, vb, 4000, 30 * 3000, **cfg)
    gst = g.insert(rep, vals, want_status=True)
    rst = r.insert(rep, vals, want_status=True)
    a, b = np.lexsort((gst, rep)), np.lexsort((rst, rep))
    assert np.array_equal(gst[a], rst[b])
    assert g.num_keys() == r.num_keys() == keys.size
    assert g.total_values() == r.total_values()
    assert g.next_free() == r.next_free()
    gb, ge, gv, _ = g.retrieve(keys)
    rb, re, rv, _ = r.retrieve(keys)
    assert np.array_equal(ge, re)
    owner = dict(zip(vals.tolist(), rep.tolist()))
    capped = cfg.get("max_values_per_key", 2**20) < 7
    for i in range(keys.size):
        got = gv[gb[i]:ge[i]].tolist()
        assert all(owner[x] == keys[i] for x in got)
        if not capped:
            assert sorted(got) == sorted(rv[rb[i]:re[i]].tolist())


def test_bucket_list_far_apart_copies():
    # 2^20 values, key i mod 2^17 + 1 (8 copies 2^17 apart), the reference
    # benchmark's shape at a small size, store bits 29 / 18 / 15
    n, distinct = 1 << 20, 1 << 17
    keys = (np.arange(n, dtype=np.uint32) % distinct) + 1
    vals = np.arange(1, n + 1, dtype=np.uint32)
    g = GpuBL(4, 4, int(distinct / 0.9), 2 * n, bits=(29, 18, 15))
    r = o.BLTable(4, 4, int(distinct / 0.9), 2 * n, bits=(29, 18, 15))
    st = g.insert(keys, vals, want_status=True)
    r.insert(keys, vals)
    assert int((st == 0).sum()) == distinct and int((st == o.ST_DUPLICATE_KEY).sum()) == n - distinct
    assert g.total_values() == n and g.num_keys() == distinct
    assert g.next_free() == r.next_free()
    q = np.arange(1, 2 * distinct + 1, dtype=np.uint32)
    gb, ge, gv, gst = g.retrieve(q)
    assert np.all(ge[:distinct] - gb[:distinct] == 8) and np.all(ge[distinct:] == ge[distinct - 1])
    assert np.all(gst[:distinct] == 0) and np.all(gst[distinct:] == o.ST_KEY_NOT_FOUND)
    got = np.sort(gv.reshape(distinct, 8), axis=1)
    want = np.sort((np.arange(8)[None, :] * distinct + np.arange(distinct)[:, None] + 1).astype(np.uint32), axis=1)
    assert np.array_equal(got, want)


def test_bucket_list_pool_exhaustion():
    # a pool of 3000 elements for 2000 keys x 4 values: appends that need a
    # new bucket fail with out_of_memory once the pool is used up; what is
    # stored stays readable and consistent
    kb = vb = 4
    keys = o.gen_unique_keys(kb, 2000, 77)
    g = GpuBL(kb, vb, 4000, 3000)
    stored = 0
    for rnd in range(4):
        v = np.full(2000, rnd + 1, dtype=np.uint32)
        st = g.insert(keys, v, want_status=True)
        dup, oom = o.ST_DUPLICATE_KEY, o.ST_OUT_OF_MEMORY
        assert set(np.unique(st).tolist()) <= {0, dup, oom, dup | oom}
        stored += int(((st & o.ST_OUT_OF_MEMORY) == 0).sum())
    assert g.total_values() == stored
    assert g.next_free() >= 3000
    assert g.pop_status() & o.ST_OUT_OF_MEMORY
    b, e, v, rst = g.retrieve(keys, fill=0xFFFFFFFF)
    assert int((e - b).sum()) == stored


def test_bucket_list_edges():
    t = wc.BucketListHashTable(1000, 10000, key_bytes=8, value_bytes=8)
    t.insert(torch.empty(0, dtype=torch.int64, device="cuda"),
             torch.empty(0, dtype=torch.int64, device="cuda"))
    assert t.num_keys() == 0 and t.num_values() == 0 and t.pool_used() == 0
    st = empty_dev(3, 4)
    t.insert(dev(np.array([0, 2**64 - 1, 5], dtype=np.uint64)),
             dev(np.array([1, 2, 3], dtype=np.uint64)), status_out=st)
    assert host(st).tolist() == [o.ST_INVALID_KEY, o.ST_INVALID_KEY, 0]
    assert t.pop_status() == o.ST_INVALID_KEY
    # configurations the store refuses
    with pytest.raises(wc.WarpcoreError):
        wc.BucketListHashTable(100, 1000, grow_factor=0.5)
    with pytest.raises(wc.WarpcoreError):
        wc.BucketListHashTable(100, 1000, min_bucket_size=4, max_bucket_size=2)
    with pytest.raises(wc.WarpcoreError):
        wc.BucketListHashTable(100, 1 << 24, bits=(24, 20, 10))
    # init empties every list and the pool
    t.insert(dev(np.array([7, 7, 8], dtype=np.uint64)), dev(np.array([1, 2, 3], dtype=np.uint64)))
    assert t.num_values() == 4 and t.num_keys() == 3   # with key 5 from above
    t.init()
    assert t.num_values() == 0 and t.num_keys() == 0 and t.pool_used() == 0


def test_bucket_list_offsets_one_apart():
    n = 100_000
    keys = o.gen_unique_keys(4, n, 62)
    rep = np.repeat(keys[: n // 2], 3)
    t = wc.BucketListHashTable(n, 4 * rep.size, key_bytes=4)
    t.insert(dev(rep), dev(np.arange(1, rep.size + 1, dtype=np.uint32)))
    dq = dev(keys)
    b = torch.zeros(n, dtype=torch.int64, device="cuda")
    e = torch.zeros(n, dtype=torch.int64, device="cuda")
    v1 = empty_dev(rep.size, 4)
    assert t.retrieve(dq, b, e, v1) == rep.size
    off = torch.full((n + 1,), 7, dtype=torch.int64, device="cuda")
    v2 = empty_dev(rep.size, 4)
    assert t.retrieve(dq, off[:-1], off[1:], v2) == rep.size
    assert torch.equal(off[:-1], b) and torch.equal(off[1:], e) and torch.equal(v1, v2)
