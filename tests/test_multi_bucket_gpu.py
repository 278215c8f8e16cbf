"""MultiBucketHashTable through the C ABI against the reference's own
outputs (tests/golden/ref_gpu, mb_* fixtures) and the oracle: insert
statuses with bucket sizes 1 to 8 and max_values_per_key, invalid keys and
values, per-key counts, offsets, every key's values in insertion order, dry
runs, unique keys, key / occupied-slot / value counts and table statuses.
In-batch duplicates are compared as per-key counts and status multisets,
since which copy lands where depends on the schedule (as in the
reference)."""
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


class GpuMB:
    """the oracle.MBTable interface over wc.MultiBucketHashTable"""

    def __init__(self, kb, vb, cap, bucket, max_values, **kw):
        self.kb, self.vb = kb, vb
        self.t = wc.MultiBucketHashTable(cap, key_bytes=kb, value_bytes=vb, bucket_size=bucket,
                                         max_values_per_key=max_values, **kw)

    @property
    def capacity(self):
        return self.t.capacity

    def insert(self, keys, values, want_status=False):
        st = empty_dev(len(keys), 4) if want_status else None
        self.t.insert(dev(keys), dev(values), status_out=st)
        return host(st) if want_status else None

    def num_keys(self):
        return self.t.num_keys()

    def num_occupied(self):
        return self.t.num_occupied()

    def size(self):
        return self.t.size()

    def pop_status(self):
        return int(self.t.pop_status())

    def retrieve(self, keys, dry_run=False):
        n = len(keys)
        b = torch.zeros(n, dtype=torch.int64, device="cuda")
        e = torch.zeros(n, dtype=torch.int64, device="cuda")
        st = empty_dev(n, 4)
        dk = dev(keys)
        if dry_run:
            self.t.retrieve(dk, b, e, None, status_out=st)
            return None, host(e), None, host(st)
        total = self.t.num_values(dk)
        v = empty_dev(max(total, 1), self.vb)
        num = self.t.retrieve(dk, b, e, v, status_out=st)
        assert num == total
        return host(b), host(e), host(v)[:num], host(st)

    def unique_keys(self):
        n = self.t.retrieve_all_keys()
        out = empty_dev(max(n, 1), self.kb)
        m = self.t.retrieve_all_keys(out)
        return host(out)[:m]


@pytest.mark.parametrize("tag,kb,vb", gs.MB_CASES)
def test_multi_bucket_golden(tag, kb, vb):
    gs.mb_scenario(F, tag, kb, vb, lambda cap, bucket, mx: GpuMB(kb, vb, cap, bucket, mx))


@pytest.mark.parametrize("kb,vb", [(4, 4), (4, 8), (8, 4), (8, 8)])
@pytest.mark.parametrize("bucket,cg", [(1, 8), (2, 8), (4, 4), (8, 8), (3, 16), (2, 32)])
@pytest.mark.parametrize("max_values", [2**64 - 1, 5])
def test_multi_bucket_vs_oracle(kb, vb, bucket, cg, max_values):
    # rounds of unique keys (each key's values arrive one per round): exact
    # statuses, counters, offsets and values in insertion order
    n = 3000
    keys = o.gen_unique_keys(kb, n + 500, 301 + cg + bucket)
    cap = 6 * n
    g = GpuMB(kb, vb, cap, bucket, max_values, cg_size=cg)
    r = o.MBTable(kb, vb, cap, bucket=bucket, cg=cg, max_values_per_key=max_values)
    assert g.capacity == r.capacity
    for rnd in range(7):
        m = n - rnd * 400
        v = o.gen_uniform(vb, m, 400 + rnd)
        v[v == 0] = 1
        assert np.array_equal(g.insert(keys[:m], v, want_status=True),
                              r.insert(keys[:m], v, want_status=True)), rnd
    assert g.num_keys() == r.num_keys()
    assert g.num_occupied() == r.num_occupied()
    assert g.size() == r.size()
    q = np.concatenate([keys, keys[:100]])
    gb, ge, gv, gst = g.retrieve(q)
    rb, re, rv, rst = r.retrieve(q)
    assert np.array_equal(gb, rb) and np.array_equal(ge, re)
    assert np.array_equal(gv, rv)
    assert np.array_equal(gst, rst)
    assert g.pop_status() == r.pop_status()
    assert np.array_equal(np.sort(g.unique_keys()), np.sort(r.unique_keys()))


@pytest.mark.parametrize("bucket,max_values", [(1, 2**64 - 1), (2, 2**64 - 1), (2, 3), (4, 4),
                                               (8, 5)])
def test_multi_bucket_in_batch_duplicates(bucket, max_values):
    # one batch with every key 6 times, shuffled: counts and per-key status
    # multisets equal the sequential oracle's; the stored values are the
    # key's own (all of them when nothing is capped)
    kb = vb = 4
    keys = o.gen_unique_keys(kb, 2000, 17 + bucket)
    rep = np.repeat(keys, 6)
    vals = np.arange(1, rep.size + 1, dtype=np.uint32)
    perm = np.random.default_rng(bucket).permutation(rep.size)
    rep, vals = rep[perm], vals[perm]
    g = GpuMB(kb, vb, 20000, bucket, max_values)
    r = o.MBTable(kb, vb, 20000, bucket=bucket, max_values_per_key=max_values)
    gst = g.insert(rep, vals, want_status=True)
    rst = r.insert(rep, vals, want_status=True)
    a, b = np.lexsort((gst, rep)), np.lexsort((rst, rep))
    assert np.array_equal(gst[a], rst[b])
    assert g.num_keys() == r.num_keys() == keys.size
    assert g.num_occupied() == r.num_occupied()
    assert g.size() == r.size()
    gb, ge, gv, _ = g.retrieve(keys)
    rb, re, rv, _ = r.retrieve(keys)
    assert np.array_equal(ge, re)
    owner = dict(zip(vals.tolist(), rep.tolist()))
    for i in range(keys.size):
        got = gv[gb[i]:ge[i]].tolist()
        assert all(owner[x] == keys[i] for x in got)
        if max_values >= 6:
            assert sorted(got) == sorted(rv[rb[i]:re[i]].tolist())


def test_multi_bucket_edges():
    kb = vb = 8
    t = GpuMB(kb, vb, 1000, 2, 2**64 - 1)
    # empty batches are no-ops
    t.t.insert(torch.empty(0, dtype=torch.int64, device="cuda"),
               torch.empty(0, dtype=torch.int64, device="cuda"))
    assert t.size() == 0 and t.num_keys() == 0
    # invalid keys (empty, tombstone) and the empty value
    keys = np.array([0, 2**64 - 1, 5, 6], dtype=np.uint64)
    vals = np.array([1, 1, 0, 9], dtype=np.uint64)
    st = t.insert(keys, vals, want_status=True)
    assert st.tolist() == [o.ST_INVALID_KEY, o.ST_INVALID_KEY, 1 << 12, 0]
    assert t.pop_status() == o.ST_INVALID_KEY | (1 << 12)
    _, e, v, st = t.retrieve(np.array([6, 5], dtype=np.uint64))
    assert e.tolist() == [1, 1] and v.tolist() == [9]
    assert st.tolist() == [0, o.ST_KEY_NOT_FOUND]
    # with a probing length of one window, a key's ninth value (bucket 1,
    # CG 8) finds no free slot: probing_length_exceeded + duplicate_key
    small = wc.MultiBucketHashTable(1000, key_bytes=4, value_bytes=4, bucket_size=1)
    got = []
    for i in range(9):
        st = empty_dev(1, 4)
        small.insert(dev(np.array([77], dtype=np.uint32)), dev(np.array([i + 1], dtype=np.uint32)),
                     probing_length=8, status_out=st)
        got.append(int(host(st)[0]))
    assert got == [0] + [o.ST_DUPLICATE_KEY] * 7 + [o.ST_PROBING_LENGTH_EXCEEDED | o.ST_DUPLICATE_KEY]
    assert small.size() == 8 and small.num_occupied() == 8 and small.num_keys() == 1
    assert small.pop_status() == o.ST_PROBING_LENGTH_EXCEEDED | o.ST_DUPLICATE_KEY
    # bucket larger than the group and a zero bucket are refused
    with pytest.raises(wc.WarpcoreError):
        wc.MultiBucketHashTable(100, bucket_size=16, cg_size=8)
    with pytest.raises(wc.WarpcoreError):
        wc.MultiBucketHashTable(100, bucket_size=0)


def test_multi_bucket_load_factors_and_init():
    t = wc.MultiBucketHashTable(10000, key_bytes=4, value_bytes=4, bucket_size=4)
    keys = dev(o.gen_unique_keys(4, 1000, 3))
    vals = dev(np.arange(1, 1001, dtype=np.uint32))
    for _ in range(3):
        t.insert(keys, vals)
    assert t.num_keys() == 1000 and t.num_occupied() == 1000 and t.size() == 3000
    assert t.key_load_factor() == pytest.approx(1000 / t.capacity)
    assert t.value_load_factor() == pytest.approx(3000 / (4 * t.capacity))
    assert t.relative_storage_density() == pytest.approx(
        (1000 * 4 + 3000 * 4) / (1000 * 4 + 3000 * 4))
    assert 0 < t.storage_density() < 1
    t.init()
    assert t.size() == 0 and t.num_keys() == 0 and t.num_occupied() == 0
    assert t.retrieve_all_keys() == 0


@pytest.mark.parametrize("table", ["mb", "mv"])
def test_offsets_begin_end_one_apart(table):
    # the reference's idiom retrieve(keys, n, offsets, offsets + 1, ...):
    # one array of n + 1 offsets, end[i] == begin[i + 1]
    n = 200_000
    keys = o.gen_unique_keys(4, n, 61)
    rep = np.repeat(keys[: n // 2], 3)
    vals = np.arange(1, rep.size + 1, dtype=np.uint32)
    if table == "mb":
        t = wc.MultiBucketHashTable(4 * n, key_bytes=4, value_bytes=4, bucket_size=2)
    else:
        t = wc.MultiValueHashTable(4 * n, key_bytes=4)
    t.insert(dev(rep), dev(vals))
    dq = dev(keys)
    b = torch.zeros(n, dtype=torch.int64, device="cuda")
    e = torch.zeros(n, dtype=torch.int64, device="cuda")
    v1 = empty_dev(rep.size, 4)
    total = t.retrieve(dq, b, e, v1)
    off = torch.full((n + 1,), 7, dtype=torch.int64, device="cuda")
    v2 = empty_dev(rep.size, 4)
    total2 = t.retrieve(dq, off[:-1], off[1:], v2)
    assert total == total2 == rep.size
    assert torch.equal(off[:-1], b) and torch.equal(off[1:], e)
    assert torch.equal(v1, v2)
