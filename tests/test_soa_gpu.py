"""SingleValueHashTable stored as a struct of arrays (SoAStore,
storage.cuh:218-432; wc_svht_create_soa) against the oracle.

The key array is probed like a hash set's slots and the values sit in a
separate array, value i belonging to key slot i.  Every answer must equal
the oracle's, as for the AoS table: per-key statuses of insert, retrieve and
erase, retrieved values and untouched misses, sizes, table Status words and
the contents as multisets (tests.test_tables_gpu.svht_round_trip with
store="soa").  The memory itself is checked too: the slot array holds keys
only, the value array the values at the same indices."""
import numpy as np
import pytest

import warpcore_b200 as wc
from oracle import oracle as o
from tests.test_tables_gpu import svht_round_trip, make_pair
from tests.wc_helpers import copy_device_words, dev, empty_dev, host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kb,vb", [(4, 4), (8, 8), (4, 8), (8, 4)])
@pytest.mark.parametrize("cg", [1, 2, 4, 8, 16, 32])
def test_soa_round_trip(kb, vb, cg):
    svht_round_trip(kb, cg, vb=vb, store="soa")


@pytest.mark.parametrize("probing", [wc.PROBING_LINEAR, wc.PROBING_QUADRATIC])
def test_soa_other_probing(probing):
    svht_round_trip(8, 8, probing=probing, store="soa")


@pytest.mark.parametrize("load", [0.9, 0.97])
def test_soa_high_load(load):
    # the smallest capacity (131101 buckets of 8), filled to the load
    cap = wc.valid_capacity(1, 8)
    svht_round_trip(4, 8, n=int(cap * load), load=load, store="soa")


@pytest.mark.parametrize("kb,vb", [(8, 8), (4, 8)])
def test_soa_memory_is_two_arrays(kb, vb):
    g, r = make_pair(o.SVHT, kb, 50000, 8, vb=vb, store="soa")
    inf = g.info()
    assert inf.values and inf.slot_bytes == kb and not inf.fingerprints
    assert inf.bytes_total >= g.capacity * (kb + vb)
    keys = o.gen_unique_keys(kb, 40000, 3)
    vals = o.gen_uniform(vb, keys.size, 4)
    g.insert(dev(keys), dev(vals))
    hk = copy_device_words(inf.slots, g.capacity, kb)
    hv = copy_device_words(inf.values, g.capacity, vb)
    valid = (hk != 0) & (hk != np.array((1 << (8 * kb)) - 1, dtype=hk.dtype))
    assert int(valid.sum()) == keys.size
    order = np.argsort(keys)
    pos = np.searchsorted(keys[order], hk[valid])
    assert np.array_equal(keys[order][pos], hk[valid])
    assert np.array_equal(vals[order][pos], hv[valid])
    # a fresh init empties both arrays
    g.init()
    assert g.size() == 0
    assert not copy_device_words(inf.values, g.capacity, vb).any()


def test_soa_host_pipe_and_size():
    # the host-buffer path and the maintained size run on SoA tables too
    import torch
    g = wc.SingleValueHashTable(200000, key_bytes=8, store="soa")
    keys = o.gen_unique_keys(8, 100000, 8)
    vals = o.gen_uniform(8, keys.size, 9)
    pipe = wc.HostPipe()
    kt = torch.from_numpy(keys.view(np.int64)).pin_memory()
    vt = torch.from_numpy(vals.view(np.int64)).pin_memory()
    g.insert_from_host(pipe, kt, vt)
    out = torch.zeros(keys.size, dtype=torch.int64).pin_memory()
    g.retrieve_to_host(pipe, kt, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.numpy().view(np.uint64), vals)
    assert g.size() == g.size_scan() == keys.size


def test_soa_tables_are_not_batched():
    g = wc.SingleValueHashTable(1000, key_bytes=4, store="soa")
    keys = dev(o.gen_unique_keys(4, 100, 1))
    vals = dev(o.gen_uniform(4, 100, 2))
    b = wc.Batch(max_requests=4)
    with pytest.raises(wc.WarpcoreError):
        b.run([(g, "insert", keys, vals)])
    with pytest.raises(wc.WarpcoreError):
        wc.SingleValueHashTable(1000, store="columnar")


def test_soa_custom_sentinels():
    # the empty and tombstone keys of the key array are the table's own
    kb, n = 4, 5000
    g, r = make_pair(o.SVHT, kb, 8000, 8, empty=7, tomb=9, store="soa")
    keys = o.gen_unique_keys(kb, n, 3)
    keys = keys[(keys != 7) & (keys != 9)]
    keys = np.concatenate([keys, np.array([0, 0xFFFFFFFF, 7, 9], dtype=np.uint32)])
    vals = o.gen_uniform(kb, keys.size, 4)
    st = empty_dev(keys.size, 4)
    g.insert(dev(keys), dev(vals), status_out=st)
    assert np.array_equal(host(st), r.insert(keys, vals, want_status=True))
    out = empty_dev(keys.size, kb, 0xA5A5A5A5)
    g.retrieve(dev(keys), out)
    r_out = r.retrieve(keys, np.full(keys.size, 0xA5A5A5A5, dtype=np.uint32))
    assert np.array_equal(host(out), r_out)
    assert g.peek_status() == r.peek_status()
    assert g.size() == g.size_scan() == r.size()


def test_soa_full_table_reports_probing_length_exceeded():
    # every key slot taken: further inserts and misses end after every bucket
    g = wc.SingleValueHashTable(1, key_bytes=4, cg_size=32, probing=wc.PROBING_LINEAR,
                                store="soa")
    cap = g.capacity
    keys = o.gen_unique_keys(4, cap + 64, 12)
    vals = o.gen_uniform(4, keys.size, 13)
    st = empty_dev(cap, 4)
    g.insert(dev(keys[:cap]), dev(vals[:cap]), status_out=st)
    assert (host(st) == 0).all()
    assert g.size() == cap
    st2 = empty_dev(64, 4)
    g.insert(dev(keys[cap:]), dev(vals[cap:]), status_out=st2)
    assert (host(st2) == wc.Status.probing_length_exceeded().base()).all()
    out = empty_dev(cap, 4)
    g.retrieve(dev(keys[:cap]), out)
    assert np.array_equal(host(out), vals[:cap])
    assert g.pop_status().has_probing_length_exceeded()


def test_soa_boolean_handler_matches_oracle():
    n = 4000
    g, r = make_pair(o.SVHT, 4, 8000, 8, store="soa")
    keys = o.gen_unique_keys(4, 2 * n, 5)
    vals = o.gen_uniform(4, n, 6)
    g.insert(dev(keys[:n]), dev(vals))
    r.insert(keys[:n], vals)
    q = np.concatenate([keys, np.array([0, 0xFFFFFFFF], dtype=np.uint32)])
    for ignore in (0, wc.Status.key_not_found().base()):
        b = empty_dev(q.size, 1, 9)
        out = empty_dev(q.size, 4)
        g.retrieve(dev(q), out, status_out=b, status_handler=wc.HANDLER_BOOLEAN, ignore=ignore)
        _, r_st = r.retrieve(q, want_status=True)
        exp = np.array([o.status_to_bool(int(s), ignore) for s in r_st], dtype=np.uint8)
        assert np.array_equal(host(b), exp)
