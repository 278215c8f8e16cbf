"""wc_slots_size_noalloc, the entry point for callers that may not allocate
device memory (they hold a table's slot array without a handle of this
library, e.g. memory received through CUDA IPC, or run inside a framework
that owns all device memory).  Its count must equal the regular
wc_table_size on the same table, on two calls in a row with different
contents, since both calls share the library's fixed scratch array.

This file is collected last so that a run stopping at the first failure has
run every other test first."""
import ctypes

import numpy as np
import pytest

import warpcore_b200 as wc
from oracle import oracle as o
from tests.wc_helpers import dev

pytestmark = pytest.mark.gpu


def noalloc_size(t):
    import torch
    inf = t.info()
    out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    rc = wc.lib().wc_slots_size_noalloc(inf.slots, inf.capacity, inf.key_bytes,
                                        inf.value_bytes, inf.empty_key, inf.tombstone_key,
                                        torch.cuda.current_stream().cuda_stream, out.data_ptr())
    assert rc == 0, wc.lib().wc_last_error()
    return int(out.item())


@pytest.mark.parametrize("kind,kb,cg", [("svht", 8, 8), ("svht", 4, 1), ("set", 4, 1),
                                        ("set", 8, 16), ("count", 4, 4)])
def test_matches_table_size_on_two_calls(kind, kb, cg):
    n = 300000
    if kind == "svht":
        t = wc.SingleValueHashTable(n, key_bytes=kb, cg_size=cg)
    elif kind == "set":
        t = wc.HashSet(n, key_bytes=kb, cg_size=cg)
    else:
        t = wc.CountingHashTable(n, key_bytes=kb, cg_size=cg)
    keys = o.gen_unique_keys(kb, n, 99)
    vals = o.gen_uniform(kb, n, 98)

    def ins(k, v):
        if kind == "svht":
            t.insert(dev(k), dev(v))
        else:
            t.insert(dev(k))

    ins(keys[: n // 2], vals[: n // 2])
    first = noalloc_size(t)
    assert first == t.size() == n // 2
    # second call on changed contents: more keys and some tombstones
    ins(keys[n // 2:], vals[n // 2:])
    t.erase(dev(keys[::7]))
    second = noalloc_size(t)
    assert second == t.size()
    assert second == n - keys[::7].size


def test_rejects_slot_arrays_beyond_the_limit():
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    t = wc.SingleValueHashTable(1000, key_bytes=8)
    inf = t.info()
    rc = wc.lib().wc_slots_size_noalloc(inf.slots, (1 << 34) + 1, 8, 8, 0, 2**64 - 1,
                                        None, out.data_ptr())
    assert rc == -1
    assert b"2^34" in wc.lib().wc_last_error()
    assert int(out.item()) == 0  # nothing was launched


def test_empty_slot_array_counts_zero():
    import torch
    out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    rc = wc.lib().wc_slots_size_noalloc(None, 0, 4, 4, 0, 2**32 - 1,
                                        torch.cuda.current_stream().cuda_stream, out.data_ptr())
    assert rc == 0
    assert int(out.item()) == 0


def noalloc_count(slots, capacity, key_bytes, value_bytes, empty, tomb):
    import torch
    out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    rc = wc.lib().wc_slots_size_noalloc(slots, capacity, key_bytes, value_bytes, empty, tomb,
                                        torch.cuda.current_stream().cuda_stream, out.data_ptr())
    assert rc == 0, wc.lib().wc_last_error()
    return int(out.item())


@pytest.mark.parametrize("kind,kb", [("svht", 4), ("set", 4), ("set", 8)])
def test_ragged_prefix_against_host_count(kind, kb):
    """A prefix of 2^18 + 3 slots of a larger table: the last chunk holds 3
    slots, fewer than one 16-byte load for 4-byte set keys, and not a
    multiple of the slots per load for 8-byte slots; the count must equal a
    host count of the same slots copied back."""
    from tests.wc_helpers import copy_device_words
    n = 400000
    t = (wc.SingleValueHashTable(n, key_bytes=kb, cg_size=1) if kind == "svht"
         else wc.HashSet(n, key_bytes=kb, cg_size=1))
    keys = o.gen_unique_keys(kb, n // 2, 97)
    if kind == "svht":
        t.insert(dev(keys), dev(o.gen_uniform(kb, n // 2, 96)))
    else:
        t.insert(dev(keys))
    t.erase(dev(keys[::5]))
    inf = t.info()
    prefix = (1 << 18) + 3
    assert inf.capacity > prefix
    vb = 0 if kind == "set" else kb
    slot_bytes = kb + vb
    words = copy_device_words(inf.slots, prefix * slot_bytes // kb, kb)
    host_keys = words[:: slot_bytes // kb]
    expect = int(((host_keys != inf.empty_key) & (host_keys != inf.tombstone_key)).sum())
    assert 0 < expect < prefix
    for _ in range(2):
        assert noalloc_count(inf.slots, prefix, kb, vb, inf.empty_key, inf.tombstone_key) == expect


def test_multi_bucket_key_array_counted_as_keys_only():
    """The multi-bucket table keeps its keys in an array of their own, and
    its info reports value_bytes equal to key_bytes.  Passed with
    value_bytes 0, the key array counts exactly the table's keys."""
    n = 50000
    t = wc.MultiBucketHashTable(4 * n, key_bytes=4, bucket_size=2)
    keys = o.gen_unique_keys(4, n, 95)
    vals = o.gen_uniform(4, n, 94)
    vals[vals == 0] = 1
    t.insert(dev(keys), dev(vals))
    inf = t.info()
    assert inf.value_bytes == inf.key_bytes
    got = noalloc_count(inf.keys, inf.capacity, inf.key_bytes, 0, inf.empty_key,
                        inf.tombstone_key)
    assert got == t.num_keys() == n


def test_soa_key_array_counted_as_keys_only():
    # a struct-of-arrays single-value table: its slot array holds keys only
    # and is counted with value_bytes 0
    import torch
    n = 200000
    t = wc.SingleValueHashTable(n, key_bytes=8, store="soa")
    keys = o.gen_unique_keys(8, n, 97)
    t.insert(dev(keys), dev(o.gen_uniform(8, n, 96)))
    t.erase(dev(keys[::5]))
    inf = t.info()
    out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    rc = wc.lib().wc_slots_size_noalloc(inf.slots, inf.capacity, inf.key_bytes, 0,
                                        inf.empty_key, inf.tombstone_key,
                                        torch.cuda.current_stream().cuda_stream, out.data_ptr())
    assert rc == 0, wc.lib().wc_last_error()
    assert int(out.item()) == t.size() == n - keys[::5].size
