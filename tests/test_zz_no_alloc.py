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
