"""L2 persistence windows: tables that fit in the device's persisting-L2
maximum launch with an access-policy window, larger ones without, and the
answers are the same with windows on and off."""
import numpy as np
import pytest
import torch

import warpcore_b200 as wc
from oracle import oracle as o
from tests.wc_helpers import copy_device_words, dev, host

pytestmark = pytest.mark.gpu


def _persist_max():
    return torch.cuda.get_device_properties(0).L2_cache_size  # upper bound of the maximum


def test_small_table_has_window_large_has_none():
    small = wc.SingleValueHashTable(1 << 16, key_bytes=4)
    b, r = small.l2_window()
    assert b == small.capacity * 8
    assert 0.0 < r <= 1.0
    big = wc.SingleValueHashTable(_persist_max() // 8 + (1 << 20), key_bytes=4)
    assert big.l2_window() == (0, 0.0)


def test_windows_off_reports_none_and_back_on():
    t = wc.SingleValueHashTable(1 << 16, key_bytes=8)
    prev = wc.set_l2_persistence(False)
    try:
        assert t.l2_window() == (0, 0.0)
    finally:
        wc.set_l2_persistence(prev)
    assert t.l2_window()[0] == t.capacity * 16


@pytest.mark.parametrize("kb", [4, 8])
def test_same_answers_with_and_without_window(kb):
    n = 200000
    keys = o.gen_unique_keys(kb, n + n // 2, 41)
    vals = o.gen_uniform(kb, n, 42)
    q = np.concatenate([keys[:n:2], keys[n:]])
    res = []
    for on in (True, False):
        prev = wc.set_l2_persistence(on)
        try:
            t = wc.SingleValueHashTable(int(n / 0.9), key_bytes=kb)
            assert (t.l2_window()[0] > 0) == on
            t.insert(dev(keys[:n]), dev(vals))
            out = torch.zeros(q.size, dtype=torch.int32 if kb == 4 else torch.int64, device="cuda")
            st = torch.zeros(q.size, dtype=torch.int32, device="cuda")
            t.retrieve(dev(q), out, status_out=st)
            res.append((host(out), host(st), t.size()))
            del t
        finally:
            wc.set_l2_persistence(prev)
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1], res[1][1])
    assert res[0][2] == res[1][2] == n
    ref = o.Table(o.SVHT, kb, kb, int(n / 0.9))
    ref.insert(keys[:n], vals)
    r_out, _ = ref.retrieve(q, np.zeros(q.size, dtype=keys.dtype), want_status=True)
    assert np.array_equal(res[0][0], r_out)


def test_bloom_window_same_words():
    keys = o.gen_unique_keys(8, 50000, 43)
    words = []
    for on in (True, False):
        prev = wc.set_l2_persistence(on)
        try:
            f = wc.BloomFilter(1 << 22, 6, key_bytes=8, slot_bytes=8, cg_size=8)
            f.insert(dev(keys))
            torch.cuda.synchronize()
            words.append(copy_device_words(f.words_ptr(), f.num_slots(), 8))
            flags = torch.zeros(keys.size, dtype=torch.uint8, device="cuda")
            f.retrieve(dev(keys), flags)
            assert host(flags).all()
        finally:
            wc.set_l2_persistence(prev)
    assert np.array_equal(words[0], words[1])


def test_windows_share_the_set_aside():
    # 16 MiB tables: windows are handed out while they fit the set-aside
    # together; a freed window's bytes go to the next table
    l2 = torch.cuda.get_device_properties(0).L2_cache_size
    tables = [wc.SingleValueHashTable((16 << 20) // 8 - 4096, key_bytes=4) for _ in range(l2 // (16 << 20) + 2)]
    win = [t.l2_window()[0] for t in tables]
    assert win[0] > 0
    assert 0 in win
    first_without = win.index(0)
    assert all(w > 0 for w in win[:first_without])
    assert sum(win) <= l2
    del tables[0]
    extra = wc.SingleValueHashTable((16 << 20) // 8 - 4096, key_bytes=4)
    assert extra.l2_window()[0] > 0
