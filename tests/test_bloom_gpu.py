"""Bloom filter parity with the oracle through the C ABI: every filter word
identical, query flags identical, zero false negatives."""
import numpy as np
import pytest

import warpcore_b200 as wc
from oracle import oracle as o
from tests.wc_helpers import copy_device_words, dev, empty_dev, host

pytestmark = pytest.mark.gpu


def words_of(f, slot_bytes):
    inf = f.info()
    return copy_device_words(inf.words, inf.num_slots, slot_bytes)


@pytest.mark.parametrize("kb,sb,cg,num_bits,k,n", [
    (8, 8, 8, 1 << 16, 8, 4000),
    (8, 8, 1, (1 << 16) + 100, 6, 3000),
    (4, 4, 4, 3000, 5, 300),
    (4, 8, 2, 5000, 3, 400),
    (8, 4, 16, 1 << 18, 7, 10000),
    (8, 8, 32, (1 << 20) + 4096 + 64, 10, 50000),
    (4, 4, 32, 12345, 4, 500),
])
def test_bloom_words_and_flags(kb, sb, cg, num_bits, k, n):
    f = wc.BloomFilter(num_bits, k, key_bytes=kb, slot_bytes=sb, cg_size=cg)
    r = o.Bloom(num_bits, k, key_bytes=kb, slot_bytes=sb, cg=cg)
    assert f.num_slots() == r.num_slots and f.num_blocks() == r.num_blocks
    allk = o.gen_unique_keys(kb, 2 * n, 77)
    keys = allk[:n]
    f.insert(dev(keys))
    r.insert(keys)
    assert np.array_equal(words_of(f, sb), r.words())
    flags = empty_dev(2 * n, 1, 9)
    f.retrieve(dev(allk), flags)
    rf = r.retrieve(allk)
    got = host(flags)
    assert np.array_equal(got, rf)
    assert got[:n].all()  # no false negatives


@pytest.mark.parametrize("kb,sb,cg,num_bits,k,n,region", [
    (8, 8, 8, 1 << 25, 8, 1 << 21, 1 << 20),              # 4 passes of 2^14 blocks
    (8, 8, 8, (1 << 25) + 512 * 3 + 64, 8, 1 << 20, 1 << 20),  # ragged last block
    (4, 4, 4, 3 << 23, 5, 1 << 19, 1 << 20),              # 16-byte blocks, 3 passes
    (8, 4, 16, (1 << 24) + 4096, 7, 1 << 18, 1 << 20),    # 3 uneven passes
])
def test_bloom_region_passes(kb, sb, cg, num_bits, k, n, region):
    """A filter larger than the random-access region runs in region passes;
    words and flags must not change."""
    prev = wc.set_region_bytes(region)
    try:
        f = wc.BloomFilter(num_bits, k, key_bytes=kb, slot_bytes=sb, cg_size=cg)
        allk = o.gen_unique_keys(kb, 2 * n, 78)
        keys = allk[:n]
        f.insert(dev(keys))
        flags = empty_dev(2 * n, 1, 9)
        f.retrieve(dev(allk), flags)
    finally:
        wc.set_region_bytes(prev)
    assert f.num_slots() * sb > region  # more than one pass ran
    r = o.Bloom(num_bits, k, key_bytes=kb, slot_bytes=sb, cg=cg)
    r.insert(keys)
    assert np.array_equal(words_of(f, sb), r.words())
    got = host(flags)
    assert np.array_equal(got, r.retrieve(allk))
    assert got[:n].all()


def test_bloom_config4_shape_fpr():
    # the filter shape of the 2^32-bit configuration at a reduced key count
    f = wc.BloomFilter(1 << 32, 8, key_bytes=8, slot_bytes=8, cg_size=8)
    assert (f.num_slots(), f.num_blocks()) == (1 << 26, 1 << 23)
    r_fpr = o.Bloom(1 << 32, 8, cg=8).fpr(1 << 20)
    assert f.fpr(1 << 20) == pytest.approx(r_fpr, rel=1e-12)
    keys = o.gen_unique_keys(8, 1 << 21, 5)
    f.insert(dev(keys[: 1 << 20]))
    flags = empty_dev(1 << 21, 1)
    f.retrieve(dev(keys), flags)
    got = host(flags)
    assert got[: 1 << 20].all()
    assert got[1 << 20:].mean() < 1e-3
