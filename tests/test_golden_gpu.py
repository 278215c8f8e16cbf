"""The CUDA library, called through the C ABI, reproduces the outputs the
reference's own CUDA code produced on the same inputs
(tests/golden/ref_gpu): per-key statuses, retrieved values, membership
flags, counts, sizes, table Status words and every Bloom filter word."""
import numpy as np
import pytest

import warpcore_b200 as wc
from tests import golden_scenarios as gs
from tests.golden_io import fixtures
from tests.wc_helpers import copy_device_words, dev, empty_dev, host

pytestmark = pytest.mark.gpu

F = fixtures("ref_gpu")


class TableAdapter:
    """numpy-in / numpy-out view of a warpcore_b200 table, shaped like
    oracle.Table"""

    def __init__(self, t, kb, vb):
        self.t, self.kb, self.vb = t, kb, vb

    @property
    def capacity(self):
        return self.t.capacity

    def size(self):
        return self.t.size()

    def pop_status(self):
        return self.t.pop_status().base()

    def insert(self, keys, values=None, want_status=False):
        st = empty_dev(keys.size, 4)
        if values is None:
            self.t.insert(dev(keys), status_out=st)
        else:
            self.t.insert(dev(keys), dev(values), status_out=st)
        return host(st)

    def retrieve(self, keys, out, want_status=True):
        o = dev(out)
        st = empty_dev(keys.size, 4)
        self.t.retrieve(dev(keys), o, status_out=st)
        return host(o), host(st)

    def erase(self, keys, want_status=True):
        st = empty_dev(keys.size, 4)
        self.t.erase(dev(keys), status_out=st)
        return host(st)


class BloomAdapter:
    def __init__(self, b, sb):
        self.b, self.sb = b, sb
        self.num_slots = b.num_slots()
        self.num_blocks = b.num_blocks()

    def insert(self, keys):
        self.b.insert(dev(keys))

    def words(self):
        inf = self.b.info()
        return copy_device_words(inf.words, inf.num_slots, self.sb)

    def retrieve(self, keys):
        f = empty_dev(keys.size, 1, 9)
        self.b.retrieve(dev(keys), f)
        return host(f)


@pytest.mark.parametrize("tag,kb,vb", gs.SVHT_CASES)
def test_svht(tag, kb, vb):
    gs.svht_scenario(F, tag, kb, lambda cap: TableAdapter(
        wc.SingleValueHashTable(cap, key_bytes=kb, value_bytes=vb), kb, vb), vb)


@pytest.mark.parametrize("tag,kb", gs.SET_CASES)
def test_hashset(tag, kb):
    gs.set_scenario(F, tag, kb, lambda cap: TableAdapter(wc.HashSet(cap, key_bytes=kb), kb, 1))


@pytest.mark.parametrize("tag,vb", gs.COUNT_CASES)
def test_counting(tag, vb):
    gs.counting_scenario(F, tag, lambda cap, mx: TableAdapter(
        wc.CountingHashTable(cap, max_count=mx, key_bytes=4, value_bytes=vb), 4, vb), vb)


@pytest.mark.parametrize("tag", gs.BLOOM_CASES)
def test_bloom(tag):
    def make(kb, sb, cg, num_bits, k):
        return BloomAdapter(wc.BloomFilter(num_bits, k, key_bytes=kb, slot_bytes=sb,
                                           cg_size=cg), sb)
    gs.bloom_scenario(F, tag, make)
