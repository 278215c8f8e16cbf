"""MultiValueHashTable through the C ABI against the reference's own outputs
(tests/golden/ref_gpu, mv_* fixtures) and the oracle: insert statuses with
max_values_per_key, per-key counts, offsets, every key's values in
insertion order, dry runs, unique keys, sizes and table statuses."""
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


class GpuMV:
    """the oracle.MVTable interface over wc.MultiValueHashTable"""

    def __init__(self, kb, cap, max_values, vb=None, **kw):
        self.kb = kb
        self.vb = kb if vb is None else vb
        self.t = wc.MultiValueHashTable(cap, key_bytes=kb, value_bytes=self.vb,
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


@pytest.mark.parametrize("tag,kb,vb", gs.MV_CASES)
def test_multi_value_golden(tag, kb, vb):
    gs.mv_scenario(F, tag, kb, lambda cap, mx: GpuMV(kb, cap, mx, vb=vb), vb)


@pytest.mark.parametrize("kb,vb", [(4, 4), (8, 8), (4, 8), (8, 4)])
@pytest.mark.parametrize("cg", [1, 4, 8, 16, 32])
def test_multi_value_vs_oracle(kb, vb, cg):
    # rounds of unique keys: values per key in insertion order; then a
    # round that mixes new keys with held ones
    n = 3000
    keys = o.gen_unique_keys(kb, n + 500, 101 + cg)
    g = GpuMV(kb, 4 * n, 4, vb=vb, cg_size=cg)
    r = o.MVTable(kb, vb, 4 * n, cg=cg, max_values_per_key=4)
    assert g.capacity == r.capacity
    for rnd in range(6):
        m = n - rnd * 400
        v = o.gen_uniform(vb, m, 200 + rnd)
        assert np.array_equal(g.insert(keys[:m], v, want_status=True),
                              r.insert(keys[:m], v, want_status=True)), rnd
    assert g.num_keys() == r.num_keys()
    assert g.size() == r.size()
    q = np.concatenate([keys, keys[:100]])
    gb, ge, gv, gs_ = g.retrieve(q)
    rb, re, rv, rs = r.retrieve(q)
    assert np.array_equal(gb, rb) and np.array_equal(ge, re)
    assert np.array_equal(gv, rv)
    assert np.array_equal(gs_, rs)
    assert g.pop_status() == r.pop_status()
    assert np.array_equal(np.sort(g.unique_keys()), np.sort(r.unique_keys()))


def test_multi_value_in_batch_duplicates():
    # one batch holding a key several times: every copy is stored (as many
    # as max_values_per_key allows); which copies is schedule-dependent
    kb = 8
    keys = o.gen_unique_keys(kb, 1000, 7)
    rep = np.repeat(keys[:200], 5)
    vals = np.arange(1, rep.size + 1, dtype=np.uint64)
    g = GpuMV(kb, 8000, 3)
    st = g.insert(rep, vals, want_status=True)
    _, e, v, s = g.retrieve(keys[:200])
    assert np.all(e == 3 * np.arange(1, 201))
    for i in range(200):
        got = set(v[3 * i: 3 * i + 3].tolist())
        assert got <= set(vals[5 * i: 5 * i + 5].tolist())
    assert int(((st & o.ST_MAX_VALUES_REACHED) != 0).sum()) == 400
    assert g.size() == 600
