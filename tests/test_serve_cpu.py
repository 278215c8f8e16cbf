"""Host logic of the served workload (no GPU): the generator keeps keys
unique per table, fills no table beyond its load target, draws hits only
from keys inserted by earlier requests of the same table, and admission
respects the device-memory budget."""
import numpy as np

from warpcore_b200 import OP_INSERT, OP_RETRIEVE
from warpcore_b200.serve import ServedWorkload


def small(**kw):
    args = dict(num_tables=64, cap_lo=1 << 8, cap_hi=1 << 14, num_requests=600,
                batch_lo=1 << 4, batch_hi=1 << 10, rate=1e5, seed=3, device="cpu")
    args.update(kw)
    return ServedWorkload(**args)


def test_arrivals_sorted_and_ops_mixed():
    w = small()
    assert np.all(np.diff(w.arrival_us) >= 0)
    frac = np.mean(w.op == OP_INSERT)
    assert 0.05 < frac < 0.45
    assert np.all(w.num >= 1)


def test_keys_unique_per_table_and_budget_respected():
    w = small()
    keys = w.keys.numpy().view(np.uint32)
    ins = np.repeat(w.op == OP_INSERT, w.num)
    tab = np.repeat(w.table, w.num)
    for t in np.unique(w.table):
        k = keys[ins & (tab == t)]
        assert np.unique(k).size == k.size
        assert k.size <= w.budget[t]
    assert not np.any((keys == 0) | (keys == 0xFFFFFFFF))


def test_hits_come_from_earlier_inserts_of_the_same_table():
    w = small()
    keys = w.keys.numpy().view(np.uint32)
    hit = w.is_hit.numpy()
    seen = {}
    for r in range(len(w.num)):
        a, b = w.offsets[r], w.offsets[r + 1]
        t = w.table[r]
        s = seen.setdefault(t, set())
        if w.op[r] == OP_INSERT:
            s.update(keys[a:b].tolist())
        else:
            for k, h in zip(keys[a:b].tolist(), hit[a:b].tolist()):
                assert (k in s) == h


def test_admission_respects_budget():
    w = small(budget_bytes=40 << 20)
    plan, used = w.admission_plan()
    assert used <= 40 << 20
    assert 0 < plan.sum() < w.num_tables
    # admitted in table order: a prefix-closed greedy plan
    w2 = small(budget_bytes=1 << 40)
    plan2, _ = w2.admission_plan()
    assert plan2.all()
