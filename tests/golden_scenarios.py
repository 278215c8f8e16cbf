"""Replays the scenarios of oracle/ref/make_golden.cu (which ran the
reference's CUDA code on a B200 and recorded its outputs in
tests/golden/ref_gpu) on any implementation with the oracle's interface, and
compares every output with the recorded one."""
import numpy as np

from oracle import oracle as o

SENT64 = 0xA5A5A5A5A5A5A5A5


def _dt(kb):
    return np.uint32 if kb == 4 else np.uint64


def svht_scenario(F, tag, kb, make_table, vb=None):
    """make_table(min_cap) -> object with insert/retrieve/erase/size/
    pop_status like oracle.Table; vb = value width (default: kb)"""
    vb = kb if vb is None else vb
    n, min_cap, kseed, cap, size1, size2, size3, s1, s2, s3, s4, s5 = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(kb, 2 * n, kseed)
    keys = allk[:n]
    vals = o.gen_uniform(vb, n, kseed + 1)
    nd = n // 8
    km = (1 << (8 * kb)) - 1
    vm = (1 << (8 * vb)) - 1
    k2 = np.concatenate([keys[:nd], np.array([0, km], dtype=_dt(kb))])
    v2 = np.concatenate([o.gen_uniform(vb, nd, kseed + 2), np.array([1, 2], dtype=_dt(vb))])
    q = np.empty(2 * n, dtype=_dt(kb))
    q[0::2] = keys
    q[1::2] = allk[n:]
    er = np.concatenate([keys[::5], allk[n:n + 16]])
    fill = np.full(2 * n, SENT64 & vm, dtype=_dt(vb))

    t = make_table(min_cap)
    assert t.capacity == cap
    assert np.array_equal(t.insert(keys, vals, want_status=True), F[tag + "_insert_status"])
    assert t.size() == size1
    assert t.pop_status() == s1
    assert np.array_equal(t.insert(k2, v2, want_status=True), F[tag + "_insert2_status"])
    assert t.size() == size2
    assert t.pop_status() == s2
    out, st = t.retrieve(q, fill.copy(), want_status=True)
    assert np.array_equal(out, F[tag + "_retrieve1_values"])
    assert np.array_equal(st, F[tag + "_retrieve1_status"])
    assert t.pop_status() == s3
    assert np.array_equal(t.erase(er, want_status=True), F[tag + "_erase_status"])
    assert t.size() == size3
    assert t.pop_status() == s4
    out, st = t.retrieve(q, fill.copy(), want_status=True)
    assert np.array_equal(out, F[tag + "_retrieve2_values"])
    assert np.array_equal(st, F[tag + "_retrieve2_status"])
    assert t.pop_status() == s5


def set_scenario(F, tag, kb, make_set):
    n, min_cap, kseed, cap, size1, size3, s1, s2, s3 = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(kb, 2 * n, kseed)
    keys = allk[:n]
    k2 = np.concatenate([keys[: n // 8], np.array([0], dtype=_dt(kb))])
    q = np.empty(2 * n, dtype=_dt(kb))
    q[0::2] = keys
    q[1::2] = allk[n:]
    er = keys[::5]
    s = make_set(min_cap)
    assert s.capacity == cap
    assert np.array_equal(s.insert(keys, want_status=True), F[tag + "_insert_status"])
    assert s.size() == size1
    assert s.pop_status() == s1
    assert np.array_equal(s.insert(k2, want_status=True), F[tag + "_insert2_status"])
    assert s.pop_status() == s2
    f, st = s.retrieve(q, np.full(2 * n, 7, dtype=np.uint8), want_status=True)
    assert np.array_equal(f, F[tag + "_contains1"])
    assert np.array_equal(st, F[tag + "_contains1_status"])
    assert np.array_equal(s.erase(er, want_status=True), F[tag + "_erase_status"])
    assert s.size() == size3
    f, st = s.retrieve(q, np.full(2 * n, 7, dtype=np.uint8), want_status=True)
    assert np.array_equal(f, F[tag + "_contains2"])
    assert np.array_equal(st, F[tag + "_contains2_status"])
    assert s.pop_status() == s3


def counting_scenario(F, tag, make_counter, vb=4):
    """u32 keys, counts of vb bytes"""
    distinct, occ, min_cap, max_count, kseed, cap, size1, s1 = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(4, distinct + distinct // 4, kseed)
    ranks = o.gen_zipf_ranks(distinct, 1.1, occ, kseed + 3)
    keys = allk[(ranks - 1).astype(np.int64)]
    c = make_counter(min_cap, max_count)
    assert c.capacity == cap
    c.insert(keys)
    assert c.pop_status() == s1
    fill = np.full(allk.size, SENT64 & ((1 << (8 * vb)) - 1), dtype=_dt(vb))
    out, st = c.retrieve(allk, fill, want_status=True)
    assert np.array_equal(out, F[tag + "_counts"])
    assert np.array_equal(st, F[tag + "_status"])
    assert c.size() == size1


def bloom_scenario(F, tag, make_bloom):
    kb, sb, cg, num_bits, k, n, kseed, num_slots, num_blocks = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(kb, 2 * n, kseed)
    b = make_bloom(kb, sb, cg, num_bits, k)
    assert (b.num_slots, b.num_blocks) == (num_slots, num_blocks)
    b.insert(allk[:n])
    assert np.array_equal(b.words(), F[tag + "_words"])
    assert np.array_equal(b.retrieve(allk), F[tag + "_flags"])


SVHT_CASES = [("svht_u32u32", 4, 4), ("svht_u64u64", 8, 8), ("svht_u32u64", 4, 8),
              ("svht_u64u32", 8, 4)]
SET_CASES = [("set_u64", 8), ("set_u32", 4)]
COUNT_CASES = [("count_u32", 4), ("count_u32_max10", 4), ("count_u32u64", 8),
               ("count_u32u64_max10", 8)]
BLOOM_CASES = ["bloom_u64_s64_cg8", "bloom_u64_s64_cg1", "bloom_u32_s32_cg4", "bloom_u32_s64_cg2"]


MV_CASES = [("mv_u32u32_max3", 4, 4), ("mv_u64u64", 8, 8), ("mv_u32u64_max3", 4, 8),
            ("mv_u64u32", 8, 4)]


def mv_scenario(F, tag, kb, make_table, vb=None):
    """make_table(min_cap, max_values_per_key) -> object with insert /
    num_keys / size / pop_status / retrieve(keys, dry_run) /
    unique_keys like oracle.MVTable"""
    (n, min_cap, kseed, cap, max_values, num_keys, size, s1, num_dry, s2, num_out, s3,
     num_unique) = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(kb, n + n // 4, kseed)
    keys = allk[:n]
    t = make_table(min_cap, max_values)
    assert t.capacity == cap
    st_all, vals_all = [], []
    for r in range(5):
        m = n - r * (n // 5)
        v = o.gen_uniform(kb if vb is None else vb, m, kseed + 10 + r)
        st_all.append(t.insert(keys[:m], v, want_status=True))
        vals_all.append(v)
    assert np.array_equal(np.concatenate(st_all), F[tag + "_insert_status"])
    assert np.array_equal(np.concatenate(vals_all), F[tag + "_insert_values"])
    assert t.num_keys() == num_keys
    assert t.size() == size
    assert t.pop_status() == s1
    _, counts, _, st = t.retrieve(allk, dry_run=True)
    assert int(counts.sum()) == num_dry
    assert np.array_equal(counts, F[tag + "_dry_counts"])
    assert np.array_equal(st, F[tag + "_dry_status"])
    assert t.pop_status() == s2
    b, e, v, st = t.retrieve(allk)
    assert np.array_equal(b, F[tag + "_begin"])
    assert np.array_equal(e, F[tag + "_end"])
    assert v.size == num_out
    assert np.array_equal(v, F[tag + "_values"])
    assert np.array_equal(st, F[tag + "_retrieve_status"])
    assert t.pop_status() == s3
    uk = np.sort(t.unique_keys())
    assert uk.size == num_unique
    assert np.array_equal(uk, F[tag + "_unique_keys_sorted"])


MB_CASES = [("mb_u32u32_b1", 4, 4), ("mb_u32u32_b2", 4, 4), ("mb_u32u32_b2_max3", 4, 4),
            ("mb_u32u32_b4_max6", 4, 4), ("mb_u32u32_b8", 4, 4), ("mb_u32u64_b2", 4, 8),
            ("mb_u64u64_b4_max2", 8, 8)]


def mb_scenario(F, tag, kb, vb, make_table):
    """make_table(min_cap, bucket, max_values_per_key) -> object with insert /
    num_keys / num_occupied / size / pop_status / retrieve(keys, dry_run) /
    unique_keys like oracle.MBTable"""
    (n, min_cap, kseed, cap, bucket, max_values, num_keys, num_occupied, size, s1, num_dry, s2,
     num_out, s3, num_unique, value_capacity) = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(kb, n + n // 4, kseed)
    keys = allk[:n]
    t = make_table(min_cap, bucket, max_values)
    assert t.capacity == cap
    assert t.capacity * bucket == value_capacity
    st_all, keys_all, vals_all = [], [], []
    for r in range(5):
        m = n - r * (n // 5)
        k = keys[:m].copy()
        v = o.gen_uniform(vb, m, kseed + 10 + r)
        v[v == 0] = 1
        if r == 0:
            k[11] = (1 << (8 * kb)) - 1      # the tombstone key: invalid_key
            v[7] = 0                         # the empty value: invalid_value
        st_all.append(t.insert(k, v, want_status=True))
        keys_all.append(k)
        vals_all.append(v)
    assert np.array_equal(np.concatenate(keys_all), F[tag + "_insert_keys"])
    assert np.array_equal(np.concatenate(vals_all), F[tag + "_insert_values"])
    assert np.array_equal(np.concatenate(st_all), F[tag + "_insert_status"])
    assert t.num_keys() == num_keys
    assert t.num_occupied() == num_occupied
    assert t.size() == size
    assert t.pop_status() == s1
    _, counts, _, st = t.retrieve(allk, dry_run=True)
    assert int(counts.sum()) == num_dry
    assert np.array_equal(counts, F[tag + "_dry_counts"])
    assert np.array_equal(st, F[tag + "_dry_status"])
    assert t.pop_status() == s2
    b, e, v, st = t.retrieve(allk)
    assert np.array_equal(b, F[tag + "_begin"])
    assert np.array_equal(e, F[tag + "_end"])
    assert v.size == num_out
    assert np.array_equal(v, F[tag + "_values"])
    assert np.array_equal(st, F[tag + "_retrieve_status"])
    assert t.pop_status() == s3
    uk = np.sort(t.unique_keys())
    assert uk.size == num_unique
    assert np.array_equal(uk, F[tag + "_unique_keys_sorted"])


BL_CASES = [("bl_u32u32", 4, 4), ("bl_u32u32_bench_bits_max6", 4, 4),
            ("bl_u32u32_min2_grow15_max4", 4, 4), ("bl_u64u64", 8, 8), ("bl_u32u32_oom", 4, 4)]

UNWRITTEN = 0xFFFFFFFF


def bl_scenario(F, tag, kb, vb, make_table):
    """make_table(key_cap, value_cap, grow, min_b, max_b, max_values, bits) ->
    object with insert(keys, values, want_status, status_fill) /
    num_keys / total_values / next_free / pop_status / retrieve(keys,
    dry_run) / all_keys like oracle.BLTable.  The reference writes no
    status for a key that found no slot (UNWRITTEN in the fixture); there
    the table may leave the fill or report the key's own status."""
    (n, key_cap, value_cap, key_capacity, value_capacity, grow_milli, min_b, max_b, max_values,
     ib, cb, sb, num_keys, num_values, vlf_bits, s1, num_dry, s2, num_out, s3, num_all,
     kseed) = F[tag + "_meta"].tolist()
    allk = o.gen_unique_keys(kb, n + n // 4, kseed)
    keys = allk[:n]
    t = make_table(key_cap, value_cap, grow_milli / 1000.0, min_b, max_b, max_values, (ib, cb, sb))
    assert t.key_capacity == key_capacity
    st_all, keys_all, vals_all = [], [], []
    for r in range(8):
        m = n - r * (n // 8)
        k = keys[:m].copy()
        v = o.gen_uniform(vb, m, kseed + 10 + r)
        if r == 0:
            k[11] = (1 << (8 * kb)) - 1      # the tombstone key: no slot
        st_all.append(t.insert(k, v, want_status=True, status_fill=UNWRITTEN))
        keys_all.append(k)
        vals_all.append(v)
    assert np.array_equal(np.concatenate(keys_all), F[tag + "_insert_keys"])
    assert np.array_equal(np.concatenate(vals_all), F[tag + "_insert_values"])
    got, want = np.concatenate(st_all), F[tag + "_insert_status"]
    written = want != UNWRITTEN
    assert np.array_equal(got[written], want[written])
    assert np.all((got[~written] == UNWRITTEN) | (got[~written] == o.ST_INVALID_KEY))
    assert t.num_keys() == num_keys
    assert t.total_values() == num_values
    vlf = np.float32(t.next_free()) / np.float32(value_capacity)
    assert vlf.view(np.uint32) == vlf_bits
    assert t.pop_status() == s1
    _, counts, _, st = t.retrieve(allk, dry_run=True)
    assert int(counts.sum()) == num_dry
    assert np.array_equal(counts, F[tag + "_dry_counts"])
    assert np.array_equal(st, F[tag + "_dry_status"])
    assert t.pop_status() == s2
    # the output starts all-ones: a list whose pool ran out is not read, so
    # its part keeps the fill here; in the reference run it keeps the fill
    # too, except at the front of the buffer, which the reference lends to
    # its offset scan as temporary storage (bucket_list_hash_table.cuh:437-443)
    fill = (1 << (8 * vb)) - 1
    b, e, v, st = t.retrieve(allk, fill=fill)
    assert np.array_equal(b, F[tag + "_begin"])
    assert np.array_equal(e, F[tag + "_end"])
    assert v.size == num_out
    gv = F[tag + "_values"]
    read = v != fill
    assert np.array_equal(v[read], gv[read])
    assert np.all((gv[~read] == fill) | (np.nonzero(~read)[0] * vb < 4096))
    assert np.array_equal(st, F[tag + "_retrieve_status"])
    assert t.pop_status() == s3
    ak = np.sort(t.all_keys())
    assert ak.size == num_all
    assert np.array_equal(ak, F[tag + "_all_keys_sorted"])
