"""The CPU oracle reproduces, bit for bit, the outputs the reference's own
CUDA code produced on a B200 (tests/golden/ref_gpu, written by
oracle/ref/make_golden.cu): exact probe positions of every probing scheme,
ReturnBoolean flags, and the per-key statuses, values, sizes and table
Status words of the table scenarios, Bloom filter words and flags."""
import numpy as np
import pytest

from oracle import oracle as o
from tests import golden_scenarios as gs
from tests.golden_io import fixtures

F = fixtures("ref_gpu")


@pytest.mark.parametrize("name,scheme", [("double", o.PROBE_DOUBLE), ("linear", o.PROBE_LINEAR),
                                         ("quadratic", o.PROBE_QUADRATIC)])
def test_probe_positions(name, scheme):
    meta = F["probe_%s_meta" % name].reshape(-1, 6)
    pos = F["probe_%s_pos" % name]
    off = 0
    for kb, cg, cap, key, seed, windows in meta.tolist():
        exp = pos[off:off + windows * cg]
        off += windows * cg
        got = o.probe_sequence(scheme, o.HASH_MURMUR, o.HASH_MURMUR, kb, cg, cap, key, seed,
                               windows * cg, windows).ravel()
        assert np.array_equal(got, exp), (kb, cg, cap, key, seed)
    assert off == pos.size


def test_return_boolean_handler():
    st = F["handler_status_in"]
    for name, ignore in (("none", 0), ("notfound", 1 << 5), ("dup_notfound", (1 << 4) | (1 << 5))):
        exp = F["handler_bool_ignore_" + name]
        got = np.array([o.status_to_bool(int(s), ignore) for s in st], dtype=np.uint8)
        assert np.array_equal(got, exp), name


@pytest.mark.parametrize("tag,kb,vb", gs.SVHT_CASES)
def test_svht(tag, kb, vb):
    gs.svht_scenario(F, tag, kb, lambda cap: o.Table(o.SVHT, kb, vb, cap), vb)


@pytest.mark.parametrize("tag,kb", gs.SET_CASES)
def test_hashset(tag, kb):
    gs.set_scenario(F, tag, kb, lambda cap: o.Table(o.HASHSET, kb, 0, cap, cg=16))


@pytest.mark.parametrize("tag,vb", gs.COUNT_CASES)
def test_counting(tag, vb):
    gs.counting_scenario(F, tag, lambda cap, mx: o.Table(o.COUNTING, 4, vb, cap, cg=4,
                                                         max_count=mx), vb)


@pytest.mark.parametrize("tag", gs.BLOOM_CASES)
def test_bloom(tag):
    def make(kb, sb, cg, num_bits, k):
        return o.Bloom(num_bits, k, key_bytes=kb, slot_bytes=sb, cg=cg)
    gs.bloom_scenario(F, tag, make)


@pytest.mark.parametrize("tag,kb,vb", gs.MV_CASES)
def test_multi_value(tag, kb, vb):
    gs.mv_scenario(F, tag, kb, lambda cap, mx: o.MVTable(kb, vb, cap, max_values_per_key=mx), vb)


@pytest.mark.parametrize("tag,kb,vb", gs.MB_CASES)
def test_multi_bucket(tag, kb, vb):
    gs.mb_scenario(F, tag, kb, vb, lambda cap, bucket, mx: o.MBTable(
        kb, vb, cap, bucket=bucket, max_values_per_key=mx))


@pytest.mark.parametrize("tag,kb,vb", gs.BL_CASES)
def test_bucket_list(tag, kb, vb):
    def make(key_cap, value_cap, grow, min_b, max_b, mx, bits):
        return o.BLTable(kb, vb, key_cap, value_cap, grow_factor=grow, min_bucket_size=min_b,
                         max_bucket_size=max_b, max_values_per_key=mx, bits=bits)
    gs.bl_scenario(F, tag, kb, vb, make)
