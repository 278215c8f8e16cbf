"""The CPU oracle pinned against golden vectors produced by the reference's
own host code (oracle/ref/make_golden.cu, `host` mode): hashers, the
capacity rule with its prime table, the Status algebra and the Bloom filter's
analytic false-positive rate.  Also restates the reference's cycle-free
probing test (tests/src/probing_schemes_test.cu:62-68) on the oracle."""
import math

import numpy as np
import pytest

from oracle import oracle as o
from tests.golden_io import fixtures

F = fixtures("ref_host")


def test_murmur32():
    xs = F["hash_inputs"]
    got = [o.hash_(o.HASH_MURMUR, 4, int(x) & 0xFFFFFFFF) for x in xs]
    assert got == F["hash_murmur32"].tolist()


def test_murmur64():
    xs = F["hash_inputs"]
    got = [o.hash_(o.HASH_MURMUR, 8, int(x)) for x in xs]
    assert got == F["hash_murmur64"].tolist()


def test_nvidia_mueller():
    xs = F["hash_inputs"]
    assert [o.hash_(o.HASH_NVIDIA, 4, int(x) & 0xFFFFFFFF) for x in xs] == F["hash_nvidia32"].tolist()
    assert [o.hash_(o.HASH_MUELLER, 4, int(x) & 0xFFFFFFFF) for x in xs] == F["hash_mueller32"].tolist()


def test_capacity_rule():
    ci = F["capacity_in"].reshape(-1, 2)
    co = F["capacity_out"]
    got = [o.valid_capacity(int(m), int(c)) for m, c in ci]
    assert got == co.tolist()


def test_prime_table_digest():
    p = o.primes()
    d = F["primes_digest"].tolist()
    x = 0
    for v in p.tolist():
        x ^= (v * 0x9E3779B97F4A7C15) & (2**64 - 1)
    assert [len(p), int(p[0]), int(p[-1]), int(p.sum(dtype=np.uint64)), x] == d


def test_status_algebra():
    from warpcore_b200 import Status
    st = F["status_algebra"].tolist()
    assert Status.error_mask().base() == st[0]
    assert Status.warning_mask().base() == st[1]
    pairs = st[2:-1]
    for b in range(13):
        assert pairs[2 * b] == 1 << b
        assert (~Status(1 << b)).base() == pairs[2 * b + 1]
    assert (~Status.none()).base() == st[-1]


def test_status_to_bool_matches_algebra():
    st = F["status_algebra"].tolist()
    pairs = st[2:-1]
    for b in range(13):
        inv = pairs[2 * b + 1]
        for s in range(13):
            assert o.status_to_bool(1 << s, 1 << b) == bool((1 << s) & inv)


def test_bloom_fpr():
    fi = F["bloom_fpr_in"].reshape(-1, 3)
    fo = F["bloom_fpr_out_f64bits"].view(np.float64)
    cgs = [8, 8, 1]
    for (nb, k, n), ref, cg in zip(fi, fo, cgs):
        b = o.Bloom(int(nb), int(k), cg=cg)
        got = b.fpr(int(n))
        if math.isnan(ref):
            assert math.isnan(got)
        else:
            assert got == pytest.approx(float(ref), rel=1e-12, abs=0.0)


@pytest.mark.parametrize("scheme", [o.PROBE_DOUBLE, o.PROBE_LINEAR])
@pytest.mark.parametrize("cg", [1, 2, 4, 8, 16, 32])
def test_probing_cycle_free(scheme, cg):
    """probing_schemes_test.cu:36-68: all capacity positions are distinct."""
    # the reference's grid of capacities, keys and seeds, thinned so the
    # whole sweep stays a few seconds on the CPU
    for min_cap in ((12345, 42424, 6969) if cg <= 4 else (6969,)):
        cap = o.valid_capacity(min_cap, cg)
        for key in ((1, 42, 69, 1337) if cg <= 4 else (1, 1337)):
            for seed in (5, 42):
                pos = o.probe_sequence(scheme, o.HASH_MURMUR, o.HASH_MURMUR, 4, cg, cap,
                                       key, seed, cap, cap // cg).ravel()
                assert pos.size == cap
                assert np.unique(pos).size == cap
