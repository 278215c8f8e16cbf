"""The parity suites again, with every table keeping fingerprints.

Fingerprints (one byte per slot) change what the bulk kernels read per
bucket, not the answers.  By default only tables larger than L2 keep them,
so the parity tests' small tables run the whole-window kernels.  This module
re-collects the golden, table, batch and host-buffer tests with the policy
set to "always": with every operation on the fingerprint kernel (the
default), the same with claims preloaded, and with only retrieve and erase
on it (inserts probe whole windows and write fingerprints).  So the fingerprint kernel,
and the fingerprint writes of the window kernels, the batch kernel and the
count-cache flush, are checked against the same oracle and fixtures.  The C++ drop-in program (the
device per-key API) runs once more with the policy taken from the
environment."""
import os
import subprocess

import numpy as np
import pytest

import warpcore_b200 as wc
from oracle import oracle as o
from tests.test_golden_gpu import *  # noqa: F401,F403  (re-collected below)
from tests.test_tables_gpu import *  # noqa: F401,F403
from tests.test_batch_gpu import (test_batch_many_tables_matches_oracle,  # noqa: F401
                                  test_batch_graph_reuse_many_runs)
from tests.test_host_pipe_gpu import test_svht_host_roundtrip, test_hashset_and_counting_host  # noqa: F401
from tests.wc_helpers import dev, empty_dev, host

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=[0b01111, 0b11111, 0b01100],
                ids=["fp-all-ops", "fp-all-ops-preload", "fp-read-ops"])
def _fingerprints_always(request):
    # every table keeps fingerprints; every operation reads them first (the
    # default), with claims preloaded, or only retrieve and erase do
    prev = wc.set_fingerprint_policy("always")
    prev_ops = wc.set_fingerprint_ops(request.param)
    yield
    wc.set_fingerprint_ops(prev_ops)
    wc.set_fingerprint_policy(prev)


def test_policy_modes():
    t = wc.SingleValueHashTable(1000, key_bytes=8)
    assert t.has_fingerprints
    wc.set_fingerprint_policy("never")
    assert not wc.SingleValueHashTable(1000, key_bytes=8).has_fingerprints
    wc.set_fingerprint_policy("auto")
    assert not wc.SingleValueHashTable(1000, key_bytes=8).has_fingerprints
    l2 = __import__("torch").cuda.get_device_properties(0).L2_cache_size
    big = wc.SingleValueHashTable(l2 // 16 + (1 << 20), key_bytes=8)
    assert big.has_fingerprints
    with pytest.raises(wc.WarpcoreError):
        wc.set_fingerprint_policy(7)


@pytest.mark.parametrize("kb", [4, 8])
def test_erase_then_reinsert_with_fingerprints(kb):
    # tombstones keep their fingerprint (1): probing passes them, inserts
    # never reuse them, and erased keys are not found
    n = 30000
    keys = o.gen_unique_keys(kb, 2 * n, 81)
    vals = o.gen_uniform(kb, 2 * n, 82)
    g = wc.SingleValueHashTable(int(1.5 * n / 0.9), key_bytes=kb)
    r = o.Table(o.SVHT, kb, kb, int(1.5 * n / 0.9))
    g.insert(dev(keys[:n]), dev(vals[:n]))
    r.insert(keys[:n], vals[:n])
    st = empty_dev(n // 2, 4)
    g.erase(dev(keys[: n // 2]), status_out=st)
    r_st = r.erase(keys[: n // 2], want_status=True)
    assert np.array_equal(host(st), r_st)
    g.insert(dev(keys[n: n + n // 2]), dev(vals[n: n + n // 2]))
    r.insert(keys[n: n + n // 2], vals[n: n + n // 2])
    q = keys[: 2 * n]
    out = empty_dev(q.size, kb, fill=7)
    st = empty_dev(q.size, 4)
    g.retrieve(dev(q), out, status_out=st)
    r_out, r_st = r.retrieve(q, np.full(q.size, 7, dtype=q.dtype), want_status=True)
    assert np.array_equal(host(out), r_out)
    assert np.array_equal(host(st), r_st)
    assert g.size() == r.size()


def test_cpp_dropin_program_with_fingerprints():
    from tests.cpp import build_dropin
    exe = build_dropin.build()
    env = dict(os.environ, WARPCORE_B200_FINGERPRINTS="always")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin ok" in r.stdout


@pytest.mark.parametrize("kb", [4, 8])
def test_near_duplicates_inserted_once(kb):
    # every key twice, 40 positions apart: the second copy reaches its lane
    # while the first one's claim is in flight in the same warp; it must
    # see that claim (duplicate_key) and not take a second slot
    n = 200_000
    cap = 4 * n
    t = wc.SingleValueHashTable(cap, key_bytes=kb)
    ref = o.Table(o.SVHT, kb, kb, cap)
    keys = o.gen_unique_keys(kb, n, 1201 + kb)
    vals = o.gen_uniform(kb, n, 1202)
    blk = 40
    m = n // blk * blk
    kk = keys[:m].reshape(-1, blk)
    vv = vals[:m].reshape(-1, blk)
    bk = np.concatenate([kk, kk], axis=1).ravel()
    bv = np.concatenate([vv, vv], axis=1).ravel()
    st = empty_dev(len(bk), 4)
    t.insert(dev(bk), dev(bv), status_out=st)
    want = ref.insert(bk, bv, want_status=True)
    got = host(st)
    a, b = np.lexsort((got, bk)), np.lexsort((want, bk))
    assert np.array_equal(got[a], want[b])
    assert t.size() == ref.size() == m
    out = empty_dev(m, kb)
    t.retrieve(dev(keys[:m]), out)
    assert np.array_equal(host(out), vals[:m])


@pytest.mark.parametrize("kind", ["svht32", "set32", "svht64"])
def test_large_insert_rebuilds_fingerprints(kind):
    # a table whose fingerprints exceed half of L2 and a batch above 1/8 of
    # it: inserted by the whole-window kernel, fingerprints rebuilt in one
    # pass, then read by the fingerprint kernel; checked by properties
    import torch
    from warpcore_b200 import datagen
    kb = 8 if kind == "svht64" else 4
    l2 = torch.cuda.get_device_properties(0).L2_cache_size
    cap = l2 // 2 + (16 << 20)           # slots
    n = cap // 4                         # > cap / 8
    if kind == "set32":
        t = wc.HashSet(cap, key_bytes=4)
    else:
        t = wc.SingleValueHashTable(cap, key_bytes=kb)
    assert t.has_fingerprints
    keys = datagen.unique_keys(kb, 0, 2 * n, 91)
    ins, absent = keys[:n].contiguous(), keys[n:].contiguous()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(92)
    if kind == "set32":
        t.insert(ins)
        flags = torch.zeros(2 * n, dtype=torch.uint8, device="cuda")
        t.retrieve(keys, flags)
        assert bool(flags[:n].all()) and not bool(flags[n:].any())
    else:
        vals = datagen.uniform_values(n, kb, gen)
        t.insert(ins, vals)
        out = torch.full((2 * n,), -1, dtype=vals.dtype, device="cuda")
        st = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
        t.retrieve(keys, out, status_out=st)
        assert torch.equal(out[:n], vals)
        assert bool((out[n:] == -1).all())
        assert bool((st[:n] == 0).all())
        assert bool((st[n:] == (1 << 5)).all())
        t.erase(ins[: n // 2])
        st.zero_()
        out.fill_(-1)
        t.retrieve(ins, out[:n], status_out=st[:n])
        assert bool((st[: n // 2] == (1 << 5)).all())
        assert torch.equal(out[n // 2: n], vals[n // 2:])
    assert t.size() == (n if kind == "set32" else n - n // 2)
