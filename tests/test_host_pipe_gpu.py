"""Bulk calls on host buffers through a HostPipe (chunked, with copies
overlapping kernels) against the oracle: every table kind, ragged chunks,
both miss policies of retrieve, pinned and pageable buffers."""
import numpy as np
import pytest
import torch

import warpcore_b200 as wc
from oracle import oracle as o

pytestmark = pytest.mark.gpu

_S = {4: np.int32, 8: np.int64}
_U = {4: np.uint32, 8: np.uint64}


def cpu(a, pinned=True):
    t = torch.from_numpy(np.ascontiguousarray(a).view(_S[a.itemsize]) if a.itemsize in _S else a)
    return t.pin_memory() if pinned else t.clone()


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("chunk,depth", [(1000, 2), (4096, 3), (1 << 22, 3)])
@pytest.mark.parametrize("pinned", [True, False])
def test_svht_host_roundtrip(kb, chunk, depth, pinned):
    n = 30011
    keys = o.gen_unique_keys(kb, n + 7000, 51)
    vals = o.gen_uniform(kb, n, 52)
    q = np.concatenate([keys[:n:3], keys[n:]])
    pipe = wc.HostPipe(chunk, depth)
    t = wc.SingleValueHashTable(int(n / 0.9), key_bytes=kb)
    s = torch.cuda.current_stream()
    t.insert_from_host(pipe, cpu(keys[:n], pinned), cpu(vals, pinned))
    # misses keep the output's content
    init = o.gen_uniform(kb, q.size, 53)
    out = cpu(init, pinned)
    t.retrieve_to_host(pipe, cpu(q, pinned), out)
    s.synchronize()
    ref = o.Table(o.SVHT, kb, kb, int(n / 0.9))
    ref.insert(keys[:n], vals)
    r_out, _ = ref.retrieve(q, init.copy(), want_status=True)
    assert np.array_equal(out.numpy().view(_U[kb]), r_out)
    # misses get miss_fill
    out2 = cpu(np.zeros(q.size, dtype=_U[kb]), pinned)
    t.retrieve_to_host(pipe, cpu(q, pinned), out2, miss_fill=-1)
    s.synchronize()
    r2, _ = ref.retrieve(q, np.full(q.size, (1 << (8 * kb)) - 1, dtype=_U[kb]), want_status=True)
    assert np.array_equal(out2.numpy().view(_U[kb]), r2)
    assert t.size() == n


def test_hashset_and_counting_host():
    n = 20000
    keys = o.gen_unique_keys(8, n + 5000, 61)
    pipe = wc.HostPipe(3000, 2)
    hs = wc.HashSet(int(n / 0.8), key_bytes=8)
    hs.insert_from_host(pipe, cpu(keys[:n]))
    flags = torch.zeros(keys.size, dtype=torch.uint8).pin_memory()
    hs.retrieve_to_host(pipe, cpu(keys), flags)
    torch.cuda.current_stream().synchronize()
    assert flags.numpy()[:n].all() and not flags.numpy()[n:].any()

    distinct = o.gen_unique_keys(4, 3000, 62)
    ranks = o.gen_zipf_ranks(3000, 1.1, 50000, 63)
    stream = distinct[ranks]
    c = wc.CountingHashTable(4000, key_bytes=4)
    c.insert_from_host(pipe, cpu(stream))
    absent = o.gen_unique_keys(4, 3500, 62)[3000:]
    qk = np.concatenate([distinct, absent])
    counts = cpu(np.zeros(qk.size, dtype=np.uint32))
    c.retrieve_to_host(pipe, cpu(qk), counts)
    torch.cuda.current_stream().synchronize()
    want = np.bincount(ranks.astype(np.int64), minlength=3000).astype(np.uint32)
    got = counts.numpy().view(np.uint32)
    assert np.array_equal(got[:3000], want)
    assert not got[3000:].any()


def test_empty_and_device_buffers_rejected():
    pipe = wc.HostPipe(1024, 2)
    t = wc.SingleValueHashTable(1000, key_bytes=4)
    empty = torch.empty(0, dtype=torch.int32)
    t.insert_from_host(pipe, empty, empty)
    with pytest.raises(wc.WarpcoreError):
        t.insert_from_host(pipe, torch.zeros(4, dtype=torch.int32, device="cuda"),
                           torch.zeros(4, dtype=torch.int32, device="cuda"))
