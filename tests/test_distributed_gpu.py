"""The CUDA partition kernel against the owner function restated in numpy,
and the sharded table's full NCCL path in a one-rank process group (this run
has one GPU; the multi-rank exchange is covered by the gloo tests)."""
import os
import socket

import numpy as np
import pytest
import torch

import warpcore_b200 as wc
from oracle import oracle as o
from tests.partition_ref import owner_np
from tests.wc_helpers import dev, host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("parts", [1, 2, 7, 8, 64, 1024])
def test_partition_kernel(kb, parts):
    from warpcore_b200.distributed import gpu_partition
    n = 100003
    keys = o.gen_unique_keys(kb, n, 17)
    vals = o.gen_uniform(kb, n, 18)
    salt = 0x1234567890ABCDEF
    ko, vo, perm, counts = gpu_partition(dev(keys), dev(vals), parts, salt, kb)
    own = owner_np(keys, salt, parts).astype(np.int64)
    assert counts == np.bincount(own, minlength=parts).tolist()
    p = host(perm).astype(np.int64)
    assert np.array_equal(np.sort(p), np.arange(n))
    assert np.array_equal(host(ko), keys[p])
    assert np.array_equal(host(vo), vals[p])
    # grouped by owner, in owner order
    assert np.all(np.diff(own[p]) >= 0)


@pytest.mark.parametrize("kb", [4, 8])
def test_partition_repeated_key_nonzero_owner(kb):
    # every key equal: all of them belong to one owner that is not 0
    salt = 0x1234567890ABCDEF
    parts = 7
    key = next(x for x in range(1, 1000) if owner_np(np.array([x], dtype=np.uint64), salt, parts)[0] != 0)
    n = 70001
    keys = np.full(n, key, dtype=np.uint32 if kb == 4 else np.uint64)
    from warpcore_b200.distributed import gpu_partition
    ko, vo, perm, counts = gpu_partition(dev(keys), None, parts, salt, kb)
    want = [0] * parts
    want[int(owner_np(keys[:1], salt, parts)[0])] = n
    assert counts == want
    assert vo is None
    assert np.array_equal(np.sort(host(perm).astype(np.int64)), np.arange(n))


@pytest.mark.parametrize("n", [0, 1, 31, 257])
def test_partition_small_and_empty(n):
    from warpcore_b200.distributed import gpu_partition
    salt = 0x5555
    keys = o.gen_unique_keys(8, max(n, 1), 3)[:n]
    ko, vo, perm, counts = gpu_partition(dev(keys), None, 5, salt, 8)
    own = owner_np(keys, salt, 5).astype(np.int64)
    assert counts == np.bincount(own, minlength=5).tolist()
    if n:
        p = host(perm).astype(np.int64)
        assert np.array_equal(host(ko), keys[p])
        assert np.all(np.diff(own[p]) >= 0)


def test_sharded_table_one_rank_nccl():
    import torch.distributed as dist
    from warpcore_b200.distributed import DistributedSingleValueHashTable
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, device_id=torch.device("cuda", 0))
    try:
        n = 50000
        allk = o.gen_unique_keys(8, n + 5000, 21)
        vals = o.gen_uniform(8, n, 22)
        t = DistributedSingleValueHashTable(2 * n, key_bytes=8)
        t.insert(dev(allk[:n]), dev(vals))
        assert t.size() == n
        q = np.concatenate([allk[:n][::3], allk[n:]])
        out = torch.full((q.size,), -1, dtype=torch.int64, device="cuda")
        st = torch.zeros(q.size, dtype=torch.int32, device="cuda")
        t.retrieve(dev(q), out, st)
        ref = o.Table(o.SVHT, 8, 8, 2 * n)
        ref.insert(allk[:n], vals)
        r_out, r_st = ref.retrieve(q, np.full(q.size, 2**64 - 1, dtype=np.uint64), want_status=True)
        assert np.array_equal(host(out), r_out)
        assert np.array_equal(host(st), r_st)
        t.erase(dev(allk[:n][::2]))
        assert t.size() == n - allk[:n][::2].size
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("vb", [4, 8])
def test_partition_restore(vb):
    from warpcore_b200.distributed import gpu_restore
    n = 50021
    rng = np.random.default_rng(7)
    perm = rng.permutation(n).astype(np.int64)
    vals = o.gen_uniform(vb, n, 71)
    status = np.where(rng.random(n) < 0.6, 0, 32).astype(np.uint32)  # 0 = hit, 32 = key_not_found
    init = o.gen_uniform(vb, n, 72)
    out = dev(init)
    st_out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    gpu_restore(dev(vals), dev(status), torch.from_numpy(perm).cuda(), out, st_out)
    want = init.copy()
    hit = status == 0
    want[perm[hit]] = vals[hit]
    want_st = np.empty(n, dtype=np.uint32)
    want_st[perm] = status
    assert np.array_equal(host(out), want)
    assert np.array_equal(host(st_out), want_st)
