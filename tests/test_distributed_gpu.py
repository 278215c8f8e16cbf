"""The CUDA partition kernels against the owner functions restated in numpy,
the Bloom filter's block-range shards against the one whole filter, and the
sharded containers' full NCCL path in a one-rank process group (this run has
one GPU; the multi-rank exchange is covered by the gloo tests)."""
import os
import socket

import numpy as np
import pytest
import torch

import warpcore_b200 as wc
from oracle import oracle as o
from tests.partition_ref import bloom_block_np, bloom_owner_np, bloom_shard_range, owner_np
from tests.wc_helpers import copy_device_words, dev, host

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


@pytest.mark.parametrize("vb", [1, 4, 8])
def test_partition_restore_without_status(vb):
    from warpcore_b200.distributed import gpu_restore
    n = 30011
    rng = np.random.default_rng(8)
    perm = rng.permutation(n).astype(np.int64)
    if vb == 1:
        vals = rng.integers(0, 2, n).astype(np.uint8)
        out = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        gpu_restore(torch.from_numpy(vals).cuda(), None, torch.from_numpy(perm).cuda(), out)
    else:
        vals = o.gen_uniform(vb, n, 81)
        out = dev(o.gen_uniform(vb, n, 82))
        gpu_restore(dev(vals), None, torch.from_numpy(perm).cuda(), out)
    want = np.empty_like(vals)
    want[perm] = vals
    assert np.array_equal(host(out) if vb > 1 else out.cpu().numpy(), want)


def _bloom_cfgs():
    # (key_bytes, slot_bytes, cg): blocks of 4 to 128 bytes
    return [(8, 8, 1), (4, 4, 1), (8, 8, 4), (4, 4, 8), (8, 8, 16), (4, 4, 32), (8, 4, 2)]


@pytest.mark.parametrize("cfg", _bloom_cfgs())
@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_bloom_partition_kernel(cfg, parts):
    kb, sb, cg = cfg
    bits = 64 * 8 * 1021 * 8  # whole blocks for every configuration here
    f = wc.BloomFilter(bits, 6, seed=0x77, key_bytes=kb, slot_bytes=sb, cg_size=cg)
    n = 70001
    keys = o.gen_unique_keys(kb, n, 31)
    ko, perm, counts = f.partition(dev(keys), parts)
    nb = f.num_blocks()
    own = bloom_owner_np(keys, 0x77, nb, parts)
    assert counts == np.bincount(own, minlength=parts).tolist()
    p = host(perm).astype(np.int64)
    assert np.array_equal(np.sort(p), np.arange(n))
    assert np.array_equal(host(ko), keys[p])
    assert np.all(np.diff(own[p]) >= 0)


@pytest.mark.parametrize("cfg", _bloom_cfgs())
@pytest.mark.parametrize("parts", [2, 3, 5])
def test_bloom_shards_are_slices_of_one_filter(cfg, parts):
    """each shard, given every key, holds exactly the whole filter's words of
    its block range, and its flags are the whole filter's for the keys of
    its blocks and 0 for the others"""
    kb, sb, cg = cfg
    bits = sb * 8 * cg * 4099
    k, seed = 5, 0x99
    whole = wc.BloomFilter(bits, k, seed=seed, key_bytes=kb, slot_bytes=sb, cg_size=cg)
    n = 20000
    keys = o.gen_unique_keys(kb, 2 * n, 41)
    whole.insert(dev(keys[:n]))
    words = copy_device_words(whole.words_ptr(), whole.num_slots(), sb)
    # the oracle's filter pins the whole one
    ref = o.Bloom(bits, k, seed=seed, key_bytes=kb, slot_bytes=sb, cg=cg)
    ref.insert(keys[:n])
    assert np.array_equal(words, ref.words())
    want_flags = ref.retrieve(keys)
    nb = whole.num_blocks()
    blk = bloom_block_np(keys, seed, nb).astype(np.int64)
    covered = 0
    for s in range(parts):
        sh = wc.BloomFilter(bits, k, seed=seed, key_bytes=kb, slot_bytes=sb, cg_size=cg,
                            shard=s, num_shards=parts)
        lo, hi = bloom_shard_range(nb, s, parts)
        assert sh.block_range() == (lo, hi - lo)
        covered += hi - lo
        sh.insert(dev(keys[:n]))
        got = copy_device_words(sh.words_ptr(), (hi - lo) * cg, sb)
        assert np.array_equal(got, words[lo * cg:hi * cg])
        fl = torch.full((2 * n,), 9, dtype=torch.uint8, device="cuda")
        sh.retrieve(dev(keys), fl)
        mine = (blk >= lo) & (blk < hi)
        assert np.array_equal(fl.cpu().numpy(), np.where(mine, want_flags, 0))
    assert covered == nb


def test_bloom_shard_errors():
    # blocks above 128 bytes, and a ragged last block, are not sharded
    with pytest.raises(wc.WarpcoreError):
        wc.BloomFilter(64 * 32 * 100, 4, key_bytes=8, slot_bytes=8, cg_size=32, shard=0, num_shards=2)
    with pytest.raises(wc.WarpcoreError):
        wc.BloomFilter(64 * 4 * 100 + 64, 4, key_bytes=8, slot_bytes=8, cg_size=4, shard=0, num_shards=2)
    with pytest.raises(wc.WarpcoreError):
        wc.BloomFilter(64 * 4 * 100, 4, key_bytes=8, slot_bytes=8, cg_size=4, shard=2, num_shards=2)
    # more shards than blocks: the extra shards hold none and answer 0
    sh = wc.BloomFilter(64 * 4 * 3, 4, key_bytes=8, slot_bytes=8, cg_size=4, shard=4, num_shards=8)
    assert sh.block_range()[1] == 0
    keys = o.gen_unique_keys(8, 1000, 5)
    sh.insert(dev(keys))
    fl = torch.full((1000,), 9, dtype=torch.uint8, device="cuda")
    sh.retrieve(dev(keys), fl)
    assert int(fl.sum()) == 0


def _one_rank_group():
    import torch.distributed as dist
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, device_id=torch.device("cuda", 0))
    return dist


def test_sharded_set_counting_bloom_one_rank_nccl():
    from warpcore_b200.distributed import (DistributedBloomFilter, DistributedCountingHashTable,
                                           DistributedHashSet)
    dist = _one_rank_group()
    try:
        n = 40000
        allk = o.gen_unique_keys(4, n + 4000, 51)
        ins = np.concatenate([allk[:n], allk[:500]])
        q = np.concatenate([allk[:n][::5], allk[n:]])
        hs = DistributedHashSet(2 * n, key_bytes=4)
        hs.insert(dev(ins))
        assert hs.size() == n
        flags = torch.full((q.size,), 9, dtype=torch.uint8, device="cuda")
        st = torch.zeros(q.size, dtype=torch.int32, device="cuda")
        hs.retrieve(dev(q), flags, st)
        rs = o.Table(o.HASHSET, 4, 0, 2 * n)
        rs.insert(ins)
        r_f, r_st = rs.retrieve(q, np.full(q.size, 9, dtype=np.uint8), want_status=True)
        assert np.array_equal(flags.cpu().numpy(), r_f)
        assert np.array_equal(host(st), r_st)
        ct = DistributedCountingHashTable(2 * n, key_bytes=4)
        ct.insert(dev(ins))
        cnt = torch.full((q.size,), 7, dtype=torch.int32, device="cuda")
        ct.retrieve(dev(q), cnt)
        rc = o.Table(o.COUNTING, 4, 4, 2 * n)
        rc.insert(ins)
        assert np.array_equal(host(cnt), rc.retrieve(q, np.full(q.size, 7, dtype=np.uint32)))
        bits = 64 * 4 * 8192
        bf = DistributedBloomFilter(bits, 6, seed=3, key_bytes=4, slot_bytes=8, cg_size=4)
        bf.insert(dev(allk[:n]))
        bfl = torch.zeros(q.size, dtype=torch.bool, device="cuda")
        bf.retrieve(dev(q), bfl)
        rb = o.Bloom(bits, 6, seed=3, key_bytes=4, slot_bytes=8, cg=4)
        rb.insert(allk[:n])
        assert np.array_equal(bfl.cpu().numpy().astype(np.uint8), rb.retrieve(q))
    finally:
        dist.destroy_process_group()


def test_bloom_shards_in_region_passes():
    """shards larger than the random-access region run in region passes over
    their own blocks; words and flags stay the whole filter's slices"""
    kb, sb, cg = 8, 8, 8
    bits = 1 << 26                      # 8 MiB: 3 shards of about 2.7 MiB
    k, seed, parts, n = 6, 0x77, 3, 1 << 19
    keys = o.gen_unique_keys(kb, 2 * n, 43)
    ref = o.Bloom(bits, k, seed=seed, key_bytes=kb, slot_bytes=sb, cg=cg)
    ref.insert(keys[:n])
    words = ref.words()
    want_flags = ref.retrieve(keys)
    nb = bits // (64 * cg)
    blk = bloom_block_np(keys, seed, nb).astype(np.int64)
    prev = wc.set_region_bytes(1 << 20)
    try:
        for s in range(parts):
            sh = wc.BloomFilter(bits, k, seed=seed, key_bytes=kb, slot_bytes=sb, cg_size=cg,
                                shard=s, num_shards=parts)
            lo, hi = bloom_shard_range(nb, s, parts)
            assert (hi - lo) * cg * sb > 2 << 20   # at least 3 passes
            sh.insert(dev(keys[:n]))
            got = copy_device_words(sh.words_ptr(), (hi - lo) * cg, sb)
            assert np.array_equal(got, words[lo * cg:hi * cg])
            fl = torch.full((2 * n,), 9, dtype=torch.uint8, device="cuda")
            sh.retrieve(dev(keys), fl)
            mine = (blk >= lo) & (blk < hi)
            assert np.array_equal(fl.cpu().numpy(), np.where(mine, want_flags, 0))
    finally:
        wc.set_region_bytes(prev)
