"""The sharded containers' routing and exchange (warpcore_b200.distributed)
on two and three gloo ranks on CPU, with the CPU oracle as each rank's
shard: every rank inserts its own keys, every rank retrieves keys owned
anywhere, and the answers equal those of one unsharded table or filter."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as o


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, kb, errq):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from tests.partition_ref import OracleShard, cpu_partition
        from warpcore_b200.distributed import (DEFAULT_SALT, DistributedSingleValueHashTable,
                                               cpu_restore)
        udt = np.uint32 if kb == 4 else np.uint64
        sdt = np.int32 if kb == 4 else np.int64
        n = 3000
        allk = o.gen_unique_keys(kb, world * n + 1000, 5)
        vals = o.gen_uniform(kb, world * n, 6)
        t = DistributedSingleValueHashTable(4 * world * n, key_bytes=kb,
                                            shard_factory=lambda cap: OracleShard(cap, kb),
                                            partition_fn=cpu_partition(world, DEFAULT_SALT, kb),
                                            restore_fn=cpu_restore)
        mine = slice(rank * n, (rank + 1) * n)
        t.insert(torch.from_numpy(allk[mine].view(sdt)), torch.from_numpy(vals[mine].view(sdt)))
        assert t.size() == world * n
        # every rank asks for keys of all ranks plus absent ones
        rng = np.random.default_rng(rank)
        q = np.concatenate([allk[rng.integers(0, world * n, 2000)], allk[world * n:]])
        out = torch.full((q.size,), 7, dtype=torch.int32 if kb == 4 else torch.int64)
        st = torch.zeros(q.size, dtype=torch.int32)
        t.retrieve(torch.from_numpy(q.view(sdt)), out, st)
        ref = o.Table(o.SVHT, kb, kb, 4 * world * n)
        ref.insert(allk[:world * n], vals)
        r_out, r_st = ref.retrieve(q, np.full(q.size, 7, dtype=udt), want_status=True)
        assert np.array_equal(out.numpy().view(udt), r_out)
        assert np.array_equal(st.numpy().view(np.uint32), r_st)
        # erase a part on every rank, then ask again
        t.erase(torch.from_numpy(allk[mine][::3].view(sdt)))
        for r in range(world):
            ref.erase(allk[r * n:(r + 1) * n][::3])
        assert t.size() == ref.size()
        out2 = torch.full((q.size,), 7, dtype=out.dtype)
        t.retrieve(torch.from_numpy(q.view(sdt)), out2)
        r_out2 = ref.retrieve(q, np.full(q.size, 7, dtype=udt))
        assert np.array_equal(out2.numpy().view(udt), r_out2)
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report to the parent
        import traceback
        errq.put((rank, traceback.format_exc()))
        raise


def _set_count_worker(rank, world, port, kb, errq):
    """HashSet and CountingHashTable shards: keys inserted on every rank
    (repeats included), asked for on every rank"""
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from tests.partition_ref import OracleShard, cpu_partition
        from warpcore_b200.distributed import (DEFAULT_SALT, DistributedCountingHashTable,
                                               DistributedHashSet, cpu_restore)
        udt = np.uint32 if kb == 4 else np.uint64
        sdt = np.int32 if kb == 4 else np.int64
        n = 2000
        allk = o.gen_unique_keys(kb, world * n + 500, 15)
        part = cpu_partition(world, DEFAULT_SALT, kb)
        hs = DistributedHashSet(4 * world * n, key_bytes=kb,
                                shard_factory=lambda cap: OracleShard(cap, kb, o.HASHSET),
                                partition_fn=part, restore_fn=cpu_restore)
        ct = DistributedCountingHashTable(4 * world * n, key_bytes=kb,
                                          shard_factory=lambda cap: OracleShard(cap, kb, o.COUNTING),
                                          partition_fn=part, restore_fn=cpu_restore)
        # rank r inserts its block of keys, and every rank the first 300 keys
        # once more (so those are counted world + 1 times)
        mine = np.concatenate([allk[rank * n:(rank + 1) * n], allk[:300]])
        hs.insert(torch.from_numpy(mine.view(sdt)))
        ct.insert(torch.from_numpy(mine.view(sdt)))
        ref_s = o.Table(o.HASHSET, kb, 0, 4 * world * n)
        ref_c = o.Table(o.COUNTING, kb, kb, 4 * world * n)
        for r in range(world):
            rk = np.concatenate([allk[r * n:(r + 1) * n], allk[:300]])
            ref_s.insert(rk)
            ref_c.insert(rk)
        assert hs.size() == ref_s.size() == world * n
        assert ct.size() == ref_c.size()
        rng = np.random.default_rng(rank + 10)
        q = np.concatenate([allk[rng.integers(0, world * n, 1500)], allk[world * n:]])
        qt = torch.from_numpy(q.view(sdt))
        flags = torch.full((q.size,), 9, dtype=torch.uint8)
        st = torch.zeros(q.size, dtype=torch.int32)
        hs.retrieve(qt, flags, st)
        r_f, r_st = ref_s.retrieve(q, np.full(q.size, 9, dtype=np.uint8), want_status=True)
        assert np.array_equal(flags.numpy(), r_f)
        assert np.array_equal(st.numpy().view(np.uint32), r_st)
        cnt = torch.full((q.size,), 7, dtype=torch.int32 if kb == 4 else torch.int64)
        st2 = torch.zeros(q.size, dtype=torch.int32)
        ct.retrieve(qt, cnt, st2)
        r_c, r_st2 = ref_c.retrieve(q, np.full(q.size, 7, dtype=udt), want_status=True)
        assert np.array_equal(cnt.numpy().view(udt), r_c)
        assert np.array_equal(st2.numpy().view(np.uint32), r_st2)
        # erase on every rank
        hs.erase(torch.from_numpy(allk[rank * n:(rank + 1) * n][::4].view(sdt)))
        for r in range(world):
            ref_s.erase(allk[r * n:(r + 1) * n][::4])
        assert hs.size() == ref_s.size()
        flags2 = torch.full((q.size,), 9, dtype=torch.uint8)
        hs.retrieve(qt, flags2)
        assert np.array_equal(flags2.numpy(), ref_s.retrieve(q, np.full(q.size, 9, dtype=np.uint8)))
        dist.barrier()
        dist.destroy_process_group()
    except Exception:  # report to the parent
        import traceback
        errq.put((rank, traceback.format_exc()))
        raise


def _bloom_worker(rank, world, port, kb, errq):
    """a filter split by blocks: every rank inserts its keys, the flags of
    keys asked anywhere equal those of one filter"""
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from tests.partition_ref import OracleBloomShard, cpu_bloom_partition
        from warpcore_b200.distributed import DistributedBloomFilter, cpu_restore
        sdt = np.int32 if kb == 4 else np.int64
        n, bits, k, seed = 4000, 1 << 17, 4, 0x1234
        ref = o.Bloom(bits, k, seed=seed, key_bytes=kb)
        f = DistributedBloomFilter(bits, k, seed=seed, key_bytes=kb,
                                   shard_factory=lambda r, w: OracleBloomShard(bits, k, seed, kb),
                                   partition_fn=cpu_bloom_partition(world, seed, ref.num_blocks, kb),
                                   restore_fn=cpu_restore)
        allk = o.gen_unique_keys(kb, world * n + 3000, 25)
        f.insert(torch.from_numpy(allk[rank * n:(rank + 1) * n].view(sdt)))
        ref.insert(allk[:world * n])
        rng = np.random.default_rng(rank + 20)
        q = np.concatenate([allk[rng.integers(0, world * n, 1000)], allk[world * n:]])
        flags = torch.full((q.size,), 9, dtype=torch.bool).view(torch.uint8)
        f.retrieve(torch.from_numpy(q.view(sdt)), flags)
        want = ref.retrieve(q)
        assert np.array_equal(flags.numpy(), want)
        # the absent keys include a few false positives at this load
        assert 0 < int(want[1000:].sum()) < 300
        dist.barrier()
        dist.destroy_process_group()
    except Exception:  # report to the parent
        import traceback
        errq.put((rank, traceback.format_exc()))
        raise


def _run(target, world, kb):
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, kb, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not errs, errs
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


@pytest.mark.parametrize("kb", [4, 8])
def test_hash_set_and_counting_gloo_ranks_match_one_table(kb):
    _run(_set_count_worker, 2, kb)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("kb", [4, 8])
def test_bloom_gloo_ranks_match_one_filter(world, kb):
    _run(_bloom_worker, world, kb)


def test_bloom_owner_matches_block_ranges():
    from tests.partition_ref import bloom_block_np, bloom_owner_np, bloom_shard_range
    keys = o.gen_unique_keys(8, 50000, 9)
    nb = 10007
    for parts in (1, 2, 3, 8):
        own = bloom_owner_np(keys, 77, nb, parts)
        blk = bloom_block_np(keys, 77, nb).astype(np.int64)
        for s in range(parts):
            lo, hi = bloom_shard_range(nb, s, parts)
            assert np.array_equal(own == s, (blk >= lo) & (blk < hi))
        assert sum(bloom_shard_range(nb, s, parts)[1] - bloom_shard_range(nb, s, parts)[0]
                   for s in range(parts)) == nb


@pytest.mark.parametrize("kb", [4, 8])
def test_two_gloo_ranks_match_one_table(kb):
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, kb, errq)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not errs, errs
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


def test_owner_function_is_balanced():
    from tests.partition_ref import owner_np
    keys = o.gen_unique_keys(8, 200000, 3)
    for parts in (2, 3, 8, 64):
        own = owner_np(keys, 0x243F6A8885A308D3, parts)
        c = np.bincount(own.astype(np.int64), minlength=parts)
        assert c.size == parts
        assert c.min() > 0.9 * keys.size / parts
