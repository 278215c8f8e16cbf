"""The sharded table's routing and exchange (warpcore_b200.distributed) on
two gloo ranks on CPU, with the CPU oracle as each rank's shard: every rank
inserts its own keys, every rank retrieves keys owned anywhere, and the
answers equal those of one unsharded table."""
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
