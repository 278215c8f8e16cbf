"""Tables and filters sharded over the ranks of a process group.

The reference is single-GPU. Here each rank owns one shard on its GPU:
- DistributedSingleValueHashTable, DistributedHashSet and
  DistributedCountingHashTable: a table of ceil(min_capacity / world)
  slots; a key's owner is a multiply-shift of a mix that is independent of
  the probing hashers (wc_partition).
- DistributedBloomFilter: a block range of one filter
  (wc_bloom_create_shard); a key's owner is the rank holding its block
  (wc_bloom_partition), so all its bits live on one rank and the answers
  are those of the one unsharded filter, bit for bit.

A bulk operation may be called on every rank with keys of any owner. Each
call runs these steps:
1. Route: the partition kernels group the keys by owner.
2. Exchange: one all-to-all of the counts, then one of keys (and values).
   On NCCL over NVLink/NVSwitch this is a grouped send/recv.
3. The owner runs the bulk kernel on its shard.
4. Retrieve only: one reverse all-to-all of the answers (and per-key
   statuses), put back in input order through the partition's
   permutation. Values and flags are written where the status is 0, as the
   reference's retrieve writes them; a filter's flags are always written.

Every rank must call every operation, in the same order (collectives).
`size()` is the sum over shards.

`partition_fn`, `restore_fn` and `shard_factory` exist so that the host
logic can be tested with the gloo backend on CPU, against the CPU oracle.
On a GPU the defaults are the CUDA partition and restore kernels and a
warpcore_b200 table or filter. There is no fallback between the two.
"""
import torch
import torch.distributed as dist

import warpcore_b200 as wc

DEFAULT_SALT = 0x243F6A8885A308D3


def gpu_partition(keys, values, parts, salt, key_bytes):
    """group keys (and values) by owner on the GPU: returns (keys_out,
    values_out or None, perm, counts as a list of ints)"""
    n = keys.numel()
    dev = keys.device
    keys_out = torch.empty_like(keys)
    values_out = torch.empty_like(values) if values is not None else None
    perm = torch.empty(n, dtype=torch.int64, device=dev)
    # one buffer: counts (parts) | offsets, cursors (2 * parts) | dropped (1)
    buf = torch.empty(3 * parts + 1, dtype=torch.int64, device=dev)
    wc._check(wc.lib().wc_partition(
        keys.data_ptr() if n else None, values.data_ptr() if values is not None and n else None,
        n, key_bytes, key_bytes if values is not None else 0, parts, salt & ((1 << 64) - 1),
        keys_out.data_ptr() if n else None, values_out.data_ptr() if values_out is not None and n else None,
        perm.data_ptr() if n else None, buf.data_ptr(), buf[parts:].data_ptr(),
        torch.cuda.current_stream(dev).cuda_stream))
    host_buf = buf.tolist()
    if host_buf[-1]:
        raise wc.WarpcoreError("wc_partition dropped %d keys whose position failed the bounds "
                               "check (keys changed during the call)" % host_buf[-1])
    return keys_out, values_out, perm, host_buf[:parts]


def gpu_restore(values, status, perm, values_out, status_out=None):
    """put answers (in owner order) back at their input positions on the
    GPU: values where the status is 0 (always if status is None), statuses
    if status_out is given"""
    n = perm.numel()
    if n == 0:
        return
    wc._check(wc.lib().wc_partition_restore(
        values.data_ptr(), status.data_ptr() if status is not None else None, perm.data_ptr(), n,
        values.element_size(), values_out.data_ptr(),
        status_out.data_ptr() if status_out is not None else None,
        torch.cuda.current_stream(values.device).cuda_stream))


def cpu_restore(values, status, perm, values_out, status_out=None):
    """the same step with torch indexing, for CPU tensors"""
    if status is None:
        values_out[perm] = values
        return
    hit = status == 0
    values_out[perm[hit]] = values[hit]
    if status_out is not None:
        status_out[perm] = status


def _bytes_view(t):
    """flags travel as uint8 (a bool tensor shares their storage)"""
    return t.view(torch.uint8) if t.dtype == torch.bool else t


class _Sharded:
    """routing and exchange shared by the sharded containers"""

    def _setup(self, group, partition_fn, restore_fn):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self._partition = partition_fn
        self._restore = restore_fn or gpu_restore

    def _counts(self, send_counts, device):
        send = torch.tensor(send_counts, dtype=torch.int64, device=device)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=self.group)
        return recv.tolist()

    def _a2a(self, x, send_counts, recv_counts):
        out = torch.empty(sum(recv_counts), dtype=x.dtype, device=x.device)
        dist.all_to_all_single(out, x, recv_counts, send_counts, group=self.group)
        return out

    def _route(self, keys, values=None):
        """steps 1 and 2: returns (keys received, values received or None,
        perm, send counts, receive counts)"""
        k, v, perm, send = self._partition(keys, values)
        recv = self._counts(send, keys.device)
        rk = self._a2a(k, send, recv)
        rv = self._a2a(v, send, recv) if v is not None else None
        return rk, rv, perm, send, recv

    def _lookup(self, keys, out, status_out, answer_dtype, run):
        """steps 1 to 4 of a retrieve: run(rk, local_out, local_status) on
        the shard, answers back to their ranks and input positions"""
        rk, _, perm, send, recv = self._route(keys)
        local_out = torch.empty(rk.numel(), dtype=answer_dtype, device=keys.device)
        local_st = torch.empty(rk.numel(), dtype=torch.int32, device=keys.device)
        if rk.numel():
            run(rk, local_out, local_st)
        back_v = self._a2a(local_out, recv, send)
        back_s = self._a2a(local_st, recv, send)
        self._restore(back_v, back_s, perm, out, status_out)
        return status_out

    def _sum(self, local):
        n = torch.tensor([int(local)], dtype=torch.int64,
                         device="cuda" if dist.get_backend(self.group) == "nccl" else "cpu")
        dist.all_reduce(n, group=self.group)
        return int(n.item())


class _ShardedTable(_Sharded):
    """a hash table sharded by the salted owner function"""

    def __init__(self, min_capacity, key_bytes, group, salt, shard_factory, partition_fn,
                 restore_fn, make_default):
        world = dist.get_world_size(group)
        self.key_bytes = key_bytes
        self.salt = salt
        shard_cap = -(-int(min_capacity) // world)
        self.shard = (shard_factory or make_default)(shard_cap)
        self._setup(group, partition_fn or (
            lambda k, v: gpu_partition(k, v, self.world, self.salt, self.key_bytes)), restore_fn)

    def erase(self, keys):
        rk, _, _, _, _ = self._route(keys)
        if rk.numel():
            self.shard.erase(rk)

    def size(self):
        return self._sum(self.shard.size())

    def init(self):
        self.shard.init()


class DistributedSingleValueHashTable(_ShardedTable):
    def __init__(self, min_capacity, key_bytes=4, seed=wc.DEFAULT_SEED, group=None,
                 salt=DEFAULT_SALT, shard_factory=None, partition_fn=None, restore_fn=None):
        super().__init__(min_capacity, key_bytes, group, salt, shard_factory, partition_fn,
                         restore_fn,
                         lambda cap: wc.SingleValueHashTable(cap, seed=seed, key_bytes=key_bytes))

    def insert(self, keys, values):
        rk, rv, _, _, _ = self._route(keys, values)
        if rk.numel():
            self.shard.insert(rk, rv)

    def retrieve(self, keys, values_out, status_out=None):
        """values_out written on hits only; status_out (int32) gets each
        key's Status bits"""
        return self._lookup(keys, values_out, status_out, values_out.dtype,
                            lambda rk, o, st: self.shard.retrieve(rk, o, status_out=st))


class DistributedHashSet(_ShardedTable):
    def __init__(self, min_capacity, key_bytes=4, seed=wc.DEFAULT_SEED, group=None,
                 salt=DEFAULT_SALT, shard_factory=None, partition_fn=None, restore_fn=None):
        super().__init__(min_capacity, key_bytes, group, salt, shard_factory, partition_fn,
                         restore_fn, lambda cap: wc.HashSet(cap, seed=seed, key_bytes=key_bytes))

    def insert(self, keys):
        rk, _, _, _, _ = self._route(keys)
        if rk.numel():
            self.shard.insert(rk)

    def retrieve(self, keys, flags_out, status_out=None):
        """membership flags (bool or uint8), written where the status is 0"""
        self._lookup(keys, _bytes_view(flags_out), status_out, torch.uint8,
                     lambda rk, o, st: self.shard.retrieve(rk, o, status_out=st))
        return status_out

    contains = retrieve


class DistributedCountingHashTable(_ShardedTable):
    def __init__(self, min_capacity, key_bytes=4, seed=wc.DEFAULT_SEED, max_count=None,
                 group=None, salt=DEFAULT_SALT, shard_factory=None, partition_fn=None,
                 restore_fn=None):
        super().__init__(min_capacity, key_bytes, group, salt, shard_factory, partition_fn,
                         restore_fn,
                         lambda cap: wc.CountingHashTable(cap, seed=seed, key_bytes=key_bytes,
                                                          max_count=max_count))

    def insert(self, keys):
        rk, _, _, _, _ = self._route(keys)
        if rk.numel():
            self.shard.insert(rk)

    def retrieve(self, keys, values_out, status_out=None):
        """counts written where the status is 0 (key present)"""
        return self._lookup(keys, values_out, status_out, values_out.dtype,
                            lambda rk, o, st: self.shard.retrieve(rk, o, status_out=st))


class DistributedBloomFilter(_Sharded):
    """One Bloom filter of num_bits bits whose blocks are split over the
    ranks in contiguous ranges. Blocks of at most 128 bytes (slot_bytes x
    cg_size), num_bits a multiple of the block's bits."""

    def __init__(self, num_bits, k, seed=wc.DEFAULT_SEED, key_bytes=8, slot_bytes=8,
                 cg_size=1, hasher=wc.HASH_MURMUR, group=None, shard_factory=None,
                 partition_fn=None, restore_fn=None):
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        if shard_factory is None:
            self.shard = wc.BloomFilter(num_bits, k, seed=seed, key_bytes=key_bytes,
                                        slot_bytes=slot_bytes, cg_size=cg_size, hasher=hasher,
                                        shard=rank, num_shards=world)
        else:
            self.shard = shard_factory(rank, world)
        self._setup(group, partition_fn or self._gpu_partition, restore_fn)

    def _gpu_partition(self, keys, values):
        ko, perm, counts = self.shard.partition(keys, self.world)
        return ko, None, perm, counts

    def insert(self, keys):
        rk, _, _, _, _ = self._route(keys)
        if rk.numel():
            self.shard.insert(rk)

    def retrieve(self, keys, flags_out):
        """one flag per key (bool or uint8), for every key"""
        rk, _, perm, send, recv = self._route(keys)
        local = torch.empty(rk.numel(), dtype=torch.uint8, device=keys.device)
        if rk.numel():
            self.shard.retrieve(rk, local)
        back = self._a2a(local, recv, send)
        self._restore(back, None, perm, _bytes_view(flags_out), None)

    contains = retrieve

    def init(self):
        self.shard.init()
