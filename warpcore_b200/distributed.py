"""A SingleValueHashTable sharded over the ranks of a process group.

The reference is single-GPU. Here each rank owns one shard: a
SingleValueHashTable of ceil(min_capacity / world) slots on its GPU. A bulk
operation may be called on every rank with keys of any owner. Each call
runs these steps:
1. Route: wc_partition groups the keys by owner. The owner is a
   multiply-shift of a mix that is independent of the probing hashers.
2. Exchange: one all-to-all of the counts, then one of keys (and values).
   On NCCL over NVLink/NVSwitch this is a grouped send/recv.
3. The owner runs the bulk kernel on its shard.
4. Retrieve only: one reverse all-to-all of the values and per-key
   statuses, put back in input order through the partition's permutation.
   Values are written on hits only, as the reference's retrieve does.

Every rank must call every operation, in the same order (collectives).
`size()` is the sum over shards.

`partition_fn`, `restore_fn` and `shard_factory` exist so that the host
logic can be tested with the gloo backend on CPU, against the CPU oracle.
On a GPU the defaults are the CUDA partition and restore kernels and a
warpcore_b200 table. There is no fallback between the two.
"""
import ctypes

import torch
import torch.distributed as dist

import warpcore_b200 as wc

DEFAULT_SALT = 0x243F6A8885A308D3


def _int_dtype(nbytes):
    return torch.int32 if nbytes == 4 else torch.int64


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
    GPU: values on hits only, statuses if status_out is given"""
    n = perm.numel()
    if n == 0:
        return
    wc._check(wc.lib().wc_partition_restore(
        values.data_ptr(), status.data_ptr(), perm.data_ptr(), n, values.element_size(),
        values_out.data_ptr(), status_out.data_ptr() if status_out is not None else None,
        torch.cuda.current_stream(values.device).cuda_stream))


def cpu_restore(values, status, perm, values_out, status_out=None):
    """the same step with torch indexing, for CPU tensors"""
    hit = status == 0
    values_out[perm[hit]] = values[hit]
    if status_out is not None:
        status_out[perm] = status


class DistributedSingleValueHashTable:
    def __init__(self, min_capacity, key_bytes=4, seed=wc.DEFAULT_SEED, group=None,
                 salt=DEFAULT_SALT, shard_factory=None, partition_fn=None, restore_fn=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.key_bytes = key_bytes
        self.salt = salt
        shard_cap = -(-int(min_capacity) // self.world)
        if shard_factory is None:
            self.shard = wc.SingleValueHashTable(shard_cap, seed=seed, key_bytes=key_bytes)
        else:
            self.shard = shard_factory(shard_cap)
        self._partition = partition_fn or (
            lambda k, v: gpu_partition(k, v, self.world, self.salt, self.key_bytes))
        self._restore = restore_fn or gpu_restore

    # -- exchange helpers --------------------------------------------------
    def _counts(self, send_counts, device):
        send = torch.tensor(send_counts, dtype=torch.int64, device=device)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=self.group)
        return recv.tolist()

    def _a2a(self, x, send_counts, recv_counts):
        out = torch.empty(sum(recv_counts), dtype=x.dtype, device=x.device)
        dist.all_to_all_single(out, x, recv_counts, send_counts, group=self.group)
        return out

    # -- operations ------------------------------------------------------
    def insert(self, keys, values):
        k, v, _, send = self._partition(keys, values)
        recv = self._counts(send, keys.device)
        rk = self._a2a(k, send, recv)
        rv = self._a2a(v, send, recv)
        if rk.numel():
            self.shard.insert(rk, rv)

    def retrieve(self, keys, values_out, status_out=None):
        """values_out written on hits only; status_out (int32) gets each
        key's Status bits"""
        k, _, perm, send = self._partition(keys, None)
        recv = self._counts(send, keys.device)
        rk = self._a2a(k, send, recv)
        # the shard writes every status and the values of hits; the restore
        # step reads a value only where the status is 0
        local_out = torch.empty(rk.numel(), dtype=values_out.dtype, device=keys.device)
        local_st = torch.empty(rk.numel(), dtype=torch.int32, device=keys.device)
        if rk.numel():
            self.shard.retrieve(rk, local_out, status_out=local_st)
        back_v = self._a2a(local_out, recv, send)
        back_s = self._a2a(local_st, recv, send)
        self._restore(back_v, back_s, perm, values_out, status_out)
        return status_out

    def erase(self, keys):
        k, _, _, send = self._partition(keys, None)
        recv = self._counts(send, keys.device)
        rk = self._a2a(k, send, recv)
        if rk.numel():
            self.shard.erase(rk)

    def size(self):
        n = torch.tensor([self.shard.size()], dtype=torch.int64,
                         device="cuda" if dist.get_backend(self.group) == "nccl" else "cpu")
        dist.all_reduce(n, group=self.group)
        return int(n.item())

    def init(self):
        self.shard.init()
