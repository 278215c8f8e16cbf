"""Test helpers for the sharded tables and filter: the owner functions
restated in numpy (used to check the partition kernels) and CPU shards over
the oracle (used to test the exchange logic with gloo on CPU)."""
import numpy as np
import torch

from oracle import oracle as o

_M64 = (1 << 64) - 1


def _fmix64(x):
    x = x.astype(np.uint64)
    x ^= x >> np.uint64(33)
    x *= np.uint64(0xFF51AFD7ED558CCD)
    x ^= x >> np.uint64(33)
    x *= np.uint64(0xC4CEB9FE1A85EC53)
    x ^= x >> np.uint64(33)
    return x


def _fmix32(x):
    x = x.astype(np.uint32)
    x ^= x >> np.uint32(16)
    x *= np.uint32(0x85EBCA6B)
    x ^= x >> np.uint32(13)
    x *= np.uint32(0xC2B2AE35)
    x ^= x >> np.uint32(16)
    return x


def owner_np(keys, salt, parts):
    x = _fmix64(keys.astype(np.uint64) ^ np.uint64(salt & _M64))
    return ((x >> np.uint64(32)) * np.uint64(parts)) >> np.uint64(32)


def bloom_block_np(keys, seed, num_blocks):
    """a key's block in a Bloom filter with the Murmur hasher: the fmix of
    (key + seed) over the key width, modulo the number of blocks"""
    if keys.dtype == np.uint32:
        h = _fmix32(keys + np.uint32(seed & 0xFFFFFFFF)).astype(np.uint64)
    else:
        h = _fmix64(keys + np.uint64(seed & _M64))
    return h % np.uint64(num_blocks)


def bloom_owner_np(keys, seed, num_blocks, parts):
    """the shard holding the key's block: block * parts // num_blocks"""
    blk = bloom_block_np(keys, seed, num_blocks).astype(object)
    return np.array([int(b) * parts // num_blocks for b in blk], dtype=np.int64)


def bloom_shard_range(num_blocks, shard, parts):
    """the blocks [lo, hi) of shard `shard`"""
    lo = -(-shard * num_blocks // parts)
    hi = -(-(shard + 1) * num_blocks // parts)
    return lo, hi


def _sorted_partition(keys, values, own, parts, key_bytes):
    udt = np.uint32 if key_bytes == 4 else np.uint64
    sdt = np.int32 if key_bytes == 4 else np.int64
    k = keys.numpy().view(udt)
    perm = np.argsort(own, kind="stable")
    counts = np.bincount(own, minlength=parts).tolist()
    ko = torch.from_numpy(np.ascontiguousarray(k[perm]).view(sdt))
    vo = torch.from_numpy(np.ascontiguousarray(values.numpy()[perm])) if values is not None else None
    return ko, vo, torch.from_numpy(perm.astype(np.int64)), counts


def cpu_partition(parts, salt, key_bytes):
    udt = np.uint32 if key_bytes == 4 else np.uint64

    def fn(keys, values):
        own = owner_np(keys.numpy().view(udt), salt, parts).astype(np.int64)
        return _sorted_partition(keys, values, own, parts, key_bytes)
    return fn


def cpu_bloom_partition(parts, seed, num_blocks, key_bytes):
    udt = np.uint32 if key_bytes == 4 else np.uint64

    def fn(keys, values):
        own = bloom_owner_np(keys.numpy().view(udt), seed, num_blocks, parts)
        return _sorted_partition(keys, values, own, parts, key_bytes)
    return fn


class OracleShard:
    """an oracle table (SVHT, HashSet or CountingHashTable) behind the
    shard interface (CPU tensors)"""

    def __init__(self, cap, key_bytes, kind=o.SVHT):
        self.kb = key_bytes
        self.kind = kind
        self.t = o.Table(kind, key_bytes, 0 if kind == o.HASHSET else key_bytes, cap)
        self.udt = np.uint32 if key_bytes == 4 else np.uint64

    def insert(self, keys, values=None):
        self.t.insert(keys.numpy().view(self.udt),
                      values.numpy().view(self.udt) if values is not None else None)

    def retrieve(self, keys, out, status_out=None):
        o_np = out.numpy() if self.kind == o.HASHSET else out.numpy().view(self.udt)
        res, st = self.t.retrieve(keys.numpy().view(self.udt), o_np, want_status=True)
        if status_out is not None:
            status_out.copy_(torch.from_numpy(st.view(np.int32)))

    def erase(self, keys):
        self.t.erase(keys.numpy().view(self.udt))

    def size(self):
        return self.t.size()

    def init(self):
        self.t.init()


class OracleBloomShard:
    """an oracle filter of the whole size behind the shard interface: with
    the keys routed to it by block, its answers are those of the rank's
    block range"""

    def __init__(self, num_bits, k, seed, key_bytes):
        self.f = o.Bloom(num_bits, k, seed=seed, key_bytes=key_bytes)
        self.udt = np.uint32 if key_bytes == 4 else np.uint64

    def insert(self, keys):
        self.f.insert(keys.numpy().view(self.udt))

    def retrieve(self, keys, out):
        out.copy_(torch.from_numpy(self.f.retrieve(keys.numpy().view(self.udt))))

    def init(self):
        pass
