"""Test helpers for the sharded table: the owner function restated in numpy
(used to check wc_partition) and a CPU shard over the oracle (used to test
the exchange logic with gloo on CPU)."""
import numpy as np
import torch

from oracle import oracle as o


def owner_np(keys, salt, parts):
    x = keys.astype(np.uint64) ^ np.uint64(salt & ((1 << 64) - 1))
    x ^= x >> np.uint64(33)
    x *= np.uint64(0xFF51AFD7ED558CCD)
    x ^= x >> np.uint64(33)
    x *= np.uint64(0xC4CEB9FE1A85EC53)
    x ^= x >> np.uint64(33)
    return ((x >> np.uint64(32)) * np.uint64(parts)) >> np.uint64(32)


def cpu_partition(parts, salt, key_bytes):
    udt = np.uint32 if key_bytes == 4 else np.uint64
    sdt = np.int32 if key_bytes == 4 else np.int64

    def fn(keys, values):
        k = keys.numpy().view(udt)
        own = owner_np(k, salt, parts).astype(np.int64)
        perm = np.argsort(own, kind="stable")
        counts = np.bincount(own, minlength=parts).tolist()
        ko = torch.from_numpy(np.ascontiguousarray(k[perm]).view(sdt))
        vo = torch.from_numpy(np.ascontiguousarray(values.numpy()[perm])) if values is not None else None
        return ko, vo, torch.from_numpy(perm.astype(np.int64)), counts
    return fn


class OracleShard:
    """the oracle table behind the shard interface (CPU tensors)"""

    def __init__(self, cap, key_bytes):
        self.kb = key_bytes
        self.t = o.Table(o.SVHT, key_bytes, key_bytes, cap)
        self.udt = np.uint32 if key_bytes == 4 else np.uint64

    def insert(self, keys, values):
        self.t.insert(keys.numpy().view(self.udt), values.numpy().view(self.udt))

    def retrieve(self, keys, out, status_out=None):
        o_np = out.numpy().view(self.udt)
        res, st = self.t.retrieve(keys.numpy().view(self.udt), o_np, want_status=True)
        if status_out is not None:
            status_out.copy_(torch.from_numpy(st.view(np.int32)))

    def erase(self, keys):
        self.t.erase(keys.numpy().view(self.udt))

    def size(self):
        return self.t.size()

    def init(self):
        self.t.init()
