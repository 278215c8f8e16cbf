"""TEST INFRASTRUCTURE ONLY: ctypes binding of the C oracle (wc_oracle.c).

The oracle is a CPU restatement of warpcore's hot path used as the checker of
the CUDA library.  Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline legs import this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libwc_oracle.so")

HASH_MURMUR, HASH_NVIDIA, HASH_MUELLER, HASH_IDENTITY32, HASH_IDENTITY64 = range(5)
PROBE_DOUBLE, PROBE_LINEAR, PROBE_QUADRATIC = range(3)
SVHT, HASHSET, COUNTING, MULTIVALUE = range(4)

ST_NONE = 0
ST_UNKNOWN_ERROR = 1 << 0
ST_PROBING_LENGTH_EXCEEDED = 1 << 1
ST_INVALID_CONFIGURATION = 1 << 2
ST_INVALID_KEY = 1 << 3
ST_DUPLICATE_KEY = 1 << 4
ST_KEY_NOT_FOUND = 1 << 5
ST_INDEX_OVERFLOW = 1 << 6
ST_OUT_OF_MEMORY = 1 << 7
ST_NOT_INITIALIZED = 1 << 8
ST_DRY_RUN = 1 << 9
ST_INVALID_PHASE_OVERLAP = 1 << 10
ST_MAX_VALUES_REACHED = 1 << 11

DEFAULT_SEED = 0x5AD0DED
DEFAULT_PROBING_LENGTH = (2**64 - 1) - 1024

_u64 = ctypes.c_uint64
_vp = ctypes.c_void_p
_i = ctypes.c_int


def build():
    """Compile libwc_oracle.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    sig = {
        "wco_hash": (_u64, [_i, _i, _u64]),
        "wco_hash_bits": (_i, [_i, _i]),
        "wco_num_primes": (_u64, []),
        "wco_primes": (None, [_vp]),
        "wco_valid_capacity": (_u64, [_u64, _u64]),
        "wco_probe_sequence": (_u64, [_i, _i, _i, _i, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
        "wco_status_to_bool": (ctypes.c_uint8, [ctypes.c_uint32, ctypes.c_uint32]),
        "wco_table_create": (_vp, [_i, _i, _i, _u64, _u64, _u64, _i, _i, _i, _u64, _u64, _u64]),
        "wco_table_destroy": (None, [_vp]),
        "wco_mv_create": (_vp, [_i, _i, _u64, _u64, _u64, _i, _i, _i, _u64, _u64, _u64]),
        "wco_mv_insert": (None, [_vp, _vp, _vp, _u64, _u64, _vp]),
        "wco_mv_num_values": (_u64, [_vp, _vp, _u64, _vp, _u64, _vp]),
        "wco_mv_retrieve": (_u64, [_vp, _vp, _u64, _vp, _vp, _vp, _u64, _vp]),
        "wco_mv_num_keys": (_u64, [_vp]),
        "wco_mv_unique_keys": (_u64, [_vp, _vp]),
        "wco_bl_create": (_vp, [_i, _i, _u64, _u64, _u64, ctypes.c_float, _u64, _u64, _u64, _u64,
                                _u64, _u64, _u64]),
        "wco_bl_destroy": (None, [_vp]),
        "wco_bl_init": (None, [_vp, _u64]),
        "wco_bl_key_capacity": (_u64, [_vp]),
        "wco_bl_insert": (None, [_vp, _vp, _vp, _u64, _u64, _vp]),
        "wco_bl_num_values": (_u64, [_vp, _vp, _u64, _vp, _u64, _vp]),
        "wco_bl_retrieve": (_u64, [_vp, _vp, _u64, _vp, _vp, _vp, _u64, _vp]),
        "wco_bl_num_keys": (_u64, [_vp]),
        "wco_bl_total_values": (_u64, [_vp]),
        "wco_bl_next_free": (_u64, [_vp]),
        "wco_bl_all_keys": (_u64, [_vp, _vp]),
        "wco_bl_peek_status": (ctypes.c_uint32, [_vp]),
        "wco_bl_pop_status": (ctypes.c_uint32, [_vp]),
        "wco_mb_create": (_vp, [_i, _i, _u64, _u64, _u64, _u64, _i, _i, _i, _u64, _u64, _u64,
                                _u64]),
        "wco_mb_destroy": (None, [_vp]),
        "wco_mb_capacity": (_u64, [_vp]),
        "wco_mb_init": (None, [_vp, _u64]),
        "wco_mb_insert": (None, [_vp, _vp, _vp, _u64, _u64, _vp]),
        "wco_mb_num_values": (_u64, [_vp, _vp, _u64, _vp, _u64, _vp]),
        "wco_mb_retrieve": (_u64, [_vp, _vp, _u64, _vp, _vp, _vp, _u64, _vp]),
        "wco_mb_num_keys": (_u64, [_vp]),
        "wco_mb_num_occupied": (_u64, [_vp]),
        "wco_mb_size": (_u64, [_vp]),
        "wco_mb_unique_keys": (_u64, [_vp, _vp]),
        "wco_mb_peek_status": (ctypes.c_uint32, [_vp]),
        "wco_mb_pop_status": (ctypes.c_uint32, [_vp]),
        "wco_table_capacity": (_u64, [_vp]),
        "wco_table_init": (None, [_vp, _u64]),
        "wco_insert": (None, [_vp, _vp, _vp, _u64, _u64, _vp]),
        "wco_retrieve": (None, [_vp, _vp, _u64, _vp, _u64, _vp]),
        "wco_erase": (None, [_vp, _vp, _u64, _u64, _vp]),
        "wco_size": (_u64, [_vp]),
        "wco_retrieve_all": (_u64, [_vp, _vp, _vp]),
        "wco_peek_status": (ctypes.c_uint32, [_vp]),
        "wco_pop_status": (ctypes.c_uint32, [_vp]),
        "wco_table_slots": (None, [_vp, _vp, _vp]),
        "wco_bloom_create": (_vp, [_i, _i, _u64, _i, _u64, _u64, _u64]),
        "wco_bloom_destroy": (None, [_vp]),
        "wco_bloom_insert": (None, [_vp, _vp, _u64]),
        "wco_bloom_retrieve": (None, [_vp, _vp, _u64, _vp]),
        "wco_bloom_num_slots": (_u64, [_vp]),
        "wco_bloom_num_blocks": (_u64, [_vp]),
        "wco_bloom_words": (None, [_vp, _vp]),
        "wco_bloom_fpr": (ctypes.c_double, [_vp, _u64]),
        "wco_gen_unique_keys": (None, [_i, _u64, _u64, _vp]),
        "wco_gen_uniform": (None, [_i, _u64, _u64, _vp]),
        "wco_gen_zipf_ranks": (None, [_u64, ctypes.c_double, _u64, _u64, _vp]),
        "wco_gen_zipf_streams": (None, [_vp, _u64, _vp, _u64, _i, ctypes.c_double, _u64]),
        "wco_mt_create": (_vp, [_i, _i, _u64, _u64, _u64]),
        "wco_mt_destroy": (None, [_vp]),
        "wco_mt_clear": (None, [_vp, _i]),
        "wco_mt_insert": (ctypes.c_double, [_vp, _vp, _vp, _u64, _i]),
        "wco_mt_retrieve": (ctypes.c_double, [_vp, _vp, _u64, _vp, _vp, _i]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _kdtype(key_bytes):
    return np.uint32 if key_bytes == 4 else np.uint64


def hash_(hasher, key_bytes, x):
    return lib().wco_hash(hasher, key_bytes, int(x))


def primes():
    n = lib().wco_num_primes()
    out = np.empty(n, dtype=np.uint64)
    lib().wco_primes(_ptr(out))
    return out


def valid_capacity(min_capacity, cg):
    return lib().wco_valid_capacity(int(min_capacity), int(cg))


def probe_sequence(scheme, h1, h2, key_bytes, cg, capacity, key, seed,
                   probing_length, max_windows):
    out = np.zeros(max_windows * cg, dtype=np.uint64)
    w = lib().wco_probe_sequence(scheme, h1, h2, key_bytes, cg, capacity,
                                 int(key), int(seed), int(probing_length),
                                 max_windows, _ptr(out))
    return out[: w * cg].reshape(w, cg)


def status_to_bool(status, ignore=0):
    return bool(lib().wco_status_to_bool(int(status), int(ignore)))


def gen_unique_keys(key_bytes, n, seed):
    out = np.empty(n, dtype=_kdtype(key_bytes))
    lib().wco_gen_unique_keys(key_bytes, n, seed, _ptr(out))
    return out


def gen_uniform(nbytes, n, seed):
    out = np.empty(n, dtype=_kdtype(nbytes))
    lib().wco_gen_uniform(nbytes, n, seed, _ptr(out))
    return out


def gen_zipf_ranks(n_in, s, n_out, seed):
    out = np.empty(n_out, dtype=np.uint64)
    lib().wco_gen_zipf_ranks(n_in, s, n_out, seed, _ptr(out))
    return out


def gen_zipf_streams(n_in, s, n_out, seed, key_bytes=8, in_=None):
    """Zipf draws with one stream per output (the library generator's form):
    1-based ranks, or in_[rank - 1]"""
    out = np.empty(n_out, dtype=_kdtype(key_bytes))
    lib().wco_gen_zipf_streams(_ptr(in_), n_in, _ptr(out), n_out, key_bytes, float(s), seed)
    return out


class Table:
    """Sequential reference-order table (SVHT, HashSet or CountingHashTable)."""

    def __init__(self, kind, key_bytes, value_bytes, min_capacity,
                 seed=DEFAULT_SEED, cg=8, scheme=PROBE_DOUBLE,
                 h1=HASH_MURMUR, h2=HASH_MURMUR, empty_key=0,
                 tombstone_key=None, max_count=None):
        if tombstone_key is None:
            tombstone_key = (1 << (8 * key_bytes)) - 1
        if max_count is None:
            max_count = (1 << (8 * value_bytes)) - 1 if value_bytes else 0
        self.kind = kind
        self.key_bytes = key_bytes
        self.value_bytes = 0 if kind == HASHSET else value_bytes
        self.h = lib().wco_table_create(kind, key_bytes, value_bytes,
                                        int(min_capacity), int(seed), cg,
                                        scheme, h1, h2, int(empty_key),
                                        int(tombstone_key), int(max_count))

    def __del__(self):
        if getattr(self, "h", None):
            lib().wco_table_destroy(self.h)
            self.h = None

    @property
    def capacity(self):
        return lib().wco_table_capacity(self.h)

    def init(self, seed=DEFAULT_SEED):
        lib().wco_table_init(self.h, int(seed))

    def insert(self, keys, values=None, probing_length=DEFAULT_PROBING_LENGTH,
               want_status=False):
        keys = np.ascontiguousarray(keys)
        if values is not None:
            values = np.ascontiguousarray(values)
        st = np.zeros(len(keys), dtype=np.uint32) if want_status else None
        lib().wco_insert(self.h, _ptr(keys), _ptr(values), len(keys),
                         int(probing_length), _ptr(st))
        return st

    def retrieve(self, keys, out=None, probing_length=DEFAULT_PROBING_LENGTH,
                 want_status=False):
        keys = np.ascontiguousarray(keys)
        if out is None:
            dt = np.uint8 if self.kind == HASHSET else _kdtype(self.value_bytes)
            out = np.zeros(len(keys), dtype=dt)
        st = np.zeros(len(keys), dtype=np.uint32) if want_status else None
        lib().wco_retrieve(self.h, _ptr(keys), len(keys), _ptr(out),
                           int(probing_length), _ptr(st))
        return (out, st) if want_status else out

    def erase(self, keys, probing_length=DEFAULT_PROBING_LENGTH,
              want_status=False):
        keys = np.ascontiguousarray(keys)
        st = np.zeros(len(keys), dtype=np.uint32) if want_status else None
        lib().wco_erase(self.h, _ptr(keys), len(keys), int(probing_length),
                        _ptr(st))
        return st

    def size(self):
        return lib().wco_size(self.h)

    def retrieve_all(self):
        cap = self.capacity
        k = np.empty(cap, dtype=_kdtype(self.key_bytes))
        v = np.empty(cap, dtype=_kdtype(self.value_bytes)) if self.value_bytes else None
        n = lib().wco_retrieve_all(self.h, _ptr(k), _ptr(v))
        return (k[:n], v[:n]) if v is not None else k[:n]

    def peek_status(self):
        return lib().wco_peek_status(self.h)

    def pop_status(self):
        return lib().wco_pop_status(self.h)


class MVTable(Table):
    """Sequential reference-order MultiValueHashTable."""

    def __init__(self, key_bytes, value_bytes, min_capacity, seed=DEFAULT_SEED, cg=8,
                 scheme=PROBE_DOUBLE, h1=HASH_MURMUR, h2=HASH_MURMUR, empty_key=0,
                 tombstone_key=None, max_values_per_key=None):
        if tombstone_key is None:
            tombstone_key = (1 << (8 * key_bytes)) - 1
        if max_values_per_key is None:
            max_values_per_key = 2**64 - 1
        self.kind = MULTIVALUE
        self.key_bytes = key_bytes
        self.value_bytes = value_bytes
        self.h = lib().wco_mv_create(key_bytes, value_bytes, int(min_capacity), int(seed), cg,
                                     scheme, h1, h2, int(empty_key), int(tombstone_key),
                                     int(max_values_per_key))

    def insert(self, keys, values, probing_length=DEFAULT_PROBING_LENGTH, want_status=False):
        keys = np.ascontiguousarray(keys)
        values = np.ascontiguousarray(values)
        st = np.zeros(len(keys), dtype=np.uint32) if want_status else None
        lib().wco_mv_insert(self.h, _ptr(keys), _ptr(values), len(keys), int(probing_length),
                            _ptr(st))
        return st

    def num_values(self, keys, probing_length=DEFAULT_PROBING_LENGTH):
        """(total, per-key counts, statuses)"""
        keys = np.ascontiguousarray(keys)
        c = np.zeros(len(keys), dtype=np.uint64)
        st = np.zeros(len(keys), dtype=np.uint32)
        total = lib().wco_mv_num_values(self.h, _ptr(keys), len(keys), _ptr(c),
                                        int(probing_length), _ptr(st))
        return total, c, st

    def retrieve(self, keys, dry_run=False, probing_length=DEFAULT_PROBING_LENGTH):
        """(begin offsets, end offsets, values, statuses); a dry run gives
        per-key counts in place of end offsets and no values"""
        keys = np.ascontiguousarray(keys)
        n = len(keys)
        b = np.zeros(n, dtype=np.uint64)
        e = np.zeros(n, dtype=np.uint64)
        st = np.zeros(n, dtype=np.uint32)
        total, _, _ = self.num_values(keys, probing_length) if not dry_run else (0, None, None)
        vals = None if dry_run else np.zeros(max(int(total), 1), dtype=_kdtype(self.value_bytes))
        lib().wco_mv_retrieve(self.h, _ptr(keys), n, _ptr(b), _ptr(e), _ptr(vals),
                              int(probing_length), _ptr(st))
        return b, e, (vals[:int(total)] if vals is not None else None), st

    def num_keys(self):
        return lib().wco_mv_num_keys(self.h)

    def unique_keys(self):
        k = np.empty(max(self.capacity, 1), dtype=_kdtype(self.key_bytes))
        n = lib().wco_mv_unique_keys(self.h, _ptr(k))
        return k[:n]


class BLTable:
    """Sequential reference-order BucketListHashTable (BucketListStore with
    index / counter / size bits; default 32 / 20 / 10)."""

    def __init__(self, key_bytes, value_bytes, key_capacity, value_capacity, seed=DEFAULT_SEED,
                 grow_factor=1.1, min_bucket_size=1, max_bucket_size=None,
                 max_values_per_key=None, bits=(32, 20, 10), cg=8):
        ib, cb, sb = bits
        if max_bucket_size is None:
            max_bucket_size = (1 << sb) - 1
        if max_values_per_key is None:
            max_values_per_key = (1 << cb) - 1
        self.key_bytes = key_bytes
        self.value_bytes = value_bytes
        self.value_capacity = value_capacity
        self.h = lib().wco_bl_create(key_bytes, value_bytes, int(key_capacity),
                                     int(value_capacity), int(seed), float(grow_factor),
                                     int(min_bucket_size), int(max_bucket_size),
                                     int(max_values_per_key), ib, cb, sb, cg)
        if not self.h:
            raise ValueError("invalid bucket list configuration")

    def __del__(self):
        if getattr(self, "h", None):
            lib().wco_bl_destroy(self.h)
            self.h = None

    @property
    def key_capacity(self):
        return lib().wco_bl_key_capacity(self.h)

    def init(self, seed=DEFAULT_SEED):
        lib().wco_bl_init(self.h, int(seed))

    def insert(self, keys, values, probing_length=DEFAULT_PROBING_LENGTH, want_status=False,
               status_fill=0):
        """statuses of keys that found no slot keep `status_fill`"""
        keys = np.ascontiguousarray(keys)
        values = np.ascontiguousarray(values)
        st = np.full(len(keys), status_fill, dtype=np.uint32) if want_status else None
        lib().wco_bl_insert(self.h, _ptr(keys), _ptr(values), len(keys), int(probing_length),
                            _ptr(st))
        return st

    def num_values(self, keys, probing_length=DEFAULT_PROBING_LENGTH):
        keys = np.ascontiguousarray(keys)
        c = np.zeros(len(keys), dtype=np.uint64)
        st = np.zeros(len(keys), dtype=np.uint32)
        total = lib().wco_bl_num_values(self.h, _ptr(keys), len(keys), _ptr(c),
                                        int(probing_length), _ptr(st))
        return total, c, st

    def retrieve(self, keys, dry_run=False, probing_length=DEFAULT_PROBING_LENGTH, fill=0):
        """(begin, end, values, statuses); a list whose pool ran out is not
        read, so its part of the values keeps `fill`"""
        keys = np.ascontiguousarray(keys)
        n = len(keys)
        b = np.zeros(n, dtype=np.uint64)
        e = np.zeros(n, dtype=np.uint64)
        st = np.zeros(n, dtype=np.uint32)
        total = 0 if dry_run else self.num_values(keys, probing_length)[0]
        vals = None if dry_run else np.full(max(int(total), 1), fill, dtype=_kdtype(self.value_bytes))
        lib().wco_bl_retrieve(self.h, _ptr(keys), n, _ptr(b), _ptr(e), _ptr(vals),
                              int(probing_length), _ptr(st))
        return b, e, (vals[:int(total)] if vals is not None else None), st

    def num_keys(self):
        return lib().wco_bl_num_keys(self.h)

    def total_values(self):
        return lib().wco_bl_total_values(self.h)

    def next_free(self):
        return lib().wco_bl_next_free(self.h)

    def all_keys(self):
        k = np.empty(max(self.key_capacity, 1), dtype=_kdtype(self.key_bytes))
        n = lib().wco_bl_all_keys(self.h, _ptr(k))
        return k[:n]

    def peek_status(self):
        return lib().wco_bl_peek_status(self.h)

    def pop_status(self):
        return lib().wco_bl_pop_status(self.h)


class MBTable:
    """Sequential reference-order MultiBucketHashTable (bucket <= cg)."""

    def __init__(self, key_bytes, value_bytes, min_capacity, bucket=2, seed=DEFAULT_SEED, cg=8,
                 scheme=PROBE_DOUBLE, h1=HASH_MURMUR, h2=HASH_MURMUR, empty_key=0,
                 tombstone_key=None, empty_value=0, max_values_per_key=None):
        if tombstone_key is None:
            tombstone_key = (1 << (8 * key_bytes)) - 1
        if max_values_per_key is None:
            max_values_per_key = 2**64 - 1
        self.key_bytes = key_bytes
        self.value_bytes = value_bytes
        self.bucket = bucket
        self.h = lib().wco_mb_create(key_bytes, value_bytes, bucket, int(min_capacity), int(seed),
                                     cg, scheme, h1, h2, int(empty_key), int(tombstone_key),
                                     int(empty_value), int(max_values_per_key))
        if not self.h:
            raise ValueError("bucket must be 1 .. cg")

    def __del__(self):
        if getattr(self, "h", None):
            lib().wco_mb_destroy(self.h)
            self.h = None

    @property
    def capacity(self):
        return lib().wco_mb_capacity(self.h)

    def init(self, seed=DEFAULT_SEED):
        lib().wco_mb_init(self.h, int(seed))

    def insert(self, keys, values, probing_length=DEFAULT_PROBING_LENGTH, want_status=False):
        keys = np.ascontiguousarray(keys)
        values = np.ascontiguousarray(values)
        st = np.zeros(len(keys), dtype=np.uint32) if want_status else None
        lib().wco_mb_insert(self.h, _ptr(keys), _ptr(values), len(keys), int(probing_length),
                            _ptr(st))
        return st

    def num_values(self, keys, probing_length=DEFAULT_PROBING_LENGTH):
        """(total, per-key counts, statuses)"""
        keys = np.ascontiguousarray(keys)
        c = np.zeros(len(keys), dtype=np.uint64)
        st = np.zeros(len(keys), dtype=np.uint32)
        total = lib().wco_mb_num_values(self.h, _ptr(keys), len(keys), _ptr(c),
                                        int(probing_length), _ptr(st))
        return total, c, st

    def retrieve(self, keys, dry_run=False, probing_length=DEFAULT_PROBING_LENGTH):
        """(begin offsets, end offsets, values, statuses); a dry run gives
        per-key counts in place of end offsets and no values"""
        keys = np.ascontiguousarray(keys)
        n = len(keys)
        b = np.zeros(n, dtype=np.uint64)
        e = np.zeros(n, dtype=np.uint64)
        st = np.zeros(n, dtype=np.uint32)
        total = 0 if dry_run else self.num_values(keys, probing_length)[0]
        vals = None if dry_run else np.zeros(max(int(total), 1), dtype=_kdtype(self.value_bytes))
        lib().wco_mb_retrieve(self.h, _ptr(keys), n, _ptr(b), _ptr(e), _ptr(vals),
                              int(probing_length), _ptr(st))
        return b, e, (vals[:int(total)] if vals is not None else None), st

    def num_keys(self):
        return lib().wco_mb_num_keys(self.h)

    def num_occupied(self):
        return lib().wco_mb_num_occupied(self.h)

    def size(self):
        return lib().wco_mb_size(self.h)

    def unique_keys(self):
        k = np.empty(max(self.capacity, 1), dtype=_kdtype(self.key_bytes))
        n = lib().wco_mb_unique_keys(self.h, _ptr(k))
        return k[:n]

    def peek_status(self):
        return lib().wco_mb_peek_status(self.h)

    def pop_status(self):
        return lib().wco_mb_pop_status(self.h)


class Bloom:
    def __init__(self, num_bits, k, seed=DEFAULT_SEED, key_bytes=8,
                 slot_bytes=8, cg=1, hasher=HASH_MURMUR):
        self.key_bytes = key_bytes
        self.h = lib().wco_bloom_create(key_bytes, slot_bytes, cg, hasher,
                                        int(num_bits), int(k), int(seed))
        self.slot_bytes = slot_bytes

    def __del__(self):
        if getattr(self, "h", None):
            lib().wco_bloom_destroy(self.h)
            self.h = None

    @property
    def num_slots(self):
        return lib().wco_bloom_num_slots(self.h)

    @property
    def num_blocks(self):
        return lib().wco_bloom_num_blocks(self.h)

    def insert(self, keys):
        keys = np.ascontiguousarray(keys)
        lib().wco_bloom_insert(self.h, _ptr(keys), len(keys))

    def retrieve(self, keys):
        keys = np.ascontiguousarray(keys)
        out = np.zeros(len(keys), dtype=np.uint8)
        lib().wco_bloom_retrieve(self.h, _ptr(keys), len(keys), _ptr(out))
        return out

    def words(self):
        out = np.empty(self.num_slots, dtype=np.uint64)
        lib().wco_bloom_words(self.h, _ptr(out))
        return out.astype(np.uint32) if self.slot_bytes == 4 else out

    def fpr(self, n):
        return lib().wco_bloom_fpr(self.h, int(n))


class MTTable:
    """Multi-threaded CPU port of the reference insert/retrieve (timed)."""

    def __init__(self, key_bytes, capacity, cg=8, seed=DEFAULT_SEED):
        self.key_bytes = key_bytes
        self.h = lib().wco_mt_create(key_bytes, key_bytes, int(capacity), cg,
                                     int(seed))

    def __del__(self):
        if getattr(self, "h", None):
            lib().wco_mt_destroy(self.h)
            self.h = None

    def clear(self, threads):
        lib().wco_mt_clear(self.h, threads)

    def insert(self, keys, values, threads):
        return lib().wco_mt_insert(self.h, _ptr(keys), _ptr(values), len(keys),
                                   threads)

    def retrieve(self, keys, out, found, threads):
        return lib().wco_mt_retrieve(self.h, _ptr(keys), len(keys), _ptr(out),
                                     _ptr(found), threads)
