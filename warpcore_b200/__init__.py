"""warpcore_b200 -- B200-native GPU hash tables and Bloom filter.

Python binding of the C ABI in ``include/warpcore_b200.h`` (ctypes).  The
classes mirror the reference's C++ class templates (warpcore's
``SingleValueHashTable``, ``HashSet``, ``CountingHashTable`` and
``BloomFilter``): same constructor arguments, same bulk methods on device
buffers, same ``Status`` flags.  Buffers are CUDA tensors (any 4- or 8-byte
dtype; bits are read as unsigned integers); ``stream`` is a
``torch.cuda.Stream`` or a raw ``cudaStream_t`` integer and defaults to the
current torch stream.

There is no CPU fallback: importing works without a GPU, but every table
operation needs the compiled ``libwarpcore_b200.so`` and a CUDA device, and
raises otherwise.
"""
import ctypes
import os

from ._status import Status  # noqa: F401

__all__ = [
    "Status", "SingleValueHashTable", "HashSet", "CountingHashTable", "MultiValueHashTable",
    "MultiBucketHashTable", "BucketListHashTable",
    "BloomFilter", "lib", "valid_capacity", "WarpcoreError", "set_l2_persistence",
    "HostPipe", "set_fingerprint_policy", "set_fingerprint_ops", "launch_count",
    "gen_uniform", "gen_unique", "gen_zipf", "FINGERPRINTS_AUTO", "FINGERPRINTS_ALWAYS",
    "FINGERPRINTS_NEVER",
    "HASH_MURMUR", "HASH_NVIDIA", "HASH_MUELLER", "HASH_IDENTITY32",
    "HASH_IDENTITY64", "PROBING_DOUBLE", "PROBING_LINEAR",
    "PROBING_QUADRATIC", "HANDLER_NOTHING", "HANDLER_STATUS",
    "HANDLER_BOOLEAN", "DEFAULT_SEED", "DEFAULT_PROBING_LENGTH", "Batch",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
# WARPCORE_B200_LIB may point at another build of the same library
LIB_PATH = os.environ.get("WARPCORE_B200_LIB") or os.path.join(_HERE, "libwarpcore_b200.so")

HASH_MURMUR, HASH_NVIDIA, HASH_MUELLER, HASH_IDENTITY32, HASH_IDENTITY64 = range(5)
PROBING_DOUBLE, PROBING_LINEAR, PROBING_QUADRATIC = range(3)
HANDLER_NOTHING, HANDLER_STATUS, HANDLER_BOOLEAN = range(3)

# defaults.cuh:21 (seed) and :27 (probing length)
DEFAULT_SEED = 0x5AD0DED
DEFAULT_PROBING_LENGTH = (2**64 - 1) - 1024


class WarpcoreError(RuntimeError):
    pass


class TableConfig(ctypes.Structure):
    _fields_ = [
        ("key_bytes", ctypes.c_uint32),
        ("value_bytes", ctypes.c_uint32),
        ("empty_key", ctypes.c_uint64),
        ("tombstone_key", ctypes.c_uint64),
        ("probing", ctypes.c_uint32),
        ("hasher1", ctypes.c_uint32),
        ("hasher2", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
    ]


class BlInfo(ctypes.Structure):
    _fields_ = [
        ("key_bytes", ctypes.c_uint32),
        ("value_bytes", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
        ("probing", ctypes.c_uint32),
        ("hasher1", ctypes.c_uint32),
        ("hasher2", ctypes.c_uint32),
        ("index_bits", ctypes.c_uint32),
        ("counter_bits", ctypes.c_uint32),
        ("size_bits", ctypes.c_uint32),
        ("grow_factor", ctypes.c_float),
        ("key_capacity", ctypes.c_uint64),
        ("value_capacity", ctypes.c_uint64),
        ("num_buckets", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("empty_key", ctypes.c_uint64),
        ("tombstone_key", ctypes.c_uint64),
        ("min_bucket_size", ctypes.c_uint64),
        ("max_bucket_size", ctypes.c_uint64),
        ("max_values_per_key", ctypes.c_uint64),
        ("bytes_total", ctypes.c_uint64),
        ("keys", ctypes.c_void_p),
        ("handles", ctypes.c_void_p),
        ("pool", ctypes.c_void_p),
        ("next_free", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("is_initialized", ctypes.c_int),
    ]


class MbInfo(ctypes.Structure):
    _fields_ = [
        ("key_bytes", ctypes.c_uint32),
        ("value_bytes", ctypes.c_uint32),
        ("bucket_size", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
        ("probing", ctypes.c_uint32),
        ("hasher1", ctypes.c_uint32),
        ("hasher2", ctypes.c_uint32),
        ("capacity", ctypes.c_uint64),
        ("value_capacity", ctypes.c_uint64),
        ("num_buckets", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("empty_key", ctypes.c_uint64),
        ("tombstone_key", ctypes.c_uint64),
        ("empty_value", ctypes.c_uint64),
        ("max_values_per_key", ctypes.c_uint64),
        ("bytes_total", ctypes.c_uint64),
        ("keys", ctypes.c_void_p),
        ("values", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("num_keys", ctypes.c_void_p),
        ("num_occupied", ctypes.c_void_p),
        ("is_initialized", ctypes.c_int),
    ]


class TableInfo(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("key_bytes", ctypes.c_uint32),
        ("value_bytes", ctypes.c_uint32),
        ("slot_bytes", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
        ("probing", ctypes.c_uint32),
        ("hasher1", ctypes.c_uint32),
        ("hasher2", ctypes.c_uint32),
        ("capacity", ctypes.c_uint64),
        ("num_buckets", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("empty_key", ctypes.c_uint64),
        ("tombstone_key", ctypes.c_uint64),
        ("max_count", ctypes.c_uint64),
        ("bytes_total", ctypes.c_uint64),
        ("slots", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("is_initialized", ctypes.c_int),
        ("fingerprints", ctypes.c_void_p),
        ("num_keys", ctypes.c_void_p),
        ("max_values_per_key", ctypes.c_uint64),
        ("live", ctypes.c_void_p),
        ("values", ctypes.c_void_p),
    ]


class BloomConfig(ctypes.Structure):
    _fields_ = [
        ("key_bytes", ctypes.c_uint32),
        ("slot_bytes", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
        ("hasher", ctypes.c_uint32),
    ]


class BloomInfo(ctypes.Structure):
    _fields_ = [
        ("key_bytes", ctypes.c_uint32),
        ("slot_bytes", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
        ("hasher", ctypes.c_uint32),
        ("num_bits", ctypes.c_uint64),
        ("num_slots", ctypes.c_uint64),
        ("num_blocks", ctypes.c_uint64),
        ("k", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("words", ctypes.c_void_p),
        ("block_base", ctypes.c_uint64),
        ("local_blocks", ctypes.c_uint64),
    ]


class BatchRequest(ctypes.Structure):
    _fields_ = [
        ("table", ctypes.c_void_p),
        ("op", ctypes.c_int),
        ("status_handler", ctypes.c_int),
        ("ignore", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("keys", ctypes.c_void_p),
        ("values", ctypes.c_void_p),
        ("values_out", ctypes.c_void_p),
        ("status_out", ctypes.c_void_p),
        ("num", ctypes.c_uint64),
    ]


class ServeRequest(ctypes.Structure):
    _fields_ = [
        ("arrival_us", ctypes.c_double),
        ("table", ctypes.c_void_p),
        ("table_id", ctypes.c_uint64),
        ("op", ctypes.c_int),
        ("reserved", ctypes.c_int),
        ("keys", ctypes.c_void_p),
        ("values", ctypes.c_void_p),
        ("values_out", ctypes.c_void_p),
        ("num", ctypes.c_uint64),
    ]


class ServeOptions(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int),
        ("streams", ctypes.c_uint32),
        ("depth", ctypes.c_uint32),
        ("max_batch_requests", ctypes.c_uint32),
        ("max_batch_keys", ctypes.c_uint64),
        ("blocks_per_sm", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("probing_length", ctypes.c_uint64),
        ("pool", ctypes.c_void_p),
    ]


class TablePoolStats(ctypes.Structure):
    _fields_ = [
        ("admissions", ctypes.c_uint64),
        ("restores", ctypes.c_uint64),
        ("evictions", ctypes.c_uint64),
        ("waits", ctypes.c_uint64),
        ("peak_bytes", ctypes.c_uint64),
        ("resident_bytes", ctypes.c_uint64),
        ("resident_tables", ctypes.c_uint64),
    ]


class ServeStats(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("max_keys_in_batch", ctypes.c_uint64),
        ("host_wall_us", ctypes.c_double),
        ("gpu_batch_us", ctypes.c_double),
        ("host_launch_us", ctypes.c_double),
    ]


class PServerOptions(ctypes.Structure):
    _fields_ = [
        ("key_bytes", ctypes.c_uint32),
        ("cg_size", ctypes.c_uint32),
        ("blocks_per_sm", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("chunk_keys", ctypes.c_uint64),
        ("idle_timeout_us", ctypes.c_uint64),
        ("probing_length", ctypes.c_uint64),
    ]


OP_INSERT, OP_RETRIEVE = 0, 2
SERVE_PLAIN, SERVE_BATCHED, SERVE_PERSISTENT = 0, 1, 2
ERR_TIMEOUT = -6

_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_i = ctypes.c_int
_pp = ctypes.POINTER(ctypes.c_void_p)

# every symbol the C header declares, with its signature
SIGNATURES = {
    "wc_last_error": (ctypes.c_char_p, []),
    "wc_version": (ctypes.c_char_p, []),
    "wc_svht_default_config": (None, [ctypes.POINTER(TableConfig), _u32, _u32]),
    "wc_hashset_default_config": (None, [ctypes.POINTER(TableConfig), _u32]),
    "wc_counting_default_config": (None, [ctypes.POINTER(TableConfig), _u32, _u32]),
    "wc_valid_capacity": (_u64, [_u64, _u64]),
    "wc_svht_create": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _i, _pp]),
    "wc_svht_create_soa": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _i, _pp]),
    "wc_table_destroy": (_i, [_vp]),
    "wc_table_init": (_i, [_vp, _u64, _vp]),
    "wc_svht_insert": (_i, [_vp, _vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_svht_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp, _u64, _vp, _i, _u32]),
    "wc_svht_erase": (_i, [_vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_table_size": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_table_size_scan": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_table_retrieve_all": (_i, [_vp, _vp, _vp, ctypes.POINTER(_u64), _vp]),
    "wc_table_peek_status": (_i, [_vp, _vp, ctypes.POINTER(_u32)]),
    "wc_table_pop_status": (_i, [_vp, _vp, ctypes.POINTER(_u32)]),
    "wc_table_get_info": (_i, [_vp, ctypes.POINTER(TableInfo)]),
    "wc_hashset_create": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _pp]),
    "wc_hashset_insert": (_i, [_vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_hashset_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp, _u64, _vp, _i, _u32]),
    "wc_hashset_erase": (_i, [_vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_counting_create": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _u64, _i, _pp]),
    "wc_counting_insert": (_i, [_vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_counting_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp, _u64, _vp, _i, _u32]),
    "wc_counting_erase": (_i, [_vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_bloom_create": (_i, [ctypes.POINTER(BloomConfig), _u64, _u64, _u64, _pp]),
    "wc_bloom_create_shard": (_i, [ctypes.POINTER(BloomConfig), _u64, _u64, _u64, _u32, _u32, _pp]),
    "wc_bloom_partition": (_i, [_vp, _vp, _u64, _u32, _vp, _vp, _vp, _vp, _vp]),
    "wc_bloom_destroy": (_i, [_vp]),
    "wc_bloom_init": (_i, [_vp, _u64, _vp]),
    "wc_bloom_insert": (_i, [_vp, _vp, _u64, _vp]),
    "wc_bloom_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp]),
    "wc_bloom_get_info": (_i, [_vp, ctypes.POINTER(BloomInfo)]),
    "wc_bloom_fpr": (_i, [_vp, _u64, ctypes.POINTER(ctypes.c_double)]),
    "wc_slots_size_noalloc": (_i, [_vp, _u64, _u32, _u32, _u64, _u64, _vp, _vp]),
    "wc_partition": (_i, [_vp, _vp, _u64, _u32, _u32, _u32, _u64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "wc_partition_restore": (_i, [_vp, _vp, _vp, _u64, _u32, _vp, _vp, _vp]),
    "wc_host_pipe_create": (_i, [_u64, _u32, _pp]),
    "wc_host_pipe_destroy": (_i, [_vp]),
    "wc_table_insert_host": (_i, [_vp, _vp, _vp, _vp, _u64, _vp, _u64]),
    "wc_table_retrieve_host": (_i, [_vp, _vp, _vp, _u64, _vp, _vp, _vp, _u64]),
    "wc_l2_persistence": (_i, [_i, ctypes.POINTER(ctypes.c_int)]),
    "wc_region_bytes": (_i, [_i, _u64, ctypes.POINTER(ctypes.c_uint64)]),
    "wc_lane_ops": (_i, [_u32, ctypes.POINTER(ctypes.c_uint32)]),
    "wc_fingerprint_policy": (_i, [_i, ctypes.POINTER(ctypes.c_int)]),
    "wc_fingerprint_ops": (_i, [_u32, ctypes.POINTER(ctypes.c_uint32)]),
    "wc_launch_count": (_i, [ctypes.POINTER(_u64)]),
    "wc_gen_uniform": (_i, [_vp, _u64, _u32, _u64, _vp]),
    "wc_gen_unique": (_i, [_vp, _u64, _u32, _u64, _vp]),
    "wc_gen_zipf": (_i, [_vp, _u64, _vp, _u64, _u32, ctypes.c_double, _u64, _vp]),
    "wc_mvht_create": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _u64, _i, _pp]),
    "wc_mvht_insert": (_i, [_vp, _vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_mvht_num_values": (_i, [_vp, _vp, _u64, ctypes.POINTER(_u64), _vp, _vp, _u64, _vp, _i, _u32]),
    "wc_mvht_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp, _vp, ctypes.POINTER(_u64), _vp, _u64, _vp,
                              _i, _u32]),
    "wc_mvht_retrieve_all_keys": (_i, [_vp, _vp, ctypes.POINTER(_u64), _vp]),
    "wc_mvht_num_keys": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_blht_create": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _u64, ctypes.c_float, _u64,
                            _u64, _u64, _u32, _u32, _u32, _i, _pp]),
    "wc_blht_destroy": (_i, [_vp]),
    "wc_blht_init": (_i, [_vp, _u64, _vp]),
    "wc_blht_insert": (_i, [_vp, _vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_blht_num_values": (_i, [_vp, _vp, _u64, ctypes.POINTER(_u64), _vp, _vp, _u64, _vp, _i, _u32]),
    "wc_blht_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp, _vp, ctypes.POINTER(_u64), _vp, _u64, _vp,
                              _i, _u32]),
    "wc_blht_retrieve_all_keys": (_i, [_vp, _vp, ctypes.POINTER(_u64), _vp]),
    "wc_blht_num_keys": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_blht_total_values": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_blht_pool_used": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_blht_peek_status": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32)]),
    "wc_blht_pop_status": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32)]),
    "wc_blht_get_info": (_i, [_vp, ctypes.POINTER(BlInfo)]),
    "wc_mbht_create": (_i, [ctypes.POINTER(TableConfig), _u32, _u64, _u64, _u64, _u64, _i, _pp]),
    "wc_mbht_destroy": (_i, [_vp]),
    "wc_mbht_init": (_i, [_vp, _vp]),
    "wc_mbht_insert": (_i, [_vp, _vp, _vp, _u64, _vp, _u64, _vp, _i, _u32]),
    "wc_mbht_num_values": (_i, [_vp, _vp, _u64, ctypes.POINTER(_u64), _vp, _vp, _u64, _vp, _i, _u32]),
    "wc_mbht_retrieve": (_i, [_vp, _vp, _u64, _vp, _vp, _vp, ctypes.POINTER(_u64), _vp, _u64, _vp,
                              _i, _u32]),
    "wc_mbht_retrieve_all_keys": (_i, [_vp, _vp, ctypes.POINTER(_u64), _vp]),
    "wc_mbht_num_keys": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_mbht_num_occupied": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_mbht_size": (_i, [_vp, _vp, ctypes.POINTER(_u64)]),
    "wc_mbht_peek_status": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32)]),
    "wc_mbht_pop_status": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32)]),
    "wc_mbht_get_info": (_i, [_vp, ctypes.POINTER(MbInfo)]),
    "wc_table_l2_window": (_i, [_vp, ctypes.POINTER(_u64), ctypes.POINTER(ctypes.c_float)]),
    "wc_tune_set": (_i, [_u32, _i, _u32, _u32, _u32, _u32]),
    "wc_tune_reset": (_i, []),
    "wc_tune_load": (_i, [ctypes.c_char_p, ctypes.POINTER(_u64)]),
    "wc_batch_create": (_i, [_u32, _u32, _pp]),
    "wc_batch_destroy": (_i, [_vp]),
    "wc_batch_run": (_i, [_vp, ctypes.POINTER(BatchRequest), _u32, _vp, _u64, _u32]),
    "wc_serve_run": (_i, [ctypes.POINTER(ServeRequest), _u64, ctypes.POINTER(ServeOptions),
                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                          ctypes.POINTER(ServeStats)]),
    "wc_pserver_start": (_i, [ctypes.POINTER(PServerOptions), _vp, _pp]),
    "wc_pserver_submit": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _u64, ctypes.POINTER(_u64)]),
    "wc_pserver_poll": (_i, [_vp, _u64, ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_double)]),
    "wc_pserver_now_us": (_i, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "wc_pserver_stop": (_i, [_vp]),
    "wc_table_pool_create": (_i, [_u64, _pp]),
    "wc_table_pool_add": (_i, [_vp, ctypes.POINTER(TableConfig), _u64, _u64, ctypes.POINTER(_u64)]),
    "wc_table_pool_table": (_i, [_vp, _u64, _pp]),
    "wc_table_pool_get_stats": (_i, [_vp, ctypes.POINTER(TablePoolStats)]),
    "wc_table_pool_destroy": (_i, [_vp]),
    "wc_svht_memory_bytes": (_i, [ctypes.POINTER(TableConfig), _u64, ctypes.POINTER(_u64)]),
    "wc_svht_create_on": (_i, [ctypes.POINTER(TableConfig), _u64, _u64, _i, _vp, _u64, _vp, _pp]),
}

_lib = None


def lib():
    """Load libwarpcore_b200.so (built in-tree by warpcore_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise WarpcoreError(
                "libwarpcore_b200.so is missing; build it with "
                "`python -m warpcore_b200.build` (nvcc, sm_100a)")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
        _load_tuning(l)
        if os.environ.get("WARPCORE_B200_L2_PERSIST", "1") == "0":
            l.wc_l2_persistence(0, None)

    return _lib


def _load_tuning(l):
    """launch geometry measured by warpcore_b200.autotune (tuning_b200.json),
    loaded by the library itself (wc_tune_load), as the C++ headers do"""
    path = os.environ.get("WARPCORE_B200_TUNING") or os.path.join(_HERE, "tuning_b200.json")
    if path == "none" or not os.path.exists(path):
        return
    n = ctypes.c_uint64(0)
    l.wc_tune_load(path.encode(), ctypes.byref(n))


def wc_svht_default_config_py(key_bytes, value_bytes):
    """wc_svht_default_config as a TableConfig"""
    cfg = TableConfig()
    lib().wc_svht_default_config(ctypes.byref(cfg), int(key_bytes), int(value_bytes))
    return cfg


def _check(rc):
    if rc != 0:
        raise WarpcoreError("warpcore_b200 error %d: %s"
                            % (rc, lib().wc_last_error().decode()))


def valid_capacity(min_capacity, cg_size):
    """The reference's capacity rule (base.cuh:27-34)."""
    return lib().wc_valid_capacity(int(min_capacity), int(cg_size))


FINGERPRINTS_AUTO, FINGERPRINTS_ALWAYS, FINGERPRINTS_NEVER = 0, 1, 2
_FP_NAMES = {"auto": FINGERPRINTS_AUTO, "always": FINGERPRINTS_ALWAYS, "never": FINGERPRINTS_NEVER}


def set_fingerprint_policy(mode):
    """Which tables created from now on keep one fingerprint byte per slot:
    "auto" (slot arrays larger than L2), "always" or "never" (or the
    FINGERPRINTS_* constants); returns the previous mode as a constant."""
    m = _FP_NAMES[mode] if isinstance(mode, str) else int(mode)
    prev = ctypes.c_int(0)
    _check(lib().wc_fingerprint_policy(m, ctypes.byref(prev)))
    return prev.value


def set_lane_ops(op_mask):
    """Operations (bit 0 insert, 2 retrieve, 3 erase) whose whole-window
    probing reads one key's window per lane (wc_lane_ops); returns the
    previous mask"""
    prev = ctypes.c_uint32(0)
    _check(lib().wc_lane_ops(int(op_mask), ctypes.byref(prev)))
    return prev.value


def set_region_bytes(nbytes, op=None):
    """Random-access region of the multi-pass kernels: a Bloom filter
    larger than this is inserted into (op "insert") or queried (op "query")
    in passes, one region of its blocks per pass (default 256 MiB for both);
    0 = always one pass.  `nbytes` is one value for both, or a
    pair (insert, query); op=None sets both.  Returns the previous value(s)
    in the same form."""
    ops = {"insert": 0, "query": 1}
    if op is not None:
        prev = ctypes.c_uint64(0)
        _check(lib().wc_region_bytes(ops[op], int(nbytes), ctypes.byref(prev)))
        return prev.value
    vals = nbytes if isinstance(nbytes, (tuple, list)) else (nbytes, nbytes)
    return tuple(set_region_bytes(v, o) for v, o in zip(vals, ("insert", "query")))


def gen_uniform(out, seed, stream=None):
    """fill a 4- or 8-byte CUDA tensor with uniform words
    (random_distributions.cuh:50-137); element i depends only on (seed, i)"""
    _check(lib().wc_gen_uniform(_ptr(out), out.numel(), out.element_size(), int(seed),
                                _stream(stream)))
    return out


def gen_unique(out, seed, stream=None):
    """fill a 4- or 8-byte CUDA tensor with distinct keys, none equal to 0 or
    all ones (random_distributions.cuh:144-251)"""
    _check(lib().wc_gen_unique(_ptr(out), out.numel(), out.element_size(), int(seed),
                               _stream(stream)))
    return out


def gen_zipf(out, n_in, s, seed, in_=None, stream=None):
    """fill `out` with Zipf(s) draws over ranks 1..n_in
    (random_distributions.cuh:259-326): in_[rank - 1], or the rank itself"""
    if in_ is not None:
        _check_width(in_, out.element_size(), "in_")
    _check(lib().wc_gen_zipf(_ptr(in_), int(n_in), _ptr(out), out.numel(), out.element_size(),
                             float(s), int(seed), _stream(stream)))
    return out


def launch_count():
    """kernels this library has launched in this process"""
    out = _u64(0)
    _check(lib().wc_launch_count(ctypes.byref(out)))
    return int(out.value)


def set_fingerprint_ops(op_mask):
    """bit mask of operations (1 insert, 2 counting insert, 4 retrieve,
    8 erase) that read fingerprints first; returns the previous mask"""
    prev = ctypes.c_uint32(0)
    _check(lib().wc_fingerprint_ops(int(op_mask), ctypes.byref(prev)))
    return prev.value


def set_l2_persistence(enable):
    """Turn the L2 access-policy windows of tables that fit in L2 on or off
    for later launches; returns the previous setting."""
    prev = ctypes.c_int(0)
    _check(lib().wc_l2_persistence(int(bool(enable)), ctypes.byref(prev)))
    return bool(prev.value)


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise WarpcoreError("buffers must be CUDA tensors (device memory)")
    if not t.is_contiguous():
        raise WarpcoreError("buffers must be contiguous")
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _check_width(t, nbytes, what):
    if t is not None and not isinstance(t, int) and t.element_size() != nbytes:
        raise WarpcoreError("%s must have %d-byte elements, got %s"
                            % (what, nbytes, t.dtype))


def _host_ptr(t):
    if t is None:
        return None
    if t.is_cuda:
        raise WarpcoreError("host-pipe buffers must be CPU tensors")
    if not t.is_contiguous():
        raise WarpcoreError("buffers must be contiguous")
    return t.data_ptr()


def _numel(t, n):
    if n is not None:
        return int(n)
    return t.numel()


class _Table:
    _kind = None

    def _make(self, create, cfg, *args):
        h = ctypes.c_void_p()
        _check(create(ctypes.byref(cfg), *args, ctypes.byref(h)))
        self._h = h
        self._cfg = cfg

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.wc_table_destroy(h)
            self._h = None

    def info(self):
        inf = TableInfo()
        _check(lib().wc_table_get_info(self._h, ctypes.byref(inf)))
        return inf

    def insert_from_host(self, pipe, keys_in, values_in=None, num_in=None, stream=None,
                         probing_length=DEFAULT_PROBING_LENGTH):
        """insert from CPU tensors (pinned for overlap) through a HostPipe;
        values_in for single-value tables only"""
        _check(lib().wc_table_insert_host(pipe._h, self._h, _host_ptr(keys_in),
                                          _host_ptr(values_in), _numel(keys_in, num_in),
                                          _stream(stream), int(probing_length)))

    def retrieve_to_host(self, pipe, keys_in, out, num_in=None, miss_fill=None, stream=None,
                         probing_length=DEFAULT_PROBING_LENGTH):
        """retrieve into a CPU tensor through a HostPipe; complete when
        `stream` passes the call.  Single-value and counting tables write
        hits only: a miss keeps `out`'s content, or gets `miss_fill`"""
        fill = None
        if miss_fill is not None:
            fill = (ctypes.c_uint64 if out.element_size() == 8 else ctypes.c_uint32)(
                int(miss_fill) & ((1 << (8 * out.element_size())) - 1))
        _check(lib().wc_table_retrieve_host(pipe._h, self._h, _host_ptr(keys_in),
                                            _numel(keys_in, num_in), _host_ptr(out),
                                            ctypes.byref(fill) if fill is not None else None,
                                            _stream(stream), int(probing_length)))

    @property
    def capacity(self):
        return self.info().capacity

    def bytes_total(self):
        return self.info().bytes_total

    @property
    def seed(self):
        return self.info().seed

    def is_initialized(self):
        return bool(self.info().is_initialized)

    @property
    def key_bytes(self):
        return self._cfg.key_bytes

    def cg_size(self):
        return self._cfg.cg_size

    def init(self, seed=None, stream=None):
        _check(lib().wc_table_init(self._h, int(self.seed if seed is None else seed),
                                   _stream(stream)))

    def size(self, stream=None):
        """valid keys: the count claims and erases maintain (one small read)"""
        out = _u64()
        _check(lib().wc_table_size(self._h, _stream(stream), ctypes.byref(out)))
        return out.value

    def size_scan(self, stream=None):
        """valid keys counted by a scan of the slot array"""
        out = _u64()
        _check(lib().wc_table_size_scan(self._h, _stream(stream), ctypes.byref(out)))
        return out.value

    @property
    def has_fingerprints(self):
        return bool(self.info().fingerprints)

    def l2_window(self):
        """(bytes, hit ratio) of the L2 persistence window this table's
        launches use; (0, 0.0) when it has none"""
        b, r = _u64(0), ctypes.c_float(0.0)
        _check(lib().wc_table_l2_window(self._h, ctypes.byref(b), ctypes.byref(r)))
        return int(b.value), float(r.value)

    def load_factor(self, stream=None):
        return float(self.size(stream)) / float(self.capacity)

    def storage_density(self, stream=None):
        return self.load_factor(stream)

    def peek_status(self, stream=None):
        out = _u32()
        _check(lib().wc_table_peek_status(self._h, _stream(stream), ctypes.byref(out)))
        return Status(out.value)

    def pop_status(self, stream=None):
        out = _u32()
        _check(lib().wc_table_pop_status(self._h, _stream(stream), ctypes.byref(out)))
        return Status(out.value)

    def retrieve_all(self, keys_out, values_out=None, stream=None):
        """Dump all valid (key, value) pairs; returns the count (blocking)."""
        _check_width(keys_out, self.key_bytes, "keys_out")
        n = _u64()
        _check(lib().wc_table_retrieve_all(self._h, _ptr(keys_out), _ptr(values_out),
                                           ctypes.byref(n), _stream(stream)))
        return n.value


def _table_config(default_fn, key_bytes, value_bytes, empty_key, tombstone_key,
                  probing, hasher1, hasher2, cg_size):
    cfg = TableConfig()
    if value_bytes is None:
        default_fn(ctypes.byref(cfg), key_bytes)
    else:
        default_fn(ctypes.byref(cfg), key_bytes, value_bytes)
    if empty_key is not None:
        cfg.empty_key = empty_key
    if tombstone_key is not None:
        cfg.tombstone_key = tombstone_key
    if probing is not None:
        cfg.probing = probing
    if hasher1 is not None:
        cfg.hasher1 = hasher1
    if hasher2 is not None:
        cfg.hasher2 = hasher2
    if cg_size is not None:
        cfg.cg_size = cg_size
    return cfg


class SingleValueHashTable(_Table):
    """warpcore::SingleValueHashTable (single_value_hash_table.cuh:29-37).

    store="aos" (default) keeps {key, value} slots; store="soa" keeps the
    keys in the slot array and the values in a separate array
    (storage::key_value::SoAStore, storage.cuh:218-432), with the same
    answers (wc_svht_create_soa)."""

    def __init__(self, min_capacity, seed=DEFAULT_SEED, no_init=False, key_bytes=4,
                 value_bytes=None, empty_key=None, tombstone_key=None, probing=None,
                 hasher1=None, hasher2=None, cg_size=None, store="aos"):
        if store not in ("aos", "soa"):
            raise WarpcoreError("store must be 'aos' or 'soa'")
        value_bytes = key_bytes if value_bytes is None else value_bytes
        cfg = _table_config(lib().wc_svht_default_config, key_bytes, value_bytes, empty_key,
                            tombstone_key, probing, hasher1, hasher2, cg_size)
        create = lib().wc_svht_create_soa if store == "soa" else lib().wc_svht_create
        self._make(create, cfg, int(min_capacity), int(seed), int(bool(no_init)))
        self.store = store

    def insert(self, keys_in, values_in, num_in=None, stream=None,
               probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
               status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(values_in, self._cfg.value_bytes, "values_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_svht_insert(self._h, _ptr(keys_in), _ptr(values_in),
                                    _numel(keys_in, num_in), _stream(stream),
                                    int(probing_length), _ptr(status_out), h, int(ignore)))

    def retrieve(self, keys_in, values_out, num_in=None, stream=None,
                 probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
                 status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(values_out, self._cfg.value_bytes, "values_out")
        h = _handler(status_out, status_handler)
        _check(lib().wc_svht_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                      _ptr(values_out), _stream(stream), int(probing_length),
                                      _ptr(status_out), h, int(ignore)))

    def erase(self, keys_in, num_in=None, stream=None,
              probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
              status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_svht_erase(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                   _stream(stream), int(probing_length), _ptr(status_out),
                                   h, int(ignore)))


class MultiValueHashTable(_Table):
    """warpcore::MultiValueHashTable (multi_value_hash_table.cuh:18-27): every
    (key, value) pair takes a slot of its own; retrieve returns each key's
    values in insertion order with begin/end offsets."""

    def __init__(self, min_capacity, seed=DEFAULT_SEED, max_values_per_key=2**64 - 1,
                 no_init=False, key_bytes=4, value_bytes=None, empty_key=None,
                 tombstone_key=None, probing=None, hasher1=None, hasher2=None, cg_size=None):
        value_bytes = key_bytes if value_bytes is None else value_bytes
        cfg = _table_config(lib().wc_svht_default_config, key_bytes, value_bytes, empty_key,
                            tombstone_key, probing, hasher1, hasher2, cg_size)
        self._make(lib().wc_mvht_create, cfg, int(min_capacity), int(seed),
                   int(max_values_per_key), int(bool(no_init)))

    def insert(self, keys_in, values_in, num_in=None, stream=None,
               probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
               status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(values_in, self._cfg.value_bytes, "values_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_mvht_insert(self._h, _ptr(keys_in), _ptr(values_in),
                                    _numel(keys_in, num_in), _stream(stream),
                                    int(probing_length), _ptr(status_out), h, int(ignore)))

    def num_values(self, keys_in, num_per_key_out=None, num_in=None, stream=None,
                   probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
                   status_handler=None, ignore=0):
        """values per key (uint64 tensor, optional); returns their sum"""
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        out = _u64(0)
        _check(lib().wc_mvht_num_values(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                        ctypes.byref(out), _ptr(num_per_key_out),
                                        _stream(stream), int(probing_length), _ptr(status_out),
                                        h, int(ignore)))
        return int(out.value)

    def retrieve(self, keys_in, begin_offsets_out, end_offsets_out, values_out=None,
                 num_in=None, stream=None, probing_length=DEFAULT_PROBING_LENGTH,
                 status_out=None, status_handler=None, ignore=0):
        """values_out None: dry run (end_offsets_out gets the counts);
        returns the total number of values"""
        _check_width(keys_in, self.key_bytes, "keys_in")
        if values_out is not None:
            _check_width(values_out, self._cfg.value_bytes, "values_out")
        h = _handler(status_out, status_handler)
        out = _u64(0)
        _check(lib().wc_mvht_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                      _ptr(begin_offsets_out), _ptr(end_offsets_out),
                                      _ptr(values_out), ctypes.byref(out), _stream(stream),
                                      int(probing_length), _ptr(status_out), h, int(ignore)))
        return int(out.value)

    def retrieve_all_keys(self, keys_out=None, stream=None):
        """each stored key once; keys_out None: only the count"""
        out = _u64(0)
        _check(lib().wc_mvht_retrieve_all_keys(self._h, _ptr(keys_out), ctypes.byref(out),
                                               _stream(stream)))
        return int(out.value)

    def num_keys(self, stream=None):
        out = _u64(0)
        _check(lib().wc_mvht_num_keys(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)


class BucketListHashTable:
    """warpcore::BucketListHashTable (bucket_list_hash_table.cuh:17-121) over
    BucketListStore<Value, index_bits, counter_bits, size_bits>: each key
    holds a list of value buckets in a pool of `value_capacity` elements;
    the first bucket has `min_bucket_size` values, each later one
    ceil(previous * grow_factor), at most `max_bucket_size`.  retrieve
    returns each key's values newest bucket first, with begin/end offsets."""

    def __init__(self, key_capacity, value_capacity, seed=DEFAULT_SEED, grow_factor=1.1,
                 min_bucket_size=1, max_bucket_size=None, max_values_per_key=None,
                 no_init=False, key_bytes=4, value_bytes=None, bits=(32, 20, 10),
                 empty_key=None, tombstone_key=None, probing=None, hasher1=None, hasher2=None,
                 cg_size=None):
        value_bytes = key_bytes if value_bytes is None else value_bytes
        ib, cb, sb = bits
        if max_bucket_size is None:
            max_bucket_size = (1 << sb) - 1
        if max_values_per_key is None:
            max_values_per_key = (1 << cb) - 1
        cfg = _table_config(lib().wc_svht_default_config, key_bytes, key_bytes, empty_key,
                            tombstone_key, probing, hasher1, hasher2, cg_size)
        cfg.value_bytes = value_bytes
        h = ctypes.c_void_p()
        _check(lib().wc_blht_create(ctypes.byref(cfg), int(key_capacity), int(value_capacity),
                                    int(seed), float(grow_factor), int(min_bucket_size),
                                    int(max_bucket_size), int(max_values_per_key), int(ib), int(cb),
                                    int(sb), int(bool(no_init)), ctypes.byref(h)))
        self._h = h
        self._cfg = cfg

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.wc_blht_destroy(h)
            self._h = None

    def info(self):
        inf = BlInfo()
        _check(lib().wc_blht_get_info(self._h, ctypes.byref(inf)))
        return inf

    @property
    def key_bytes(self):
        return self._cfg.key_bytes

    @property
    def value_bytes(self):
        return self._cfg.value_bytes

    @property
    def key_capacity(self):
        return self.info().key_capacity

    @property
    def value_capacity(self):
        return self.info().value_capacity

    def bytes_total(self):
        return self.info().bytes_total

    def init(self, seed=None, stream=None):
        s = self.info().seed if seed is None else seed
        _check(lib().wc_blht_init(self._h, int(s), _stream(stream)))

    def insert(self, keys_in, values_in, num_in=None, stream=None,
               probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
               status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(values_in, self.value_bytes, "values_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_blht_insert(self._h, _ptr(keys_in), _ptr(values_in),
                                    _numel(keys_in, num_in), _stream(stream),
                                    int(probing_length), _ptr(status_out), h, int(ignore)))

    def num_values(self, keys_in=None, num_per_key_out=None, num_in=None, stream=None,
                   probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
                   status_handler=None, ignore=0):
        """list lengths per key (uint64 tensor, optional) and their sum; with
        no keys, the number of values in the table"""
        if keys_in is None:
            return self._counter(lib().wc_blht_total_values, stream)
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        out = _u64(0)
        _check(lib().wc_blht_num_values(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                        ctypes.byref(out), _ptr(num_per_key_out),
                                        _stream(stream), int(probing_length), _ptr(status_out),
                                        h, int(ignore)))
        return int(out.value)

    def retrieve(self, keys_in, begin_offsets_out, end_offsets_out, values_out=None,
                 num_in=None, stream=None, probing_length=DEFAULT_PROBING_LENGTH,
                 status_out=None, status_handler=None, ignore=0):
        """values_out None: dry run (end_offsets_out gets the counts);
        returns the total number of values"""
        _check_width(keys_in, self.key_bytes, "keys_in")
        if values_out is not None:
            _check_width(values_out, self.value_bytes, "values_out")
        h = _handler(status_out, status_handler)
        out = _u64(0)
        _check(lib().wc_blht_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                      _ptr(begin_offsets_out), _ptr(end_offsets_out),
                                      _ptr(values_out), ctypes.byref(out), _stream(stream),
                                      int(probing_length), _ptr(status_out), h, int(ignore)))
        return int(out.value)

    def retrieve_all_keys(self, keys_out=None, stream=None):
        out = _u64(0)
        _check(lib().wc_blht_retrieve_all_keys(self._h, _ptr(keys_out), ctypes.byref(out),
                                               _stream(stream)))
        return int(out.value)

    def _counter(self, fn, stream):
        out = _u64(0)
        _check(fn(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)

    def num_keys(self, stream=None):
        return self._counter(lib().wc_blht_num_keys, stream)

    def pool_used(self, stream=None):
        """pool elements handed out (values and bucket headers)"""
        return self._counter(lib().wc_blht_pool_used, stream)

    def key_load_factor(self, stream=None):
        return self.num_keys(stream) / self.key_capacity

    def value_load_factor(self, stream=None):
        return self.pool_used(stream) / self.value_capacity

    def peek_status(self, stream=None):
        out = ctypes.c_uint32(0)
        _check(lib().wc_blht_peek_status(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)

    def pop_status(self, stream=None):
        out = ctypes.c_uint32(0)
        _check(lib().wc_blht_pop_status(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)


class MultiBucketHashTable:
    """warpcore::MultiBucketHashTable (multi_bucket_hash_table.cuh:88-110):
    a slot holds a key and a bucket of `bucket_size` values (ArrayBucket's
    B, 1 .. cg_size); a key's values fill its last bucket before it takes
    another slot.  The empty value (default 0) marks a free place and cannot
    be stored.  retrieve returns each key's values in insertion order with
    begin/end offsets."""

    def __init__(self, min_capacity, seed=DEFAULT_SEED, max_values_per_key=2**64 - 1,
                 no_init=False, key_bytes=4, value_bytes=None, bucket_size=2, empty_value=0,
                 empty_key=None, tombstone_key=None, probing=None, hasher1=None, hasher2=None,
                 cg_size=None):
        value_bytes = key_bytes if value_bytes is None else value_bytes
        cfg = _table_config(lib().wc_svht_default_config, key_bytes, key_bytes, empty_key,
                            tombstone_key, probing, hasher1, hasher2, cg_size)
        cfg.value_bytes = value_bytes
        h = ctypes.c_void_p()
        _check(lib().wc_mbht_create(ctypes.byref(cfg), int(bucket_size), int(empty_value),
                                    int(min_capacity), int(seed), int(max_values_per_key),
                                    int(bool(no_init)), ctypes.byref(h)))
        self._h = h
        self._cfg = cfg

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.wc_mbht_destroy(h)
            self._h = None

    def info(self):
        inf = MbInfo()
        _check(lib().wc_mbht_get_info(self._h, ctypes.byref(inf)))
        return inf

    @property
    def key_bytes(self):
        return self._cfg.key_bytes

    @property
    def value_bytes(self):
        return self._cfg.value_bytes

    @property
    def capacity(self):
        return self.info().capacity

    @property
    def value_capacity(self):
        return self.info().value_capacity

    def bucket_size(self):
        return self.info().bucket_size

    def bytes_total(self):
        return self.info().bytes_total

    def init(self, stream=None):
        _check(lib().wc_mbht_init(self._h, _stream(stream)))

    def insert(self, keys_in, values_in, num_in=None, stream=None,
               probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
               status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(values_in, self.value_bytes, "values_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_mbht_insert(self._h, _ptr(keys_in), _ptr(values_in),
                                    _numel(keys_in, num_in), _stream(stream),
                                    int(probing_length), _ptr(status_out), h, int(ignore)))

    def num_values(self, keys_in=None, num_per_key_out=None, num_in=None, stream=None,
                   probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
                   status_handler=None, ignore=0):
        """values per key (uint64 tensor, optional) and their sum; with no
        keys, the number of values in the table (size)"""
        if keys_in is None:
            return self.size(stream)
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        out = _u64(0)
        _check(lib().wc_mbht_num_values(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                        ctypes.byref(out), _ptr(num_per_key_out),
                                        _stream(stream), int(probing_length), _ptr(status_out),
                                        h, int(ignore)))
        return int(out.value)

    def retrieve(self, keys_in, begin_offsets_out, end_offsets_out, values_out=None,
                 num_in=None, stream=None, probing_length=DEFAULT_PROBING_LENGTH,
                 status_out=None, status_handler=None, ignore=0):
        """values_out None: dry run (end_offsets_out gets the counts);
        returns the total number of values"""
        _check_width(keys_in, self.key_bytes, "keys_in")
        if values_out is not None:
            _check_width(values_out, self.value_bytes, "values_out")
        h = _handler(status_out, status_handler)
        out = _u64(0)
        _check(lib().wc_mbht_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                      _ptr(begin_offsets_out), _ptr(end_offsets_out),
                                      _ptr(values_out), ctypes.byref(out), _stream(stream),
                                      int(probing_length), _ptr(status_out), h, int(ignore)))
        return int(out.value)

    def retrieve_all_keys(self, keys_out=None, stream=None):
        """each stored key once; keys_out None: only the count"""
        out = _u64(0)
        _check(lib().wc_mbht_retrieve_all_keys(self._h, _ptr(keys_out), ctypes.byref(out),
                                               _stream(stream)))
        return int(out.value)

    def _counter(self, fn, stream):
        out = _u64(0)
        _check(fn(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)

    def num_keys(self, stream=None):
        return self._counter(lib().wc_mbht_num_keys, stream)

    def num_occupied(self, stream=None):
        return self._counter(lib().wc_mbht_num_occupied, stream)

    def size(self, stream=None):
        return self._counter(lib().wc_mbht_size, stream)

    def key_load_factor(self, stream=None):
        return self.num_occupied(stream) / self.capacity

    def value_load_factor(self, stream=None):
        return self.size(stream) / self.value_capacity

    def storage_density(self, stream=None):
        payload = self.num_keys(stream) * self.key_bytes + self.size(stream) * self.value_bytes
        return payload / self.bytes_total()

    def relative_storage_density(self, stream=None):
        values = self.size(stream) * self.value_bytes
        payload = self.num_keys(stream) * self.key_bytes + values
        return payload / (self.num_occupied(stream) * self.key_bytes + values)

    def peek_status(self, stream=None):
        out = ctypes.c_uint32(0)
        _check(lib().wc_mbht_peek_status(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)

    def pop_status(self, stream=None):
        out = ctypes.c_uint32(0)
        _check(lib().wc_mbht_pop_status(self._h, _stream(stream), ctypes.byref(out)))
        return int(out.value)


class HashSet(_Table):
    """warpcore::HashSet (hash_set.cuh:16-22); default CG 16."""

    def __init__(self, min_capacity, seed=DEFAULT_SEED, key_bytes=4, empty_key=None,
                 tombstone_key=None, probing=None, hasher1=None, hasher2=None,
                 cg_size=None):
        cfg = _table_config(lib().wc_hashset_default_config, key_bytes, None, empty_key,
                            tombstone_key, probing, hasher1, hasher2, cg_size)
        self._make(lib().wc_hashset_create, cfg, int(min_capacity), int(seed))

    def insert(self, keys_in, num_in=None, stream=None,
               probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
               status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_hashset_insert(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                       _stream(stream), int(probing_length),
                                       _ptr(status_out), h, int(ignore)))

    def retrieve(self, keys_in, flags_out, num_in=None, stream=None,
                 probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
                 status_handler=None, ignore=0):
        """Membership flags (one byte per key: bool / uint8 tensor)."""
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(flags_out, 1, "flags_out")
        h = _handler(status_out, status_handler)
        _check(lib().wc_hashset_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                         _ptr(flags_out), _stream(stream),
                                         int(probing_length), _ptr(status_out), h,
                                         int(ignore)))

    contains = retrieve

    def erase(self, keys_in, num_in=None, stream=None,
              probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
              status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_hashset_erase(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                      _stream(stream), int(probing_length),
                                      _ptr(status_out), h, int(ignore)))


class CountingHashTable(_Table):
    """warpcore::CountingHashTable (counting_hash_table.cuh:18-26); default CG 4."""

    def __init__(self, min_capacity, seed=DEFAULT_SEED, max_count=None, no_init=False,
                 key_bytes=4, value_bytes=None, empty_key=None, tombstone_key=None,
                 probing=None, hasher1=None, hasher2=None, cg_size=None):
        value_bytes = key_bytes if value_bytes is None else value_bytes
        if max_count is None:
            max_count = (1 << (8 * value_bytes)) - 1
        cfg = _table_config(lib().wc_counting_default_config, key_bytes, value_bytes,
                            empty_key, tombstone_key, probing, hasher1, hasher2, cg_size)
        self._make(lib().wc_counting_create, cfg, int(min_capacity), int(seed),
                   int(max_count), int(bool(no_init)))

    @property
    def max_count(self):
        return self.info().max_count

    def insert(self, keys_in, num_in=None, stream=None,
               probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
               status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_counting_insert(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                        _stream(stream), int(probing_length),
                                        _ptr(status_out), h, int(ignore)))

    def retrieve(self, keys_in, values_out, num_in=None, stream=None,
                 probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
                 status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        _check_width(values_out, self._cfg.value_bytes, "values_out")
        h = _handler(status_out, status_handler)
        _check(lib().wc_counting_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                          _ptr(values_out), _stream(stream),
                                          int(probing_length), _ptr(status_out), h,
                                          int(ignore)))

    def erase(self, keys_in, num_in=None, stream=None,
              probing_length=DEFAULT_PROBING_LENGTH, status_out=None,
              status_handler=None, ignore=0):
        _check_width(keys_in, self.key_bytes, "keys_in")
        h = _handler(status_out, status_handler)
        _check(lib().wc_counting_erase(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                       _stream(stream), int(probing_length),
                                       _ptr(status_out), h, int(ignore)))


class BloomFilter:
    """warpcore::BloomFilter<Key, Hasher, Slot, CGSize> (bloom_filter.cuh:15-20).

    With num_shards > 1, this object is shard `shard` of the filter
    (num_bits, k, seed): it holds the blocks b with
    b * num_shards // num_blocks == shard, skips the keys of other blocks on
    insert and reports them absent on retrieve (wc_bloom_create_shard)."""

    def __init__(self, num_bits, k, seed=DEFAULT_SEED, key_bytes=8, slot_bytes=8,
                 cg_size=1, hasher=HASH_MURMUR, shard=0, num_shards=1):
        cfg = BloomConfig(key_bytes, slot_bytes, cg_size, hasher)
        h = ctypes.c_void_p()
        if num_shards == 1 and shard == 0:
            _check(lib().wc_bloom_create(ctypes.byref(cfg), int(num_bits), int(k), int(seed),
                                         ctypes.byref(h)))
        else:
            _check(lib().wc_bloom_create_shard(ctypes.byref(cfg), int(num_bits), int(k),
                                               int(seed), int(shard), int(num_shards),
                                               ctypes.byref(h)))
        self._h = h
        self._cfg = cfg
        self.num_shards = int(num_shards)

    def block_range(self):
        """(first block, number of blocks) this object holds"""
        inf = self.info()
        return inf.block_base, inf.local_blocks

    def partition(self, keys_in, num_parts=None, stream=None):
        """group keys by the shard holding their block: returns (keys_out,
        perm, counts as a list of ints), perm[j] = input position of
        keys_out[j] (wc_bloom_partition)"""
        import torch
        _check_width(keys_in, self._cfg.key_bytes, "keys_in")
        parts = self.num_shards if num_parts is None else int(num_parts)
        n = keys_in.numel()
        keys_out = torch.empty_like(keys_in)
        perm = torch.empty(n, dtype=torch.int64, device=keys_in.device)
        buf = torch.zeros(3 * parts + 1, dtype=torch.int64, device=keys_in.device)
        _check(lib().wc_bloom_partition(self._h, _ptr(keys_in) if n else None, n, parts,
                                        _ptr(keys_out) if n else None, _ptr(perm) if n else None,
                                        buf.data_ptr(), buf[parts:].data_ptr(), _stream(stream)))
        host_buf = buf.tolist()
        if host_buf[-1]:
            raise WarpcoreError("wc_bloom_partition dropped %d keys whose position failed the "
                                "bounds check (keys changed during the call)" % host_buf[-1])
        return keys_out, perm, host_buf[:parts]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.wc_bloom_destroy(h)
            self._h = None

    def info(self):
        inf = BloomInfo()
        _check(lib().wc_bloom_get_info(self._h, ctypes.byref(inf)))
        return inf

    def num_bits(self):
        return self.info().num_bits

    def num_slots(self):
        return self.info().num_slots

    def num_blocks(self):
        return self.info().num_blocks

    def k(self):
        return self.info().k

    def words_ptr(self):
        return self.info().words

    def words_tensor(self):
        """The words this object holds (local_blocks x cg_size of them) as a
        torch tensor viewing the filter's device memory, int32 or int64
        holding the unsigned bit patterns.  The view does not own the memory:
        it is valid while the filter lives and is not re-created."""
        import torch
        inf = self.info()
        count = int(inf.local_blocks) * int(inf.cg_size)

        class _DeviceWords:
            __cuda_array_interface__ = {
                "shape": (count,), "typestr": "<i%d" % inf.slot_bytes,
                "data": (int(inf.words or 0), False), "version": 3, "strides": None}
        return torch.as_tensor(_DeviceWords(), device="cuda")

    def init(self, seed=None, stream=None):
        _check(lib().wc_bloom_init(self._h, int(self.info().seed if seed is None else seed),
                                   _stream(stream)))

    def insert(self, keys_in, num_in=None, stream=None):
        _check_width(keys_in, self._cfg.key_bytes, "keys_in")
        _check(lib().wc_bloom_insert(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                     _stream(stream)))

    def retrieve(self, keys_in, flags_out, num_in=None, stream=None):
        _check_width(keys_in, self._cfg.key_bytes, "keys_in")
        _check_width(flags_out, 1, "flags_out")
        _check(lib().wc_bloom_retrieve(self._h, _ptr(keys_in), _numel(keys_in, num_in),
                                       _ptr(flags_out), _stream(stream)))

    def fpr(self, n):
        out = ctypes.c_double()
        _check(lib().wc_bloom_fpr(self._h, int(n), ctypes.byref(out)))
        return out.value


class HostPipe:
    """Device staging for bulk calls on host buffers (wc_host_pipe): copies
    of one chunk overlap the kernel of the previous one."""

    def __init__(self, chunk_keys=1 << 22, depth=3):
        h = ctypes.c_void_p()
        _check(lib().wc_host_pipe_create(int(chunk_keys), int(depth), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.wc_host_pipe_destroy(h)
            self._h = None


class Batch:
    """Runs many requests on many single-value tables in one launch
    (wc_batch_run): a list of (table, op, keys, values or values_out)."""

    def __init__(self, max_requests=4096, depth=2):
        h = ctypes.c_void_p()
        _check(lib().wc_batch_create(int(max_requests), int(depth), ctypes.byref(h)))
        self._h = h
        self.max_requests = max_requests

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.wc_batch_destroy(h)
            self._h = None

    def run(self, requests, stream=None, probing_length=DEFAULT_PROBING_LENGTH, blocks_per_sm=0):
        """requests: iterable of (table, "insert"|"retrieve", keys, values_or_out)
        or dicts with the same fields plus optional status_out/status_handler."""
        arr = (BatchRequest * len(requests))()
        keep = []
        for r, q in zip(arr, requests):
            if isinstance(q, dict):
                table, op, keys, buf = q["table"], q["op"], q["keys"], q["buffer"]
                status_out = q.get("status_out")
                handler = q.get("status_handler")
                ignore = q.get("ignore", 0)
            else:
                table, op, keys, buf = q
                status_out, handler, ignore = None, None, 0
            r.table = table._h.value
            r.op = OP_INSERT if op == "insert" else OP_RETRIEVE
            r.keys = _ptr(keys)
            if r.op == OP_INSERT:
                r.values = _ptr(buf)
            else:
                r.values_out = _ptr(buf)
            r.status_out = _ptr(status_out)
            r.status_handler = _handler(status_out, handler)
            r.ignore = ignore
            r.num = keys.numel()
            keep.append((keys, buf, status_out))
        _check(lib().wc_batch_run(self._h, arr, len(requests), _stream(stream),
                                  int(probing_length), int(blocks_per_sm)))
        return keep


def _handler(status_out, status_handler):
    if status_handler is not None:
        return int(status_handler)
    if status_out is None:
        return HANDLER_NOTHING
    return HANDLER_STATUS if status_out.element_size() == 4 else HANDLER_BOOLEAN
