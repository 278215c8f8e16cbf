"""The C-ABI library loads without a GPU, exports every function that
include/warpcore_b200.h declares, and its host-only entry points (capacity
rule, default knobs) agree with the oracle and the reference's defaults."""
import ctypes
import os
import re
import subprocess

import pytest

import warpcore_b200 as wc
from oracle import oracle as o

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "warpcore_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wc_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "wc_svht_insert" in names and "wc_bloom_retrieve" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = wc.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []
    out = subprocess.run(["nm", "-D", "--defined-only", wc.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (wc_[a-z0-9_]+)", out))
    assert set(declared_functions()) <= exported


def test_python_binding_covers_header():
    assert set(declared_functions()) == set(wc.SIGNATURES)


def test_valid_capacity_matches_oracle():
    for m in (0, 1, 12345, 1310720, 2**27 / 0.9, 2**24 / 0.85, 10**10, 2**40):
        for cg in (1, 2, 4, 8, 16, 32):
            assert wc.valid_capacity(int(m), cg) == o.valid_capacity(int(m), cg)


def test_reference_capacities():
    # reference-exact capacities
    assert wc.valid_capacity(1310720, 8) == 2097496
    assert wc.valid_capacity(int(2**27 / 0.9), 8) == 149963432
    assert wc.valid_capacity(int(2**27 / 0.9), 16) == 151011248
    assert wc.valid_capacity(int(2**24 / 0.85), 4) == 19925396


def test_default_configs():
    cfg = wc.TableConfig()
    wc.lib().wc_svht_default_config(ctypes.byref(cfg), 4, 4)
    assert (cfg.cg_size, cfg.empty_key, cfg.tombstone_key, cfg.probing, cfg.hasher1) == \
        (8, 0, 0xFFFFFFFF, wc.PROBING_DOUBLE, wc.HASH_MURMUR)
    wc.lib().wc_hashset_default_config(ctypes.byref(cfg), 8)
    assert (cfg.cg_size, cfg.tombstone_key) == (16, 2**64 - 1)
    wc.lib().wc_counting_default_config(ctypes.byref(cfg), 4, 4)
    assert cfg.cg_size == 4


def test_invalid_config_is_rejected_without_gpu():
    cfg = wc.TableConfig()
    wc.lib().wc_svht_default_config(ctypes.byref(cfg), 4, 4)
    cfg.cg_size = 3
    h = ctypes.c_void_p()
    rc = wc.lib().wc_svht_create(ctypes.byref(cfg), 1000, 1, 0, ctypes.byref(h))
    assert rc == -1 and h.value is None
    assert b"cg_size" in wc.lib().wc_last_error()
    wc.lib().wc_svht_default_config(ctypes.byref(cfg), 4, 4)
    cfg.tombstone_key = 0
    assert wc.lib().wc_svht_create(ctypes.byref(cfg), 1000, 1, 0, ctypes.byref(h)) == -1


def test_ops_on_null_handle_fail_cleanly():
    lib = wc.lib()
    assert lib.wc_svht_insert(None, None, None, 10, None, 1, None, 0, 0) == -1
    assert lib.wc_table_destroy(None) == 0


def test_tune_set_validates_arguments():
    lib = wc.lib()
    assert lib.wc_tune_set(4, 0, 0, 0, 64, 0) == 0
    assert lib.wc_tune_set(3, 0, 0, 0, 64, 0) == -1
    assert lib.wc_tune_set(4, 5, 0, 0, 64, 0) == -1
    assert lib.wc_tune_set(4, 0, 4, 0, 64, 0) == -1
    assert lib.wc_tune_set(4, 0, 0, 12, 64, 0) == -1
    assert lib.wc_tune_set(4, 0, 0, 0, 48, 0) == -1
    assert lib.wc_tune_set(4, 0, 0, 0, 512, 0) == -1
    lib.wc_tune_reset()
    wc._load_tuning(lib)


def test_shipped_tuning_table_is_well_formed():
    import json
    import os
    path = os.path.join(os.path.dirname(wc.__file__), "tuning_b200.json")
    d = json.load(open(path))
    assert "B200" in d["device"]
    for kb, op, lb, sb, block, bps in d["entries"]:
        assert kb in (4, 8) and op in (0, 1, 2) and 0 <= lb < 4 and 0 <= sb < 12
        assert block in (32, 64, 128, 256)


def test_tune_load_reads_the_committed_table():
    """wc_tune_load (used by the Python binding and the C++ headers) parses
    the committed tuning file's entries; a missing file is an error and
    "none" loads nothing (no GPU needed)"""
    import ctypes
    import json
    import os
    import warpcore_b200 as wc
    path = os.path.join(os.path.dirname(wc.__file__), "tuning_b200.json")
    n = ctypes.c_uint64(0)
    assert wc.lib().wc_tune_load(path.encode(), ctypes.byref(n)) == 0
    assert n.value == len(json.load(open(path))["entries"]) > 0
    assert wc.lib().wc_tune_load(b"none", ctypes.byref(n)) == 0 and n.value == 0
    assert wc.lib().wc_tune_load(b"/nonexistent/tuning.json", ctypes.byref(n)) != 0
    # the library's own default location is the same file
    assert wc.lib().wc_tune_load(None, ctypes.byref(n)) == 0 and n.value > 0
