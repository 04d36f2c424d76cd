"""Tuning table (zeknox_tune_*): host-side behaviour, no GPU needed.

The knobs only choose launch shapes; that results do not depend on them is
checked on the GPU in test_gpu_tune.py.
"""
import os
import subprocess
import sys

import pytest

import zeknox_b200 as zk
from zeknox_b200 import autotune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KNOBS = {"leaf_threads": {64, 128, 256}, "lde_chunk_mib": None, "lde_last_logr": set(range(1, 9)),
         "wide_level_nodes": None, "coop_leaves": None, "lde_host_chunk_mib": None,
         "ntt_split_logr": {0, 7, 8, 9, 10}, "transpose_bulk": set(range(10))}


@pytest.fixture
def clean_table():
    zk.load()
    zk.tune_clear()
    yield
    zk.tune_clear()
    if os.path.exists(zk.TUNE_TABLE):
        zk.tune_load(zk.TUNE_TABLE)


def test_set_get_and_size_fallback(clean_table):
    assert zk.tune_get("lde_chunk_mib", 18, 64) == 64
    zk.tune_set("lde_chunk_mib", 32)  # every size
    assert zk.tune_get("lde_chunk_mib", 18, 64) == 32
    zk.tune_set("lde_chunk_mib", 96, lg=18)  # this size wins over the size-free entry
    assert zk.tune_get("lde_chunk_mib", 18, 64) == 96
    assert zk.tune_get("lde_chunk_mib", 17, 64) == 32
    assert zk.tune_get("lde_chunk_mib", None, 64) == 32
    zk.tune_clear()
    assert zk.tune_get("lde_chunk_mib", 18, 64) == 64


def test_load_table_with_comments_and_blank_lines(clean_table, tmp_path):
    p = tmp_path / "t.txt"
    p.write_text("# header\n\nleaf_threads.3 18 128   # per size\n  lde_last_logr * 8\n\t\nwide_level_nodes.0 20 8192\n")
    zk.tune_load(p)
    assert zk.tune_get("leaf_threads.3", 18, 256) == 128
    assert zk.tune_get("leaf_threads.3", 17, 256) == 256
    assert zk.tune_get("lde_last_logr", 15, 9) == 8
    assert zk.tune_get("wide_level_nodes.0", 20, 1 << 15) == 8192


@pytest.mark.parametrize("bad", ["lde_chunk_mib 18\n", "lde_chunk_mib x 32\n", "lde_chunk_mib 18 32 7\n",
                                 "lde_chunk_mib 18 -\n", "lde_chunk_mib 999 32\n"])
def test_malformed_table_changes_nothing(clean_table, tmp_path, bad):
    p = tmp_path / "t.txt"
    p.write_text("leaf_threads.3 18 64\n" + bad)
    with pytest.raises(zk.ZeknoxError) as e:
        zk.tune_load(p)
    assert ":2:" in str(e.value)
    assert zk.tune_get("leaf_threads.3", 18, 256) == 256  # the good first line was not applied


def test_missing_table_is_an_error(clean_table, tmp_path):
    with pytest.raises(zk.ZeknoxError):
        zk.tune_load(tmp_path / "absent.txt")


def test_env_table_read_by_the_c_library(tmp_path):
    # a C-ABI consumer (no Python) gets the table through ZEKNOX_TUNE_FILE
    p = tmp_path / "t.txt"
    p.write_text("lde_chunk_mib * 48\n")
    code = ("import ctypes; L = ctypes.CDLL(%r); L.zeknox_tune_get.restype = ctypes.c_uint64;"
            "L.zeknox_tune_get.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint64];"
            "print(L.zeknox_tune_get(b'lde_chunk_mib', 18, 64))" % zk.LIB_PATH)
    env = dict(os.environ, ZEKNOX_TUNE_FILE=str(p))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "48"
    env["ZEKNOX_TUNE_FILE"] = "none"
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "64"


def test_committed_table_is_well_formed():
    if not os.path.exists(zk.TUNE_TABLE):
        pytest.skip("no tuning table committed")
    for ln, line in enumerate(open(zk.TUNE_TABLE), 1):
        body = line.split("#", 1)[0].split()
        if not body:
            continue
        name, lg, value = body
        base = name.split(".")[0]
        assert base in KNOBS, (ln, name)
        if "." in name:
            assert int(name.split(".")[1]) in autotune.HASH_NAMES, (ln, name)
        assert lg == "*" or 0 <= int(lg) <= 32, (ln, lg)
        allowed = KNOBS[base]
        assert allowed is None or int(value) in allowed, (ln, value)
        assert int(value) > 0 or (allowed is not None and 0 in allowed), (ln, value)


def test_autotune_partial_run_keeps_other_knobs(tmp_path):
    """A run of some searches only (--only) keeps the other knobs' lines."""
    p = tmp_path / "t.txt"
    p.write_text("# header\nleaf_threads.3 18 128   # ms\nntt_split_logr 20 9 # ms\n"
                 "transpose_bulk 18 3\nlde_last_logr 13 8\n")
    kept = autotune.kept_table_lines(str(p), {"ntt_split_logr", "transpose_bulk"})
    assert [k.split()[0] for k in kept] == ["leaf_threads.3", "lde_last_logr"]
    assert autotune.kept_table_lines(str(tmp_path / "missing.txt"), {"lde_last_logr"}) == []


def test_autotune_candidates_include_the_defaults():
    for knob, dflt in autotune.DEFAULTS.items():
        assert autotune.CANDIDATES[knob][0] == dflt
        assert all(v in KNOBS[knob] for v in autotune.CANDIDATES[knob]) if KNOBS[knob] else True
    for lg, cols in autotune.lde_shapes(False):
        assert cols >= 16 and (cols << (lg + autotune.RATE)) <= 1 << 27
