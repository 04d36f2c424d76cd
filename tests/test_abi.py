"""The C-ABI library loads, exports what include/*.h declares, and keeps the
reference's struct layouts (no GPU needed; no GPU compute is called)."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import HASHES, MERKLE_CASES, FULL_DIGESTS_MAX, merkle_seed, sha256

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(INCLUDE, "**", "*.h"), recursive=True):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:ZK_EXTERN|ZK_EXTERNC)?\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**([a-z_][a-z0-9_]*)\s*\(",
                             src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = zk.load()
    decl = declared_functions()
    assert set(zk.ABI_SYMBOLS) <= decl, sorted(set(zk.ABI_SYMBOLS) - decl)
    assert set(zk.EXT_SYMBOLS) <= decl
    for name in sorted(decl):
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", zk.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert decl <= exported, sorted(decl - exported)


def test_static_archive_has_the_abi():
    a = os.path.join(os.path.dirname(zk.LIB_PATH), "libzeknox.a")
    out = subprocess.run(["nm", "--defined-only", a], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(zk.ABI_SYMBOLS) <= exported


def test_struct_layout_matches_reference(tmp_path):
    # sizes/offsets as a C compiler sees include/ntt/ntt.h (the Go binding's view)
    c = tmp_path / "l.c"
    c.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "lib.h"\n'
                 'int main(){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(NTT_Config), sizeof(NTT_TransposeConfig),'
                 ' offsetof(NTT_Config, extension_rate_bits), offsetof(NTT_Config, with_coset),'
                 ' offsetof(NTT_Config, salt_size), sizeof(RustError)); return 0;}\n')
    exe = tmp_path / "l"
    subprocess.run(["gcc", "-I", INCLUDE, str(c), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals == [24, 8, 12, 18, 20, 16]
    assert ctypes.sizeof(zk.NTTConfig) == 24 and ctypes.sizeof(zk.TransposeConfig) == 8
    assert zk.NTTConfig.salt_size.offset == 20 and zk.NTTConfig.with_coset.offset == 18


def test_headers_compile_as_cxx(tmp_path):
    c = tmp_path / "l.cpp"
    c.write_text('#include "lib.h"\n#include "zeknox_b200.h"\nint main(){return sizeof(NTT_Config) == 24 ? 0 : 1;}\n')
    subprocess.run(["g++", "-I", INCLUDE, str(c), "-o", str(tmp_path / "lx")], check=True)
    assert subprocess.run([str(tmp_path / "lx")]).returncode == 0


@pytest.mark.parametrize("name", list(HASHES))
def test_exported_cpu_builder_vs_reference(merkle_ref, name):
    """fill_digests_buf_linear_cpu is part of the ABI (a host builder), not a fallback."""
    import torch
    h = HASHES[name]
    for ci, (nl, ls, ch) in enumerate(MERKLE_CASES):
        key = "%s_%d_%d_%d" % (name, nl, ls, ch)
        leaves = torch.from_numpy(O.field_data(merkle_seed(ci, h), nl * ls).view(np.int64).copy())
        n_dig, n_cap = zk.merkle_sizes(nl, ch)
        dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64)
        cap = torch.zeros(n_cap * 4, dtype=torch.int64)
        zk.fill_digests_buf_linear_cpu(dig, cap, leaves, nl, ls, ch, h)
        assert np.array_equal(cap.numpy().view(np.uint64).reshape(-1, 4), merkle_ref[key + "_caps"]), key
        d = dig.numpy().view(np.uint64).reshape(-1, 4)[:n_dig]
        if nl <= FULL_DIGESTS_MAX:
            assert np.array_equal(d, merkle_ref[key + "_digests"]), key
        else:
            assert sha256(d) == merkle_ref[key + "_digests_sha256"].tobytes(), key


def test_cpu_builder_rejects_bad_geometry():
    import torch
    leaves = torch.zeros(16 * 5, dtype=torch.int64)
    dig = torch.zeros(64, dtype=torch.int64)
    cap = torch.zeros(8, dtype=torch.int64)
    with pytest.raises(zk.ZeknoxError):
        # 3 caps is not 2^cap_height
        zk.load().fill_digests_buf_linear_cpu(zk._ptr(dig), zk._ptr(cap), zk._ptr(leaves), 26, 3, 16, 5, 1, 0)
        raise zk.ZeknoxError(1, zk.last_error() or "")
    assert "cap_buf_size" in zk.last_error()


def _rejects(fn, *args):
    """Call an entry point that must refuse its arguments before touching a GPU."""
    e = fn(*args)
    msg = ctypes.string_at(e.message).decode() if e.message else ""
    if e.message:
        zk._libc.free(e.message)
    return e.code, msg


@pytest.mark.parametrize("lg_n,rate", [(1, 0xFFFFFFFF), (0xFFFFFFFF, 1), (16, 0xFFFFFFF0), (31, 2), (33, 1)])
def test_size_checks_do_not_wrap(lg_n, rate):
    """lg_n + rate_bits in 32-bit arithmetic can wrap to a small value; each
    term is checked on its own, so these sizes are refused with
    cudaErrorInvalidValue (1) before any kernel could be launched."""
    L = zk.load()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the checks come first
    code, msg = _rejects(L.zeknox_lde_rows, 0, dummy, dummy, lg_n, rate, 4, 7, None)
    assert code == 1 and "2^32" in msg, msg
    code, msg = _rejects(L.zeknox_lde_rows_noalloc, 0, dummy, dummy, lg_n, rate, 4, 7, None)
    assert code == 1 and "static limit" in msg, msg
    cfg = zk.NTTConfig(batches=1, extension_rate_bits=rate, are_inputs_on_device=True, are_outputs_on_device=True)
    code, msg = _rejects(L.compute_batched_lde, 0, dummy, dummy, lg_n, 0, cfg)
    assert code == 1, msg
    job = zk.CommitJob(lg_n=lg_n, rate_bits=rate, cols=4, cap_height=0, hash_type=0, input=16, leaves=16,
                       digests=16, caps=16)
    code, msg = _rejects(L.zeknox_commit, 0, ctypes.byref(job), None)
    assert code == 1 and "2^32" in msg, msg


def test_noalloc_refuses_beyond_its_static_limit():
    L = zk.load()
    dummy = ctypes.c_void_p(16)
    for lg_n, rate in ((16, 3), (18, 1), (17, 2)):
        code, msg = _rejects(L.zeknox_lde_rows_noalloc, 0, dummy, dummy, lg_n, rate, 4, 7, None)
        assert code == 1 and "static limit" in msg, msg
