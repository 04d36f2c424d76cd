#!/usr/bin/env python3
"""Golden NTT / LDE / transpose / Merkle vectors from the reference's own CUDA
library, run on a GPU host.

The reference has no CPU NTT, so the NTT family is pinned by running its CUDA
path (native/lib.cu compute_batched_ntt / compute_batched_lde /
compute_transpose_rev, rebuilt for sm_100a by ``make -C oracle ref_gpu`` into
oracle/_ref/libzeknox_ref_gpu.so) on the same seeded inputs the tests use.
Outputs go to <out> (default golden_gpu_new.npz in the working directory); small results are
stored whole, large ones as sha256 of their bytes.  The committed copy is
tests/golden/golden_gpu.npz.

    python tests/golden/make_golden_gpu.py [--out PATH]
"""
import argparse
import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
import zeknox_b200 as zk  # noqa: E402  (ctypes struct layouts only)

NTT_CASES = [(lg, b) for lg in (2, 4, 8, 10, 12, 13, 16) for b in (1, 3)]
LDE_CASES = [(2, 1, 2), (3, 2, 3), (8, 3, 2), (12, 1, 3), (13, 3, 2), (15, 3, 2)]
TRANSPOSE_CASES = [(5, 3), (10, 33), (12, 256)]
MERKLE_GPU_CASES = [(16, 7, 1, 0), (64, 8, 0, 3), (1024, 12, 4, 4), (4096, 7, 1, 0), (4096, 9, 2, 1), (1 << 14, 20, 3, 3)]
FULL_MAX = 4096


def ntt_seed(lg, b, inverse, coset):
    return 5000 + 97 * lg + 13 * b + 3 * inverse + coset


def lde_seed(lg, rate, b):
    return 7000 + 31 * lg + 7 * rate + b


def store(out, key, arr):
    arr = np.ascontiguousarray(arr, dtype=np.uint64)
    if arr.size <= FULL_MAX:
        out[key] = arr
    else:
        out[key + "_sha256"] = np.frombuffer(hashlib.sha256(arr.tobytes()).digest(), dtype=np.uint8)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="golden_gpu_new.npz")
    args = ap.parse_args()
    R = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libzeknox_ref_gpu.so"))
    R.init_twiddle_factors.restype = zk.RustError
    R.init_twiddle_factors.argtypes = [ctypes.c_size_t, ctypes.c_size_t]
    R.init_coset.restype = zk.RustError
    R.init_coset.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_uint64]
    R.compute_batched_ntt.restype = zk.RustError
    R.compute_batched_ntt.argtypes = [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, zk.NTTConfig]
    R.compute_batched_lde.restype = zk.RustError
    R.compute_batched_lde.argtypes = [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                      zk.NTTConfig]
    R.compute_transpose_rev.restype = zk.RustError
    R.compute_transpose_rev.argtypes = [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                        zk.TransposeConfig]
    R.fill_digests_buf_linear_gpu_with_gpu_ptr.restype = None
    R.fill_digests_buf_linear_gpu_with_gpu_ptr.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64] * 7

    def ok(e, what):
        assert e.code == 0, (what, e.code)

    lgs = sorted({lg for lg, _ in NTT_CASES} | {lg + r for lg, r, _ in LDE_CASES})
    for lg in lgs:
        ok(R.init_twiddle_factors(0, lg), "twiddles %d" % lg)
    ok(R.init_coset(0, max(lgs), 7), "coset")

    out = {}
    mism = 0
    for lg, b in NTT_CASES:
        for inverse in (0, 1):
            for coset in (0, 1):
                x = O.field_data(ntt_seed(lg, b, inverse, coset), b << lg)
                y = x.copy()
                cfg = zk.ntt_config(b, 0, False, False, bool(coset))
                ok(R.compute_batched_ntt(0, y.ctypes.data, lg, inverse, cfg), "ntt")
                store(out, "ntt_%d_%d_%d_%d" % (lg, b, inverse, coset), y)
                mism += not np.array_equal(y, O.batched_ntt(x, lg, b, inverse=bool(inverse), with_coset=bool(coset)))
    for lg, rate, b in LDE_CASES:
        for coset in (0, 1):
            c = O.field_data(lde_seed(lg, rate, b), b << lg)
            y = np.zeros(b << (lg + rate), dtype=np.uint64)
            cfg = zk.ntt_config(b, rate, False, False, bool(coset))
            ok(R.compute_batched_lde(0, y.ctypes.data, c.ctypes.data, lg, 0, cfg), "lde")
            store(out, "lde_%d_%d_%d_%d" % (lg, rate, b, coset), y)
            mism += not np.array_equal(y, O.batched_lde(c, lg, rate, b, with_coset=bool(coset)))
    for lg, b in TRANSPOSE_CASES:
        x = O.field_data(9000 + lg + b, b << lg)
        y = np.zeros_like(x)
        cfg = zk.TransposeConfig()
        cfg.batches, cfg.are_inputs_on_device, cfg.are_outputs_on_device = b, False, False
        ok(R.compute_transpose_rev(0, y.ctypes.data, x.ctypes.data, lg, cfg), "transpose")
        store(out, "transpose_%d_%d" % (lg, b), y)
        mism += not np.array_equal(y, O.transpose_rev(x, lg, b))
    import torch
    for nl, ls, ch, h in MERKLE_GPU_CASES:
        leaves = O.field_data(11000 + nl + ls + ch + h, nl * ls)
        n_dig, n_cap = O.merkle_sizes(nl, ch)
        lv = torch.from_numpy(leaves.view(np.int64).copy()).cuda()
        dg = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
        cp = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
        R.fill_digests_buf_linear_gpu_with_gpu_ptr(dg.data_ptr(), cp.data_ptr(), lv.data_ptr(), n_dig, n_cap, nl, ls,
                                                   ch, h, 0)
        torch.cuda.synchronize()
        d = dg.cpu().numpy().view(np.uint64).reshape(-1, 4)[:n_dig]
        c = cp.cpu().numpy().view(np.uint64).reshape(-1, 4)
        store(out, "merkle_%d_%d_%d_%d_digests" % (nl, ls, ch, h), d)
        store(out, "merkle_%d_%d_%d_%d_caps" % (nl, ls, ch, h), c)
        d2, c2 = O.merkle(leaves, ls, ch, h)
        mism += not (np.array_equal(d, d2) and np.array_equal(c, c2))
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez_compressed(args.out, **out)
    print("wrote %s: %d entries; oracle mismatches vs reference GPU: %d" % (args.out, len(out), mism))


if __name__ == "__main__":
    main()
