"""Golden NTT / LDE / transpose / Merkle vectors produced by the reference's
own CUDA library (tests/golden/make_golden_gpu.py, run on a B200 against
oracle/_ref/libzeknox_ref_gpu.so built from the reference sources).

The CPU tests pin the oracle to them; the GPU tests check this library."""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden.make_golden_gpu import (LDE_CASES, MERKLE_GPU_CASES, NTT_CASES, TRANSPOSE_CASES, lde_seed,
                                          ntt_seed)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_gpu.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLDEN))


def same(gold, key, arr):
    arr = np.ascontiguousarray(arr, dtype=np.uint64)
    if key in gold:
        return np.array_equal(gold[key], arr)
    return hashlib.sha256(arr.tobytes()).digest() == gold[key + "_sha256"].tobytes()


def test_oracle_ntt_matches_reference_gpu(gold):
    for lg, b in NTT_CASES:
        for inv in (0, 1):
            for cs in (0, 1):
                x = O.field_data(ntt_seed(lg, b, inv, cs), b << lg)
                y = O.batched_ntt(x, lg, b, inverse=bool(inv), with_coset=bool(cs))
                assert same(gold, "ntt_%d_%d_%d_%d" % (lg, b, inv, cs), y), (lg, b, inv, cs)


def test_oracle_lde_transpose_merkle_match_reference_gpu(gold):
    for lg, rate, b in LDE_CASES:
        for cs in (0, 1):
            c = O.field_data(lde_seed(lg, rate, b), b << lg)
            assert same(gold, "lde_%d_%d_%d_%d" % (lg, rate, b, cs), O.batched_lde(c, lg, rate, b, with_coset=bool(cs)))
    for lg, b in TRANSPOSE_CASES:
        x = O.field_data(9000 + lg + b, b << lg)
        assert same(gold, "transpose_%d_%d" % (lg, b), O.transpose_rev(x, lg, b))
    for nl, ls, ch, h in MERKLE_GPU_CASES:
        leaves = O.field_data(11000 + nl + ls + ch + h, nl * ls)
        d, c = O.merkle(leaves, ls, ch, h)
        assert same(gold, "merkle_%d_%d_%d_%d_digests" % (nl, ls, ch, h), d)
        assert same(gold, "merkle_%d_%d_%d_%d_caps" % (nl, ls, ch, h), c)


@pytest.mark.gpu
def test_library_matches_reference_gpu(gold):
    import torch

    import zeknox_b200 as zk
    from tests.helpers import to_dev, to_np
    for lg, b in NTT_CASES:
        for inv in (0, 1):
            for cs in (0, 1):
                t = to_dev(O.field_data(ntt_seed(lg, b, inv, cs), b << lg))
                zk.ntt_batch(0, t, lg, b, with_coset=bool(cs), inverse=bool(inv))
                assert same(gold, "ntt_%d_%d_%d_%d" % (lg, b, inv, cs), to_np(t)), (lg, b, inv, cs)
    for lg, rate, b in LDE_CASES:
        for cs in (0, 1):
            out = torch.zeros(b << (lg + rate), dtype=torch.int64, device="cuda")
            zk.lde_batch(0, out, to_dev(O.field_data(lde_seed(lg, rate, b), b << lg)), lg, b, rate, with_coset=bool(cs))
            assert same(gold, "lde_%d_%d_%d_%d" % (lg, rate, b, cs), to_np(out))
    for lg, b in TRANSPOSE_CASES:
        out = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
        zk.transpose_rev_batch(0, out, to_dev(O.field_data(9000 + lg + b, b << lg)), lg, b)
        assert same(gold, "transpose_%d_%d" % (lg, b), to_np(out))
    for nl, ls, ch, h in MERKLE_GPU_CASES:
        n_dig, n_cap = zk.merkle_sizes(nl, ch)
        dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
        cap = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
        zk.fill_digests_buf_linear_gpu(dig, cap, to_dev(O.field_data(11000 + nl + ls + ch + h, nl * ls)), nl, ls, ch, h)
        torch.cuda.synchronize()
        assert same(gold, "merkle_%d_%d_%d_%d_digests" % (nl, ls, ch, h), to_np(dig)[:n_dig * 4].reshape(-1, 4))
        assert same(gold, "merkle_%d_%d_%d_%d_caps" % (nl, ls, ch, h), to_np(cap).reshape(-1, 4))
