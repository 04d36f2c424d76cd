"""The vector host builders fill_digests_buf_linear_cpu_avx / _avx512
(native/merkle/merkle.h:64-88, native/merkle/merkle_avx.cpp): Poseidon forests
bit-identical to the oracle (whose Merkle is pinned to the reference's
fill_digests_buf_linear_cpu), on CPU."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O

CASES = [(4, 7, 2), (1, 9, 0), (2, 9, 0), (2, 12, 1), (1 << 10, 135, 4), (1 << 11, 84, 0), (1 << 9, 8, 3),
         (1 << 9, 4, 2), (1 << 8, 1, 1), (1 << 10, 17, 10), (8, 5, 1), (16, 13, 0), (32, 16, 3)]


def t(a):
    return torch.from_numpy(a.view(np.int64))


def build(vector, leaves, nl, ls, ch, h=0):
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    dig = np.zeros(max(n_dig, 1) * 4, dtype=np.uint64)
    cap = np.zeros(n_cap * 4, dtype=np.uint64)
    zk.fill_digests_buf_linear_cpu(t(dig), t(cap), t(leaves), nl, ls, ch, h, vector=vector)
    return dig[:n_dig * 4].reshape(-1, 4), cap.reshape(-1, 4)


@pytest.mark.parametrize("vector", ["avx", "avx512"])
@pytest.mark.parametrize("nl,ls,ch", CASES)
def test_matches_oracle(vector, nl, ls, ch):
    leaves = O.field_data(nl * 7 + ls + ch, nl * ls)
    d, c = build(vector, leaves, nl, ls, ch)
    d2, c2 = O.merkle(leaves, ls, ch, 0)
    assert np.array_equal(c, c2)
    assert np.array_equal(d, d2)


@pytest.mark.parametrize("vector", ["avx", "avx512"])
def test_reference_test_shape(vector):
    # native/tests/tests.cu:720-818: 4 copies of a 7-element leaf, caps == leaves
    leaf = np.array([8395359103262935841, 1377884553022145855, 2370707998790318766, 3651132590097252162,
                     1141848076261006345, 12736915248278257710, 9898074228282442027], dtype=np.uint64)
    leaves = np.tile(leaf, 4)
    _, c = build(vector, leaves, 4, 7, 2)
    _, c2 = O.merkle(leaves, 7, 2, 0)
    assert np.array_equal(c, c2)
    assert all(np.array_equal(c[0], c[i]) for i in range(4))


@pytest.mark.parametrize("vector", ["avx", "avx512"])
@pytest.mark.parametrize("h", [1, 2, 3, 4, 7])
def test_other_hashes_rejected_without_writing(vector, h):
    leaves = O.field_data(3, 16 * 9)
    n_dig, n_cap = zk.merkle_sizes(16, 1)
    dig = np.full(n_dig * 4, 7, dtype=np.uint64)
    cap = np.full(n_cap * 4, 7, dtype=np.uint64)
    with pytest.raises(zk.ZeknoxError, match="only Poseidon"):
        zk.fill_digests_buf_linear_cpu(t(dig), t(cap), t(leaves), 16, 9, 1, h, vector=vector)
    assert (dig == 7).all() and (cap == 7).all()


@pytest.mark.parametrize("vector", ["avx", "avx512"])
def test_bad_geometry_rejected(vector):
    L = zk.load()
    dig = torch.zeros(64, dtype=torch.int64)
    cap = torch.zeros(8, dtype=torch.int64)
    leaves = torch.zeros(12 * 9, dtype=torch.int64)
    fn = L.fill_digests_buf_linear_cpu_avx if vector == "avx" else L.fill_digests_buf_linear_cpu_avx512
    before = zk.last_error()
    fn(zk._ptr(dig), zk._ptr(cap), zk._ptr(leaves), 20, 2, 12, 9, 1, 0)  # 12 leaves: not 2 x a power of two
    assert zk.last_error() != before
