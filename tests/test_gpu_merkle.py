"""GPU Merkle builder (fill_digests_buf_linear_gpu_with_gpu_ptr) vs the oracle
and the reference's golden forests; bit-exact."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import HASHES, MERKLE_CASES, FULL_DIGESTS_MAX, merkle_seed, sha256, to_dev, to_np, empty_dev

pytestmark = pytest.mark.gpu


def run_gpu(leaves_np, nl, ls, ch, h):
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    leaves = to_dev(leaves_np)
    dig = empty_dev(n_dig * 4)
    cap = empty_dev(n_cap * 4)
    zk.fill_digests_buf_linear_gpu(dig, cap, leaves, nl, ls, ch, h)
    torch.cuda.synchronize()
    return to_np(dig)[:n_dig * 4].reshape(-1, 4), to_np(cap).reshape(-1, 4)


@pytest.mark.parametrize("name", list(HASHES))
def test_golden_forests(merkle_ref, name):
    h = HASHES[name]
    for ci, (nl, ls, ch) in enumerate(MERKLE_CASES):
        key = "%s_%d_%d_%d" % (name, nl, ls, ch)
        dig, cap = run_gpu(O.field_data(merkle_seed(ci, h), nl * ls), nl, ls, ch, h)
        assert np.array_equal(cap, merkle_ref[key + "_caps"]), key
        if nl <= FULL_DIGESTS_MAX:
            assert np.array_equal(dig, merkle_ref[key + "_digests"]), key
        else:
            assert sha256(dig) == merkle_ref[key + "_digests_sha256"].tobytes(), key


@pytest.mark.parametrize("name", list(HASHES))
@pytest.mark.parametrize("nl,ls,ch", [(1 << 12, 135, 4), (1 << 13, 84, 0), (1 << 14, 9, 2), (1 << 11, 4, 3),
                                      (1 << 11, 1, 1), (1 << 10, 17, 10), (1 << 12, 8, 11), (1 << 16, 12, 0)])
def test_vs_oracle(name, nl, ls, ch):
    h = HASHES[name]
    leaves = O.field_data(nl + ls + ch, nl * ls)
    dig, cap = run_gpu(leaves, nl, ls, ch, h)
    d2, c2 = O.merkle(leaves, ls, ch, h)
    assert np.array_equal(cap, c2)
    assert np.array_equal(dig, d2)


def test_kat_tree4x7(kat):
    lv = np.array(kat["tree4x7_leaves"], dtype=np.uint64)
    for name, h in HASHES.items():
        dig, cap = run_gpu(lv, 4, 7, 0, h)
        exp = np.array(kat["tree4x7_" + name], dtype=np.uint64)
        # digests: [n01, n23, leaf0..leaf3]; cap: root
        assert np.array_equal(dig[2:6], exp[0:4]) and np.array_equal(dig[0:2], exp[4:6])
        assert np.array_equal(cap[0], exp[6])


def test_kat_single_hashes(kat):
    # caps == leaves: the caps are the leaf hashes
    leaf = np.array(kat["poseidon_leaf"], dtype=np.uint64)
    for k in range(5, 10):
        _, cap = run_gpu(leaf[:k], 1, k, 0, 0)
        assert [int(x) for x in cap[0]] == kat["poseidon_expected"][k]
    _, cap = run_gpu(np.array(kat["poseidon2_input"], dtype=np.uint64), 1, 12, 0, 3)
    assert [int(x) for x in cap[0]] == kat["poseidon2_expected"]
    _, cap = run_gpu(np.array(kat["monolith_input"], dtype=np.uint64), 1, 12, 0, 4)
    assert [int(x) for x in cap[0]] == kat["monolith_expected"]
    _, cap = run_gpu(np.array(kat["poseidon_bn128_input"], dtype=np.uint64), 1, 12, 0, 2)
    assert [int(x) for x in cap[0]] == kat["poseidon_bn128_expected"]
    for size in (4, 5, 6):
        _, cap = run_gpu(np.array(kat["keccak_data"][:size], dtype=np.uint64), 1, size, 0, 1)
        assert [int(x) for x in cap[0]] == kat["keccak_expected"][size]


def test_rejects_bad_geometry_without_writing():
    leaves = to_dev(O.field_data(5, 16 * 5))
    dig = torch.full((64,), 7, dtype=torch.int64, device="cuda")
    cap = torch.full((8,), 7, dtype=torch.int64, device="cuda")
    with pytest.raises(zk.ZeknoxError):
        zk.load().fill_digests_buf_linear_gpu_with_gpu_ptr(zk._ptr(dig), zk._ptr(cap), zk._ptr(leaves), 26, 3, 16, 5, 1,
                                                            0, 0)
        raise zk.ZeknoxError(1, zk.last_error() or "")
    with pytest.raises(zk.ZeknoxError):
        zk.fill_digests_buf_linear_gpu(dig, cap, leaves, 16, 5, 1, 7)  # no hash type 7
    torch.cuda.synchronize()
    assert bool((dig == 7).all()) and bool((cap == 7).all())


def test_multigpu_entry_matches_single():
    nl, ls, ch = 1 << 12, 20, 3
    leaves_np = O.field_data(3, nl * ls)
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    leaves = to_dev(leaves_np)
    dig, cap = empty_dev(n_dig * 4), empty_dev(n_cap * 4)
    zk.fill_digests_buf_linear_multigpu(dig, cap, leaves, nl, ls, ch, 3)
    d2, c2 = O.merkle(leaves_np, ls, ch, 3)
    assert np.array_equal(to_np(cap).reshape(-1, 4), c2)
    assert np.array_equal(to_np(dig).reshape(-1, 4), d2)


def test_merkle_batch_mixed_hashes():
    cases = [(1 << 12, 135, 4, 3), (1 << 12, 135, 4, 4), (1 << 12, 135, 4, 1), (1 << 10, 9, 0, 0), (64, 5, 6, 3)]
    jobs, bufs = [], []
    for k, (nl, ls, ch, h) in enumerate(cases):
        leaves_np = O.field_data(500 + k, nl * ls)
        n_dig, n_cap = zk.merkle_sizes(nl, ch)
        lv, dg, cp = to_dev(leaves_np), empty_dev(n_dig * 4), empty_dev(n_cap * 4)
        jobs.append(zk.merkle_job(lv, dg, cp, nl, ls, ch, h))
        bufs.append((leaves_np, lv, dg, cp, n_dig, ls, ch, h))
    for _ in range(2):  # capture, then replay
        zk.merkle_batch(0, jobs)
        for leaves_np, lv, dg, cp, n_dig, ls, ch, h in bufs:
            d2, c2 = O.merkle(leaves_np, ls, ch, h)
            assert np.array_equal(to_np(cp).reshape(-1, 4), c2)
            assert np.array_equal(to_np(dg)[:n_dig * 4].reshape(-1, 4), d2)
