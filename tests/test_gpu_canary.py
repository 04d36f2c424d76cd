"""Output canaries: every GPU entry point writes its result between guard
words (a fixed pattern on each side of the buffer, 4 KiB worth) and must
leave the guards untouched, on ragged shapes (odd column counts, sizes that
are not multiples of the tile, leaves of <= 4 words, caps == leaves).  The
GPU has no sanitizer here; this is its stand-in for out-of-bounds writes."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import HASHES, to_dev, to_np

pytestmark = pytest.mark.gpu

GUARD = 512  # words on each side
PATTERN = 0x5A5A5A5AA5A5A5A5  # the guard word (a valid int64)


def guarded(n):
    """(whole buffer, interior view of n words): guards of PATTERN, interior
    zero (Keccak leaves of < 4 words leave the rest of their digest as the
    buffer held it, zero in the oracle's)."""
    t = torch.full((n + 2 * GUARD,), PATTERN, dtype=torch.int64, device="cuda")
    t[GUARD:GUARD + n] = 0
    return t, t[GUARD:GUARD + n]


def intact(t, n):
    torch.cuda.synchronize()
    head, tail = t[:GUARD], t[GUARD + n:]
    return bool((head == PATTERN).all()) and bool((tail == PATTERN).all())


@pytest.mark.parametrize("lg,b,inverse,coset", [(1, 3, False, False), (5, 7, True, True), (11, 5, False, True),
                                                (13, 3, True, False)])
def test_ntt_in_place_stays_in_bounds(lg, b, inverse, coset):
    x = O.field_data(lg + 100 * b, b << lg)
    whole, inner = guarded(b << lg)
    inner.copy_(to_dev(x))
    zk.ntt_batch(0, inner, lg, b, with_coset=coset, inverse=inverse)
    assert intact(whole, b << lg)
    assert np.array_equal(to_np(inner), O.batched_ntt(x, lg, b, inverse=inverse, with_coset=coset))


@pytest.mark.parametrize("lg,rate,b", [(1, 1, 1), (4, 3, 3), (10, 2, 17), (12, 1, 5)])
def test_lde_entry_points_stay_in_bounds(lg, rate, b):
    c = O.field_data(lg + 7 * b, b << lg)
    N = 1 << (lg + rate)
    whole, inner = guarded(b * N)
    zk.lde_batch(0, inner, to_dev(c), lg, b, rate)
    assert intact(whole, b * N)
    assert np.array_equal(to_np(inner), O.batched_lde(c, lg, rate, b))
    whole2, rows = guarded(b * N)
    zk.lde_rows(0, rows, to_dev(c), lg, rate, b)
    assert intact(whole2, b * N)
    assert np.array_equal(to_np(rows), O.lde_rows(c, lg, rate, b))


@pytest.mark.parametrize("lg,b", [(0, 1), (3, 5), (6, 2), (7, 33), (10, 64)])
def test_transpose_stays_in_bounds(lg, b):
    x = O.field_data(lg + 11 * b, b << lg)
    whole, inner = guarded(b << lg)
    zk.transpose_rev_batch(0, inner, to_dev(x), lg, b)
    assert intact(whole, b << lg)
    assert np.array_equal(to_np(inner), O.transpose_rev(x, lg, b))


@pytest.mark.parametrize("name", list(HASHES))
@pytest.mark.parametrize("nl,ls,ch", [(1 << 9, 9, 2), (1 << 8, 3, 1), (1 << 6, 135, 6), (1 << 10, 17, 0)])
def test_forest_stays_in_bounds(name, nl, ls, ch):
    h = HASHES[name]
    leaves = O.field_data(nl + ls + h, nl * ls)
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    wd, dig = guarded(max(n_dig, 1) * 4)
    wc, cap = guarded(n_cap * 4)
    zk.fill_digests_buf_linear_gpu(dig, cap, to_dev(leaves), nl, ls, ch, h)
    assert intact(wd, max(n_dig, 1) * 4) and intact(wc, n_cap * 4)
    d, c = O.merkle(leaves, ls, ch, h)
    assert np.array_equal(to_np(cap).reshape(-1, 4), c)
    if n_dig:
        assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d)


@pytest.mark.parametrize("lg,rate,cols,cap,h", [(3, 1, 5, 1, 3), (9, 3, 19, 4, 0), (8, 2, 1, 10, 1)])
def test_commit_stays_in_bounds(lg, rate, cols, cap, h):
    c = O.field_data(lg * 31 + cols, cols << lg)
    N = 1 << (lg + rate)
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    wl, leaves = guarded(N * cols)
    wd, dig = guarded(max(n_dig, 1) * 4)
    wc, caps = guarded(n_cap * 4)
    zk.commit(0, zk.commit_job(lg, rate, cols, cap, h, to_dev(c), leaves, dig, caps))
    assert intact(wl, N * cols) and intact(wd, max(n_dig, 1) * 4) and intact(wc, n_cap * 4)
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    assert np.array_equal(to_np(leaves), rows)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
