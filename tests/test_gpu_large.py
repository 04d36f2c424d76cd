"""Sizes past 2^31 elements (the reference indexes with 32-bit ints there and
overflows) checked through size-independent properties: spot evaluations of
the LDE polynomial at sampled rows, the transpose's index map at sampled
positions (the last ones included), and the Merkle layout's own relations
(leaf digest = hash of the leaf row, node = hash of its two children, cap =
hash of the subtree's top two nodes) at sampled nodes.  About 40 GB of HBM."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O

pytestmark = pytest.mark.gpu
P = O.P
G = 7  # coset shift


def rev(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2) if bits else 0


def u64(t):
    return t.cpu().numpy().view(np.uint64)


def sample(rng, hi, k, edges=True):
    s = set(int(v) for v in rng.integers(0, hi, size=k))
    if edges:
        s |= {0, hi - 1}
    return sorted(s)


def test_transpose_rev_past_2_31_elements():
    lg, cols = 28, 9  # 2.4 G elements, 19.3 GB each way
    n = 1 << lg
    inp = torch.randint(0, 1 << 62, (cols * n,), dtype=torch.int64, device="cuda")
    out = torch.empty_like(inp)
    zk.transpose_rev_batch(0, out, inp, lg, cols)
    torch.cuda.synchronize()
    rng = np.random.default_rng(5)
    ii = sample(rng, n, 2048)
    bb = [int(b) for b in rng.integers(0, cols, size=len(ii))]
    bb[-1] = cols - 1
    src = torch.tensor([b * n + i for i, b in zip(ii, bb)], device="cuda")
    dst = torch.tensor([rev(i, lg) * cols + b for i, b in zip(ii, bb)], device="cuda")
    assert torch.equal(out[dst], inp[src])
    del inp, out


def test_lde_past_2_31_outputs():
    lg, rate, cols = 25, 3, 8  # 2^31 output elements (16 GB)
    n, N = 1 << lg, 1 << (lg + rate)
    coeffs = torch.randint(0, 1 << 62, (cols * n,), dtype=torch.int64, device="cuda")
    out = torch.empty(cols * N, dtype=torch.int64, device="cuda")
    zk.lde_batch(0, out, coeffs, lg, cols, rate)
    torch.cuda.synchronize()
    c = u64(coeffs).reshape(cols, n)
    w = O.omega(lg + rate)
    rng = np.random.default_rng(6)
    rows = sample(rng, N, 6)
    for j, i in enumerate(rows):
        b = cols - 1 if j % 2 else j % cols
        x = G * pow(w, i, P) % P
        assert int(u64(out[b * N + i:b * N + i + 1])[0]) == O.eval_poly(c[b], x), (b, i)
    del coeffs, out


@pytest.mark.parametrize("h", [3, 1])
def test_commit_past_2_31_leaf_elements(h):
    """Fused LDE -> leaf rows -> forest with 2^28 leaves x 8 (2^31 row
    elements): sampled rows are evaluations, sampled leaves and nodes hash
    to what the layout says, and the caps close the subtrees."""
    lg, rate, cols, cap = 25, 3, 8, 4
    n, N = 1 << lg, 1 << (lg + rate)
    coeffs = torch.randint(0, 1 << 62, (cols * n,), dtype=torch.int64, device="cuda")
    rows = torch.empty(cols * N, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
    caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
    zk.commit(0, zk.commit_job(lg, rate, cols, cap, h, coeffs, rows, dig, caps))
    torch.cuda.synchronize()
    c = u64(coeffs).reshape(cols, n)
    w = O.omega(lg + rate)
    rng = np.random.default_rng(7 + h)
    L = N >> cap            # leaves per subtree
    D = 2 * L - 2           # digests per subtree

    def digest(k, idx):
        return u64(dig[4 * (k * D + idx):4 * (k * D + idx) + 4])

    # rows: evaluations at g * w_N^rev(r); leaf digests: the hash of the row
    for r in sample(rng, N, 3):
        row = u64(rows[r * cols:(r + 1) * cols])
        x = G * pow(w, rev(r, lg + rate), P) % P
        assert [int(v) for v in row] == [O.eval_poly(c[b], x) for b in range(cols)], r
        k, i = divmod(r, L)
        assert np.array_equal(digest(k, L - 2 + i), O.hash_one(h, row)), r
    # internal nodes: a level of m nodes starts at m - 2; node j's children are
    # nodes 2j and 2j + 1 of the level of 2m nodes, which starts at 2m - 2
    for t in range(24):
        k = int(rng.integers(0, n_cap)) if t else n_cap - 1
        m = 1 << int(rng.integers(1, L.bit_length() - 1))
        j = int(rng.integers(0, m)) if t else m - 1
        left = (2 * m - 2) + 2 * j
        assert np.array_equal(digest(k, m - 2 + j), O.hash_two(h, digest(k, left), digest(k, left + 1))), (k, m, j)
    for k in (0, n_cap - 1):
        assert np.array_equal(u64(caps[4 * k:4 * k + 4]), O.hash_two(h, digest(k, 0), digest(k, 1))), k
    del coeffs, rows, dig, caps


@pytest.mark.parametrize("lg,b", [(24, 4), (22, 16)])
def test_ntt_round_trip_large(lg, b):
    """compute_batched_ntt then its inverse is the identity (2^24-point transforms)."""
    x = torch.randint(0, 1 << 62, (b << lg,), dtype=torch.int64, device="cuda")
    y = x.clone()
    zk.ntt_batch(0, y, lg, b)
    assert not torch.equal(x, y)
    zk.intt_batch(0, y, lg, b)
    assert torch.equal(x, y)


def test_lde_rows_additive_at_headline_size():
    """The fused LDE is linear: rows(a + b) = rows(a) + rows(b) mod p, at the
    headline shape (256 columns x 2^15, rate 3)."""
    lg, rate, cols = 15, 3, 256
    N = 1 << (lg + rate)
    a = torch.randint(0, 1 << 62, (cols << lg,), dtype=torch.int64, device="cuda")
    b = torch.randint(0, 1 << 62, (cols << lg,), dtype=torch.int64, device="cuda")
    p = np.uint64(P)

    def add(x, y):
        s = x + y
        return np.where((s < x) | (s >= p), s - p, s)

    c = torch.from_numpy(add(u64(a), u64(b)).view(np.int64)).cuda()
    rows = [torch.empty(cols * N, dtype=torch.int64, device="cuda") for _ in range(3)]
    for r, x in zip(rows, (a, b, c)):
        zk.lde_rows(0, r, x, lg, rate, cols)
    torch.cuda.synchronize()
    with np.errstate(over="ignore"):
        assert np.array_equal(u64(rows[2]), add(u64(rows[0]), u64(rows[1])))
