"""Field corner cases through every product path, bit-exact against the oracle.

The device arithmetic keeps lanes lazily reduced and takes its rare carry,
borrow and wrap branches only near the field's edges (0, p - 1, the 2^32
neighbourhood, 2^64 - 2^32, non-canonical words in [p, 2^64)), which seeded
uniform data reaches about once in 2^32 operations.  Real Plonky2 witnesses
are full of zeros and p - 1.  Here the operands are chosen:
  * every device primitive on every triple of corner values
    (zeknox_field_selftest) against exact integer arithmetic;
  * whole permutations (one thread and the cooperative form) on corner states,
    canonical and not, against the oracle's permutations;
  * NTT / iNTT / coset / LDE on columns of corner values;
  * Merkle forests of corner leaves for all five hashes, including short
    leaves and Keccak's copied-through leaves;
  * fused commits whose leaves are corner values (constant polynomials), from
    coefficients and from values.
"""
import itertools

import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import HASHES, empty_dev, to_dev, to_np

pytestmark = pytest.mark.gpu

P = O.P
CORNERS = np.array(O.CORNERS, dtype=np.uint64)
CANON = np.array(O.CANONICAL_CORNERS, dtype=np.uint64)


def _pick(values, n, seed):
    return np.random.default_rng(seed).choice(values, size=n)


def test_field_primitives_on_all_corner_triples():
    trip = np.array(list(itertools.product(O.CORNERS, repeat=3)), dtype=np.uint64)
    rnd = np.stack([O.field_data(900 + k, 4096) for k in range(3)], axis=1)
    # uniform words over all of [0, 2^64), non-canonical ones included
    wide = np.random.default_rng(901).integers(0, 1 << 64, size=(4096, 3), dtype=np.uint64)
    ops = np.concatenate([trip, rnd, wide])
    a, b, c = (np.ascontiguousarray(ops[:, k]) for k in range(3))
    n = a.size
    out = torch.full((zk.SELFTEST_OPS * n,), -1, dtype=torch.int64, device="cuda")
    zk.field_selftest(0, to_dev(a), to_dev(b), to_dev(c), out)
    got = to_np(out).reshape(zk.SELFTEST_OPS, n)
    exp = O.field_ops_expected(a, b, c)
    for k in range(zk.SELFTEST_OPS):
        bad = np.nonzero(got[k] != exp[k])[0]
        assert bad.size == 0, "op %d: %d mismatches, first at a=%d b=%d c=%d: got %d want %d" % (
            k, bad.size, a[bad[0]], b[bad[0]], c[bad[0]], got[k][bad[0]], exp[k][bad[0]])


def _corner_states(width, seed, canonical):
    vals = CANON if canonical else CORNERS
    fixed = [np.zeros(width, np.uint64), np.full(width, P - 1, np.uint64), np.full(width, P - (1 << 32), np.uint64),
             np.full(width, (1 << 32) - 1, np.uint64), np.full(width, 1 << 32, np.uint64),
             np.array([0, P - 1] * (width // 2) + [0] * (width % 2), np.uint64),
             np.array([P - 1, 1] * (width // 2) + [P - 1] * (width % 2), np.uint64)]
    if not canonical:
        fixed += [np.full(width, (1 << 64) - 1, np.uint64), np.full(width, P, np.uint64),
                  np.array([P, (1 << 64) - 1] * (width // 2) + [P] * (width % 2), np.uint64)]
    picked = _pick(vals, 512 * width, seed).reshape(512, width)
    one_hot = np.zeros((len(vals) * width, width), np.uint64)
    for k, v in enumerate(vals):
        for j in range(width):
            one_hot[k * width + j, j] = v
    return np.concatenate([np.stack(fixed), picked, one_hot])


@pytest.mark.parametrize("name,coop", [("poseidon", False), ("poseidon", True), ("poseidon2", False),
                                       ("poseidon2", True), ("monolith", False), ("poseidon_bn128", False)])
def test_permutation_on_corner_states(name, coop):
    h = HASHES[name]
    # lanes are any 64-bit representative for the Goldilocks permutations; the
    # BN128 one takes canonical lanes (as its reference does)
    states = _corner_states(12, 910 + h, canonical=(h == zk.HASH_POSEIDON_BN128))
    t = to_dev(states.reshape(-1))
    zk.permute(0, t, h, cooperative=coop)
    got = to_np(t).reshape(-1, 12)
    canon = np.where(states >= np.uint64(P), states - np.uint64(P), states)
    for i in range(states.shape[0]):
        assert np.array_equal(got[i], O.permute(h, canon[i])), (name, coop, i, [int(v) for v in states[i]])


def test_keccak_f_on_corner_states():
    states = _corner_states(25, 920, canonical=False)
    t = to_dev(states.reshape(-1))
    zk.permute(0, t, zk.HASH_KECCAK)
    got = to_np(t).reshape(-1, 25)
    for i in range(states.shape[0]):
        assert np.array_equal(got[i], O.keccak_f(states[i])), i


def _corner_columns(lg, seed):
    n = 1 << lg
    cols = [np.zeros(n, np.uint64), np.full(n, P - 1, np.uint64), np.tile(np.array([0, P - 1], np.uint64), n // 2),
            np.tile(np.array([P - 1, 1], np.uint64), n // 2), np.full(n, P - (1 << 32), np.uint64),
            np.full(n, (1 << 32) - 1, np.uint64), _pick(CANON, n, seed), _pick(CANON, n, seed + 1)]
    return np.concatenate(cols)


@pytest.mark.parametrize("lg", [1, 4, 10, 13, 16])
@pytest.mark.parametrize("inverse,coset", [(False, False), (True, False), (False, True), (True, True)])
def test_ntt_on_corner_columns(lg, inverse, coset):
    x = _corner_columns(lg, 930 + lg)
    b = x.size >> lg
    t = to_dev(x)
    zk.ntt_batch(0, t, lg, b, with_coset=coset, inverse=inverse)
    assert np.array_equal(to_np(t), O.batched_ntt(x, lg, b, inverse=inverse, with_coset=coset))


@pytest.mark.parametrize("lg,rate", [(2, 1), (9, 3), (12, 2), (15, 3)])
def test_lde_on_corner_columns(lg, rate):
    c = _corner_columns(lg, 940 + lg)
    b = c.size >> lg
    out = torch.zeros(b << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_batch(0, out, to_dev(c), lg, b, rate)
    assert np.array_equal(to_np(out), O.batched_lde(c, lg, rate, b))
    rows = torch.zeros_like(out)
    zk.lde_rows(0, rows, to_dev(c), lg, rate, b)
    assert np.array_equal(to_np(rows), O.lde_rows(c, lg, rate, b))


def _corner_leaves(nl, ls, seed):
    fixed = [np.zeros(ls, np.uint64), np.full(ls, P - 1, np.uint64), np.full(ls, P - (1 << 32), np.uint64),
             np.full(ls, (1 << 32) - 1, np.uint64), np.full(ls, 1 << 32, np.uint64),
             np.array([0, P - 1] * ls, np.uint64)[:ls], np.array([P - 1, 0] * ls, np.uint64)[:ls]]
    rows = [fixed[i % len(fixed)] for i in range(nl // 2)]
    rest = _pick(CANON, (nl - len(rows)) * ls, seed).reshape(-1, ls)
    return np.concatenate([np.stack(rows), rest]).reshape(-1)


FOREST_SHAPES = [(1 << 10, 135, 2), (1 << 12, 8, 0), (1 << 11, 84, 3), (1 << 9, 4, 1), (1 << 9, 3, 2),
                 (1 << 10, 1, 0), (1 << 14, 12, 4), (1 << 8, 16, 8)]
# Poseidon-BN128 is ~30x slower per permutation: its forests take the shapes of
# at most 2^16 words
FOREST_CASES = [(name, *shape) for name in HASHES for shape in FOREST_SHAPES
                if name != "poseidon_bn128" or shape[0] * shape[1] <= (1 << 16)]


@pytest.mark.parametrize("name,nl,ls,ch", FOREST_CASES)
def test_merkle_on_corner_leaves(name, nl, ls, ch):
    h = HASHES[name]
    leaves = _corner_leaves(nl, ls, 950 + ls)
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    dig, cap = empty_dev(n_dig * 4), empty_dev(n_cap * 4)
    zk.fill_digests_buf_linear_gpu(dig, cap, to_dev(leaves), nl, ls, ch, h)
    torch.cuda.synchronize()
    d2, c2 = O.merkle(leaves, ls, ch, h)
    # (Keccak copies leaves of < 4 words into their digests and leaves the
    # other words as they were: zero here and in the oracle's buffer)
    assert np.array_equal(to_np(cap).reshape(-1, 4), c2)
    assert np.array_equal(to_np(dig)[:n_dig * 4].reshape(-1, 4), d2)


@pytest.mark.parametrize("name", list(HASHES))
@pytest.mark.parametrize("values", [False, True])
def test_commit_with_corner_leaves(name, values):
    """A constant polynomial evaluates to its constant everywhere, so columns
    whose only coefficient is a corner value give leaves made of corner values
    (and, from values, constant value columns give the same)."""
    h = HASHES[name]
    lg, rate = (7, 2) if h == zk.HASH_POSEIDON_BN128 else (11, 3)
    consts = np.concatenate([CANON, CANON[::-1]])
    cols = consts.size
    n = 1 << lg
    inp = np.zeros(cols << lg, np.uint64)
    if values:
        inp[:] = np.repeat(consts, n)
    else:
        inp[::n] = consts
    coeffs = np.zeros(cols << lg, np.uint64)
    coeffs[::n] = consts
    N = n << rate
    leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, 3)
    dig, caps = empty_dev(n_dig * 4), empty_dev(n_cap * 4)
    job = zk.commit_job(lg, rate, cols, 3, h, to_dev(inp), leaves, dig, caps, input_is_values=values)
    zk.commit(0, job)
    rows = O.lde_rows(coeffs, lg, rate, cols)
    assert np.array_equal(rows.reshape(N, cols), np.tile(consts, (N, 1)))
    assert np.array_equal(to_np(leaves), rows)
    d, c = O.merkle(rows, cols, 3, h)
    assert np.array_equal(to_np(caps).reshape(-1, 4), c)
    assert np.array_equal(to_np(dig)[:n_dig * 4].reshape(-1, 4), d)
