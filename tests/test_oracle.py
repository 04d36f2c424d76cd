"""The CPU oracle against the reference's golden vectors and the math (no GPU).

Pins oracle/zk_oracle.c before it is trusted as the parity checker:
  * hashes: the reference's own known-answer tests (native/tests/tests.cu) and
    hash_one/hash_two of the reference CPU hashers (tests/golden/hash_ref.npz);
  * Merkle: the reference's fill_digests_buf_linear_cpu on seeded forests
    (tests/golden/merkle_ref.npz);
  * NTT family: the O(n^2) DFT definition with the reference's root table, and
    Plonky2's coset-LDE definition (wrappers/rust/tests/ntt.rs:332-479).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import HASHES, MERKLE_CASES, FULL_DIGESTS_MAX, merkle_seed, sha256

P = O.P


def test_roots_match_reference_table(kat):
    for k in range(33):
        assert O.omega(k) == kat["omega"][k]
        assert O.omega(k, inverse=True) == kat["omega_inv"][k]
    for k in range(1, 33):
        assert O.mul(kat["omega"][k], kat["omega"][k]) == kat["omega"][k - 1]
        assert O.mul(kat["omega"][k], kat["omega_inv"][k]) == 1
        assert O.mul(kat["domain_size_inv"][k], 1 << k) == 1


def test_keccak_kat(kat):
    data = np.array(kat["keccak_data"], dtype=np.uint64)
    for size in range(1, 7):
        out = np.zeros(4, dtype=np.uint64)  # <4 inputs leave the other limbs untouched
        O.hash_one(1, data[:size], out)
        assert [int(x) for x in out] == kat["keccak_expected"][size]


def test_poseidon_kat(kat):
    leaf = np.array(kat["poseidon_leaf"], dtype=np.uint64)
    for k in range(1, 10):
        assert [int(x) for x in O.hash_one(0, leaf[:k])] == kat["poseidon_expected"][k]


def test_poseidon2_monolith_kat(kat):
    assert [int(x) for x in O.hash_one(3, np.array(kat["poseidon2_input"], dtype=np.uint64))] == kat["poseidon2_expected"]
    assert [int(x) for x in O.hash_one(4, np.array(kat["monolith_input"], dtype=np.uint64))] == kat["monolith_expected"]


def test_poseidon_bn128_kat(kat):
    inp = np.array(kat["poseidon_bn128_input"], dtype=np.uint64)
    assert [int(x) for x in O.hash_one(2, inp)] == kat["poseidon_bn128_expected"]


@pytest.mark.parametrize("name", list(HASHES))
def test_tree4x7(kat, name):
    h = HASHES[name]
    lv = np.array(kat["tree4x7_leaves"], dtype=np.uint64)
    d = [O.hash_one(h, lv[7 * i:7 * i + 7]) for i in range(4)]
    n01, n23 = O.hash_two(h, d[0], d[1]), O.hash_two(h, d[2], d[3])
    got = [[int(x) for x in v] for v in d + [n01, n23, O.hash_two(h, n01, n23)]]
    assert got == kat["tree4x7_" + name]


@pytest.mark.parametrize("name", list(HASHES))
def test_hashes_vs_reference(hash_ref, name):
    h = HASHES[name]
    data = hash_ref["one_inputs"]
    for ln in range(1, 21):
        exp = hash_ref[name + "_one"][ln - 1]
        out = np.zeros(4, dtype=np.uint64)
        O.hash_one(h, data[20 * (ln - 1):20 * (ln - 1) + ln], out)
        assert np.array_equal(out, exp), (name, ln)
    pairs = data[400:464].reshape(8, 8)
    for i in range(8):
        assert np.array_equal(O.hash_two(h, pairs[i, :4], pairs[i, 4:]), hash_ref[name + "_two"][i])


@pytest.mark.parametrize("name", list(HASHES))
def test_merkle_vs_reference(merkle_ref, name):
    h = HASHES[name]
    for ci, (nl, ls, ch) in enumerate(MERKLE_CASES):
        key = "%s_%d_%d_%d" % (name, nl, ls, ch)
        leaves = O.field_data(merkle_seed(ci, h), nl * ls)
        dig, cap = O.merkle(leaves, ls, ch, h)
        assert np.array_equal(cap, merkle_ref[key + "_caps"]), key
        if nl <= FULL_DIGESTS_MAX:
            assert np.array_equal(dig, merkle_ref[key + "_digests"]), key
        else:
            assert sha256(dig) == merkle_ref[key + "_digests_sha256"].tobytes(), key


@pytest.mark.skipif(not O.ref_available(), reason="reference CPU library not built")
@pytest.mark.parametrize("name", list(HASHES))
def test_fresh_random_vs_reference_cpu(name):
    h = HASHES[name]
    for seed in range(5):
        leaves = O.field_data(77 + seed, 128 * 11)
        d1, c1 = O.merkle(leaves, 11, 2, h)
        d2, c2 = O.ref_merkle(leaves, 11, 2, h)
        assert np.array_equal(d1, d2) and np.array_equal(c1, c2)


@pytest.mark.parametrize("lg", range(1, 9))
def test_ntt_matches_dft_definition(lg):
    n = 1 << lg
    x = O.field_data(lg, 2 * n)
    fwd = O.batched_ntt(x, lg, 2)
    for b in range(2):
        assert np.array_equal(fwd[b * n:(b + 1) * n], O.dft_naive(x[b * n:(b + 1) * n]))
    inv = O.batched_ntt(fwd, lg, 2, inverse=True)
    assert np.array_equal(inv, x)


def test_coset_ntt_and_inverse_quirk():
    lg, n, g = 5, 32, 7
    x = O.field_data(5, n)
    scaled = np.array([O.mul(int(x[j]), pow(g, j, P)) for j in range(n)], dtype=np.uint64)
    assert np.array_equal(O.batched_ntt(x, lg, 1, with_coset=True), O.dft_naive(scaled))
    # inverse + coset: forward powers applied before 1/n (native/ntt/ntt.cu:137-143)
    y = O.dft_naive(x, inverse=True)
    ninv = pow(n, P - 2, P)
    exp = np.array([O.mul(O.mul(int(y[i]), pow(g, i, P)), ninv) for i in range(n)], dtype=np.uint64)
    assert np.array_equal(O.batched_ntt(x, lg, 1, inverse=True, with_coset=True), exp)


@pytest.mark.parametrize("lg,rate", [(1, 1), (3, 2), (6, 3), (8, 1)])
def test_lde_definition(lg, rate):
    n, N, g = 1 << lg, 1 << (lg + rate), 7
    c = O.field_data(100 + lg, 3 * n)
    out = O.batched_lde(c, lg, rate, 3, with_coset=True)
    w = O.omega(lg + rate)
    for b in range(3):
        for i in range(N):
            x = O.mul(g, pow(w, i, P))
            assert int(out[b * N + i]) == O.eval_poly(c[b * n:(b + 1) * n], x)
    # without coset: plain NTT of the zero-extended column
    out0 = O.batched_lde(c, lg, rate, 3, with_coset=False)
    for b in range(3):
        assert np.array_equal(out0[b * N:(b + 1) * N], O.dft_naive(np.concatenate([c[b * n:(b + 1) * n], np.zeros(N - n, np.uint64)])))


def test_transpose_rev_definition():
    lg, B = 5, 3
    x = O.field_data(9, B << lg)
    out = O.transpose_rev(x, lg, B)
    for i in range(1 << lg):
        r = int(format(i, "05b")[::-1], 2)
        for b in range(B):
            assert out[r * B + b] == x[b * (1 << lg) + i]
