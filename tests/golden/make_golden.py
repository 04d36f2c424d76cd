#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout that has the zeknox reference tree and its CPU library built
(``make -C oracle ref``)::

    python tests/golden/make_golden.py [--ref /path/to/zeknox]

Produces
  kat.json        known-answer vectors copied as data from the reference's own
                  tests (native/tests/tests.cu:164-173 Keccak, :204 Monolith,
                  :279-292 Poseidon, :425-428 Poseidon2, :492-501 Poseidon-BN128)
                  plus the 4-leaf x 7
                  trees of :241-274 / :338-375 / :451-489 hashed by the
                  reference CPU hashers, and the root tables of
                  native/ff/gl64_params.hpp.
  hash_ref.npz    hash_one for lengths 1..20 and hash_two on seeded inputs,
                  from the reference CPU hashers (oracle/_ref).
  merkle_ref.npz  fill_digests_buf_linear_cpu (the reference's own
                  native/merkle/merkle.cpp) on seeded leaves for every hash and
                  a spread of leaf counts, leaf sizes and cap heights.
"""
import argparse
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REPO_ROOT = ROOT
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HASHES = {"poseidon": 0, "keccak": 1, "poseidon2": 3, "monolith": 4, "poseidon_bn128": 2}

# (n_leaves, leaf_size, cap_height) per hash: special cases (caps == leaves,
# 2-leaf subtrees), odd leaf sizes, <= 4-element leaves and several levels.
MERKLE_CASES = [
    (4, 7, 0), (4, 7, 1), (4, 7, 2), (8, 5, 0), (16, 6, 2), (16, 4, 0), (16, 3, 1), (32, 9, 3), (64, 8, 0),
    (64, 13, 5), (256, 17, 2), (512, 84, 0), (1024, 12, 4), (4096, 7, 1), (2048, 135, 4),
]
FULL_DIGESTS_MAX = 1024  # larger trees store caps + sha256 of the digest bytes


def merkle_seed(case_index, hash_type):
    """Seed of the leaves of MERKLE_CASES[case_index] (regenerate with oracle.field_data)."""
    return 1000 + 31 * case_index + hash_type


def parse_u64_list(text):
    return [int(t.rstrip("uUlL"), 0) for t in re.findall(r"0x[0-9a-fA-F]+[uUlL]*|\b\d+[uUlL]*\b", text)]


def block_after(src, marker):
    i = src.index(marker)
    j = src.index("{", i)
    depth, k = 0, j
    while True:
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[j + 1:k]
        k += 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ZEKNOX_REFERENCE_DIR", os.path.join(REPO_ROOT, "..", "reference")),
                    help="the reference tree (default: $ZEKNOX_REFERENCE_DIR, else ../reference beside this repository)")
    args = ap.parse_args()
    tests = open(os.path.join(args.ref, "native/tests/tests.cu")).read()
    params = open(os.path.join(args.ref, "native/ff/gl64_params.hpp")).read()

    kat = {}
    # Keccak: data[6] and expected[7][4] (tests.cu:164-173)
    seg = tests[tests.index("TEST(LIBCUDA, keccak_test)"):]
    kat["keccak_data"] = parse_u64_list(block_after(seg, "u64 data[6]"))
    exp = parse_u64_list(block_after(seg, "expected[7][4]"))
    kat["keccak_expected"] = [exp[0:1] + [0, 0, 0]] + [exp[1 + 4 * i:5 + 4 * i] for i in range(6)]
    # Monolith 0..11 (tests.cu:203-204)
    seg = tests[tests.index("TEST(LIBCUDA, monolith_test1)"):]
    kat["monolith_input"] = parse_u64_list(block_after(seg, "u64 inp[12]"))
    kat["monolith_expected"] = parse_u64_list(block_after(seg, "expected[4]"))
    # Poseidon prefixes (tests.cu:279-292)
    seg = tests[tests.index("TEST(LIBCUDA, poseidon_test1)"):]
    kat["poseidon_leaf"] = parse_u64_list(block_after(seg, "u64 leaf[9]"))
    exp = parse_u64_list(block_after(seg, "expected[11][4]"))
    kat["poseidon_expected"] = [exp[0:1] + [0, 0, 0]] + [exp[1 + 4 * i:5 + 4 * i] for i in range(10)]
    # Poseidon2 Fibonacci (tests.cu:410-428)
    seg = tests[tests.index("TEST(LIBCUDA, poseidon2_test1)"):tests.index("TEST(LIBCUDA, poseidon2_test1)") + 1500]
    kat["poseidon2_input"] = [0, 1]
    for _ in range(10):
        kat["poseidon2_input"].append(kat["poseidon2_input"][-1] + kat["poseidon2_input"][-2])
    kat["poseidon2_expected"] = [int(x, 16) for x in re.findall(r"h1\[\d\] == (0x[0-9a-fA-F]+)", seg)]
    assert len(kat["poseidon2_expected"]) == 4
    # Poseidon-BN128 (tests.cu:492-501)
    seg = tests[tests.index("TEST(LIBCUDA, poseidonbn128_test1)"):]
    kat["poseidon_bn128_input"] = parse_u64_list(block_after(seg, "u64 inp[12]"))
    kat["poseidon_bn128_expected"] = parse_u64_list(block_after(seg, "expected[4]"))
    # 4 leaves x 7 test tree (tests.cu:241-244), hashed by the reference CPU hashers
    seg = tests[tests.index("TEST(LIBCUDA, monolith_test2)"):]
    leaves = parse_u64_list(block_after(seg, "u64 test_leaves[28]"))
    kat["tree4x7_leaves"] = leaves
    lv = np.array(leaves, dtype=np.uint64)
    for name, h in HASHES.items():
        d = [O.ref_hash_one(h, lv[7 * i:7 * i + 7]) for i in range(4)]
        n01 = O.ref_hash_two(h, d[0], d[1])
        n23 = O.ref_hash_two(h, d[2], d[3])
        root = O.ref_hash_two(h, n01, n23)
        kat["tree4x7_" + name] = [[int(x) for x in v] for v in d + [n01, n23, root]]
    # roots of unity (gl64_params.hpp:15-121)
    kat["omega"] = parse_u64_list(block_after(params, "OMEGA[33]"))
    kat["omega_inv"] = parse_u64_list(block_after(params, "OMEGA_INV[33]"))
    kat["domain_size_inv"] = parse_u64_list(block_after(params, "DOMAIN_SIZE_INV[33]"))
    kat["group_generator"] = 7
    # reference CPU agrees with its own KATs
    assert [int(x) for x in O.ref_hash_one(3, np.array(kat["poseidon2_input"], dtype=np.uint64))] == kat["poseidon2_expected"]
    assert [int(x) for x in O.ref_hash_one(2, np.array(kat["poseidon_bn128_input"], dtype=np.uint64))] == \
        kat["poseidon_bn128_expected"]
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)

    # single hashes
    out = {}
    rng_data = O.field_data(11, 20 * 20 + 64)
    for name, h in HASHES.items():
        ones = np.zeros((20, 4), dtype=np.uint64)
        for ln in range(1, 21):
            ones[ln - 1] = O.ref_hash_one(h, rng_data[20 * (ln - 1):20 * (ln - 1) + ln])
        out[name + "_one"] = ones
        pairs = rng_data[400:464].reshape(8, 8)
        twos = np.stack([O.ref_hash_two(h, pairs[i, :4], pairs[i, 4:]) for i in range(8)])
        out[name + "_two"] = twos
    out["one_inputs"] = rng_data
    np.savez_compressed(os.path.join(HERE, "hash_ref.npz"), **out)

    # Merkle forests
    out = {}
    for name, h in HASHES.items():
        for ci, (nl, ls, ch) in enumerate(MERKLE_CASES):
            leaves = O.field_data(merkle_seed(ci, h), nl * ls)
            dig, cap = O.ref_merkle(leaves, ls, ch, h)
            key = "%s_%d_%d_%d" % (name, nl, ls, ch)
            if nl <= FULL_DIGESTS_MAX:
                out[key + "_digests"] = dig
            else:
                out[key + "_digests_sha256"] = np.frombuffer(hashlib.sha256(dig.tobytes()).digest(), dtype=np.uint8)
            out[key + "_caps"] = cap
    np.savez_compressed(os.path.join(HERE, "merkle_ref.npz"), **out)
    print("wrote kat.json, hash_ref.npz, merkle_ref.npz")


if __name__ == "__main__":
    main()
