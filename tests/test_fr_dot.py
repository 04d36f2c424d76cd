"""The Poseidon-BN128 dot products (zeknox_b200/csrc/bn254.cuh, host build of
the code the device runs): one Montgomery reduction of a five-product sum
equals five reduced products added, and both equal sum a_j b_j 2^-256 mod r,
canonical, at the bound (every operand r - 1) and on corner and random
operands."""
import os
import random
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "zeknox_b200", "csrc")
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001  # BN254 scalar field order
RINV = pow(1 << 256, -1, R)


@pytest.fixture(scope="module")
def fr_dot(tmp_path_factory):
    exe = tmp_path_factory.mktemp("fr") / "fr_dot"
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-I", CSRC, os.path.join(ROOT, "tests", "c", "fr_dot.cpp"), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(exe)


def test_dot_products_one_reduction_equal_five(fr_dot):
    corners = [0, 1, 2, R - 1, R - 2, (1 << 255) % R, (1 << 256) % R, (R - 1) // 2, 1 << 192, (1 << 192) - 1]
    rng = random.Random(11)
    cases = [[R - 1] * 10, [0] * 10, [R - 1, 1] * 5, [1, R - 1] * 5]
    for _ in range(300):
        cases.append([rng.choice(corners) for _ in range(10)])
    for _ in range(300):
        cases.append([rng.randrange(R) for _ in range(10)])
    text = "\n".join(" ".join("%064x" % v for v in c) for c in cases) + "\n"
    out = subprocess.run([fr_dot], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
    for c, line in zip(cases, out):
        one, five = (int(x, 16) for x in line.split())
        want = sum(c[2 * j] * c[2 * j + 1] for j in range(5)) * RINV % R
        assert one == want and five == want, c
    assert len([l for l in out if l]) == len(cases)
