"""ctypes front end of the CPU oracle (test infrastructure only).

Two checkers live here:
  * ``liboracle.so`` -- this project's C restatement of the reference
    algorithms (zk_oracle.c), exact mod p = 2^64 - 2^32 + 1;
  * ``_ref/libzkref_cpu.so`` -- the reference's own CPU hash/Merkle sources
    compiled by ``make -C oracle ref`` (present when it was built next to the
    reference tree; it travels with the repository copy as a prebuilt file).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg use this
module; the library under test never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
P = 0xFFFFFFFF00000001

HASH_POSEIDON, HASH_KECCAK, HASH_POSEIDON_BN128, HASH_POSEIDON2, HASH_MONOLITH = 0, 1, 2, 3, 4

_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None
_ref = None


def _ptr(a):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        u64, u32, i = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int
        L.zko_mul.restype = L.zko_add.restype = L.zko_sub.restype = L.zko_pow.restype = u64
        L.zko_mul.argtypes = L.zko_add.argtypes = L.zko_sub.argtypes = L.zko_pow.argtypes = [u64, u64]
        L.zko_omega.restype = u64
        L.zko_omega.argtypes = [u32, i]
        L.zko_dft_naive.argtypes = [_u64p, _u64p, u32, i]
        L.zko_batched_ntt.argtypes = [_u64p, u32, u32, i, i, u64]
        L.zko_batched_lde.argtypes = [_u64p, _u64p, u32, u32, u32, i, i, u64]
        L.zko_transpose_rev.argtypes = [_u64p, _u64p, u32, u32]
        L.zko_hash_one.argtypes = [i, _u64p, u64, _u64p]
        L.zko_hash_two.argtypes = [i, _u64p, _u64p, _u64p]
        L.zko_permute.argtypes = [i, _u64p]
        L.zko_keccak_f.argtypes = [_u64p]
        L.zko_merkle.argtypes = [_u64p, _u64p, _u64p, u64, u64, u64, u64, u64, i]
        L.zko_eval_poly.restype = u64
        L.zko_eval_poly.argtypes = [_u64p, u64, u64]
        L.zko_num_threads.restype = i
        L.zko_set_num_threads.argtypes = [i]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libzkref_cpu.so"))


def ref():
    """The reference's own CPU hashers and Merkle builder (compiled from its sources)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libzkref_cpu.so")
        if not os.path.exists(path):
            raise RuntimeError("reference CPU library not built: run `make -C oracle ref`")
        R = ctypes.CDLL(path)
        u64, i = ctypes.c_uint64, ctypes.c_int
        R.zkref_hash_one.argtypes = [i, _u64p, u64, _u64p]
        R.zkref_hash_two.argtypes = [i, _u64p, _u64p, _u64p]
        R.fill_digests_buf_linear_cpu.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p] + [u64] * 6
        R.fill_digests_buf_linear_cpu.restype = None
        _ref = R
    return _ref


# ----------------------------------------------------------------- field / ntt

def mul(a, b):
    return lib().zko_mul(a, b)


def omega(lg, inverse=False):
    return lib().zko_omega(lg, int(inverse))


def dft_naive(x, inverse=False):
    x = np.ascontiguousarray(x, dtype=np.uint64)
    lg = int(x.size).bit_length() - 1
    out = np.empty_like(x)
    lib().zko_dft_naive(_ptr(x), _ptr(out), lg, int(inverse))
    return out


def batched_ntt(x, lg, batches, inverse=False, with_coset=False, coset_gen=7):
    """compute_batched_ntt semantics on a (batches, 2^lg) array; returns a new array."""
    a = np.array(x, dtype=np.uint64, copy=True).reshape(-1)
    assert a.size == batches << lg
    lib().zko_batched_ntt(_ptr(a), lg, batches, int(inverse), int(with_coset), coset_gen)
    return a


def batched_lde(x, lg, rate_bits, batches, inverse=False, with_coset=True, coset_gen=7):
    a = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1)
    assert a.size == batches << lg
    out = np.empty(batches << (lg + rate_bits), dtype=np.uint64)
    lib().zko_batched_lde(_ptr(out), _ptr(a), lg, rate_bits, batches, int(inverse), int(with_coset), coset_gen)
    return out


def eval_poly(coeffs, x):
    c = np.ascontiguousarray(coeffs, dtype=np.uint64)
    return lib().zko_eval_poly(_ptr(c), c.size, x)


def lde_rows(coeffs, lg, rate_bits, cols, coset_gen=7):
    """LDE then bit-reverse transpose: the leaf-major matrix a commit hashes."""
    ev = batched_lde(coeffs, lg, rate_bits, cols, with_coset=True, coset_gen=coset_gen)
    return transpose_rev(ev, lg + rate_bits, cols)


def transpose_rev(x, lg, batches):
    a = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1)
    out = np.empty_like(a)
    lib().zko_transpose_rev(_ptr(out), _ptr(a), lg, batches)
    return out


# ---------------------------------------------------------------------- hashes

def hash_one(h, data, out=None):
    d = np.ascontiguousarray(data, dtype=np.uint64)
    o = np.zeros(4, dtype=np.uint64) if out is None else out
    rc = lib().zko_hash_one(h, _ptr(d), d.size, _ptr(o))
    assert rc == 0
    return o


def hash_two(h, left, right):
    l = np.ascontiguousarray(left, dtype=np.uint64)
    r = np.ascontiguousarray(right, dtype=np.uint64)
    o = np.zeros(4, dtype=np.uint64)
    assert lib().zko_hash_two(h, _ptr(l), _ptr(r), _ptr(o)) == 0
    return o


def permute(h, state):
    s = np.array(state, dtype=np.uint64, copy=True)
    assert lib().zko_permute(h, _ptr(s)) == 0
    return s


def keccak_f(state):
    """Keccak-f[1600] of one 25-lane state; returns a new array."""
    s = np.array(state, dtype=np.uint64, copy=True)
    assert s.size == 25
    lib().zko_keccak_f(_ptr(s))
    return s


def merkle_sizes(n_leaves, cap_height):
    n_caps = 1 << cap_height
    return 2 * (n_leaves - n_caps), n_caps


def merkle(leaves, leaf_size, cap_height, h):
    """Linear Merkle forest; returns (digests (n_dig, 4), caps (n_cap, 4))."""
    lv = np.ascontiguousarray(leaves, dtype=np.uint64).reshape(-1)
    n_leaves = lv.size // leaf_size
    n_dig, n_cap = merkle_sizes(n_leaves, cap_height)
    dig = np.zeros((max(n_dig, 1), 4), dtype=np.uint64)
    cap = np.zeros((n_cap, 4), dtype=np.uint64)
    rc = lib().zko_merkle(_ptr(dig), _ptr(cap), _ptr(lv), n_dig, n_cap, n_leaves, leaf_size, cap_height, h)
    assert rc == 0
    return dig[:n_dig], cap


def ref_merkle(leaves, leaf_size, cap_height, h):
    lv = np.ascontiguousarray(leaves, dtype=np.uint64).reshape(-1)
    n_leaves = lv.size // leaf_size
    n_dig, n_cap = merkle_sizes(n_leaves, cap_height)
    dig = np.zeros((max(n_dig, 1), 4), dtype=np.uint64)
    cap = np.zeros((n_cap, 4), dtype=np.uint64)
    ref().fill_digests_buf_linear_cpu(dig.ctypes.data, cap.ctypes.data, lv.ctypes.data, n_dig, n_cap, n_leaves,
                                      leaf_size, cap_height, h)
    return dig[:n_dig], cap


def ref_hash_one(h, data):
    d = np.array(data, dtype=np.uint64, copy=True)
    o = np.zeros(4, dtype=np.uint64)
    assert ref().zkref_hash_one(h, _ptr(d), d.size, _ptr(o)) == 0
    return o


def ref_hash_two(h, left, right):
    l = np.array(left, dtype=np.uint64, copy=True)
    r = np.array(right, dtype=np.uint64, copy=True)
    o = np.zeros(4, dtype=np.uint64)
    assert ref().zkref_hash_two(h, _ptr(l), _ptr(r), _ptr(o)) == 0
    return o


def set_threads(n):
    lib().zko_set_num_threads(n)


def num_threads():
    return lib().zko_num_threads()


# ----------------------------------------------------------------- synthetic data

def field_data(seed, n):
    """Seeded field elements in [0, p): splitmix64 over counters seed*2^32 + k,
    values >= p folded by subtracting p.  Deterministic across numpy versions."""
    k = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64((seed << 32) & 0xFFFFFFFFFFFFFFFF) + (k + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return np.where(z >= np.uint64(P), z - np.uint64(P), z)


# ----------------------------------------------------------- field corner cases

# Operands at the edges of the lazily reduced arithmetic: 0 and small values,
# the 2^32 neighbourhood (EPS = 2^32 - 1 = 2^64 mod p), 2^63, the top of the
# canonical range (p - 2^32 and p - 1 = 2^64 - 2^32), and non-canonical words
# in [p, 2^64).
CORNERS = sorted({0, 1, 2, 3, 7, (1 << 31), (1 << 32) - 2, (1 << 32) - 1, 1 << 32, (1 << 32) + 1, (1 << 33) - 1,
                  (1 << 63) - 1, 1 << 63, (1 << 63) + 1, P - (1 << 32) - 1, P - (1 << 32), P - (1 << 32) + 1, P - 3,
                  P - 2, P - 1, P, P + 1, P + (1 << 31), (1 << 64) - (1 << 31), (1 << 64) - 3, (1 << 64) - 2,
                  (1 << 64) - 1})
CANONICAL_CORNERS = [v for v in CORNERS if v < P]


def field_ops_expected(a, b, c):
    """Exact values of the device self-test operations (ZK_SELFTEST_OPS rows,
    include/zeknox_b200.h) for operand arrays a, b, c of any 64-bit words;
    Python integers, so the arithmetic is the definition mod p."""
    rows = [[] for _ in range(34)]
    for x, y, z in zip((int(v) for v in a), (int(v) for v in b), (int(v) for v in c)):
        xc, yc = x % P, y % P
        lo28 = (1 << 28) - 1
        vals = [
            (xc + yc) % P, (xc - yc) % P, (xc + yc) % P,
            x * y % P, x * y % P, x * y % P, x * x % P, x * x % P,
            (x * y + z) % P, (x * y + z) % P, pow(x, 7, P), pow(x, 7, P),
            x * pow(2, z % 192, P) % P, (x + yc) % P,
            4 * (x * y + y * z + z * x) % P, 4 * (x * y + y * z + z * x) % P,
            (x + 5 * y + 6 * z) % P, (4 * (41 * x + 39 * y + 34 * z) + yc) % P,
            ((x & lo28) + ((y & lo28) << 22) + ((z & lo28) << 44)) % P,
            (x + (y << 64)) % P, (x + ((y & 0xFFFFFFFF) << 64)) % P, x * (1 << (y % 64)) % P,
            (x + y) % P, (x - y) % P,
        ] + [x * (1 << e) % P for e in (1, 24, 31, 32, 60, 63, 64, 72, 84, 95)]
        for k, v in enumerate(vals):
            rows[k].append(v)
    return np.array(rows, dtype=np.uint64)
