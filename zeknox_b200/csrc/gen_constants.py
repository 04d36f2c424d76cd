#!/usr/bin/env python3
"""Generate ``zk_constants.h``: every fixed table the Goldilocks commit path needs.

Bit-exactness with zeknox forces these tables to hold the same *values* as the
reference (they are Plonky2's published parameters); the layout, names and the
way they are produced are this project's own:

* Goldilocks roots of unity (``ZK_OMEGA``/``ZK_OMEGA_INV``/``ZK_DOMAIN_SIZE_INV``)
  are *derived* here from Plonky2's 2^32-th root of unity 1753635133440165772
  and the multiplicative generator 7 (zeknox scripts/configs/gl64.json), by
  repeated squaring. When the reference tree is present they are cross-checked
  against native/ff/gl64_params.hpp:15-121.
* Keccak-f[1600] round constants, rotation offsets and the pi lane walk are
  *derived* from the Keccak specification (LFSR rc(t), offsets (t+1)(t+2)/2) and
  cross-checked against native/keccak/keccak.cu:16-37.
* Poseidon's sparse partial-round tables (first-round constants, per-round
  scalars, the dense initial matrix and the per-round row/column vectors) are
  *derived* from the MDS matrix and round constants (derive_poseidon_fast) and
  cross-checked against native/poseidon/poseidon.hpp:38-801.
* BN254 Montgomery parameters (modulus limbs, R^2 mod r, -r^-1) are *derived*
  from the field order and cross-checked against native/poseidon/element_bn128.cu;
  the Poseidon-BN128 round constants and matrices (iden3's t = 5 parameters in
  Montgomery form) are read as numbers from
  native/poseidon/poseidon_bn128_constants.h.
* Poseidon round constants (native/poseidon/poseidon.hpp:803-1164, 360 values,
  MDS circulant row and diagonal :35-36), Poseidon2 round constants and internal
  diagonal (native/poseidon2/poseidon2.cu:8-59) and Monolith round constants and
  circulant row (native/monolith/monolith.cu:12-106) are parameter data with no
  closed form here; they are read as numbers from the reference sources.

Run from anywhere:  python zeknox_b200/csrc/gen_constants.py [--ref <zeknox root>]
The output is committed, so the build never needs the reference tree.
"""
import argparse
import os
import re
import sys

P = 0xFFFFFFFF00000001
REPO_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
ROOT_2_32 = 1753635133440165772  # primitive 2^32-th root of unity (Plonky2)
GENERATOR = 7


def derive_roots():
    omega = [0] * 33
    omega[32] = ROOT_2_32
    for k in range(32, 0, -1):
        omega[k - 1] = omega[k] * omega[k] % P
    assert omega[0] == 1 and omega[1] == P - 1
    omega_inv = [pow(w, P - 2, P) for w in omega]
    size_inv = [pow(1 << k, P - 2, P) for k in range(33)]
    return omega, omega_inv, size_inv


def derive_keccak():
    # round constants: RC[i] bit (2^j - 1) = rc(j + 7i), rc from the degree-8 LFSR
    def rc_bit(t):
        if t % 255 == 0:
            return 1
        r = 1
        for _ in range(t % 255):
            r <<= 1
            if r & 0x100:
                r ^= 0x171
        return r & 1

    rndc = []
    for i in range(24):
        v = 0
        for j in range(7):
            if rc_bit(j + 7 * i):
                v |= 1 << ((1 << j) - 1)
        rndc.append(v)
    # rho offsets and pi walk starting at lane (x, y) = (1, 0)
    rotc, piln = [], []
    x, y = 1, 0
    for t in range(24):
        rotc.append(((t + 1) * (t + 2) // 2) % 64)
        x, y = y, (2 * x + 3 * y) % 5
        piln.append(x + 5 * y)
    return rndc, rotc, piln


def _numbers(text):
    return [int(tok.rstrip("uUlL"), 0) for tok in re.findall(r"0x[0-9a-fA-F]+[uUlL]*|\b\d+[uUlL]*\b", text)]


def _block(src, start_pat):
    m = re.search(start_pat, src)
    if not m:
        raise SystemExit("pattern not found: " + start_pat)
    i = src.index("{", m.end() - 1)
    depth, j = 0, i
    while True:
        c = src[j]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return src[i + 1:j]
        j += 1


# BN254 scalar field order (the Poseidon-BN128 hash works over it)
BN_R = 21888242871839275222246405745257275088548364400416034343698204186575808495617


def derive_bn254():
    """Montgomery parameters of F_r with R = 2^256: r's 32-bit limbs,
    R^2 mod r (to enter Montgomery form) and -r^-1 mod 2^32."""
    limbs32 = [(BN_R >> (32 * i)) & 0xFFFFFFFF for i in range(8)]
    r2 = (1 << 512) % BN_R
    nprime32 = (-pow(BN_R, -1, 1 << 32)) % (1 << 32)
    return limbs32, r2, nprime32


def _limbs64(x):
    return [(x >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)]


def read_reference(ref):
    nat = os.path.join(ref, "native")
    with open(os.path.join(nat, "poseidon/poseidon.hpp")) as f:
        pos = f.read()
    with open(os.path.join(nat, "poseidon2/poseidon2.cu")) as f:
        p2 = f.read()
    with open(os.path.join(nat, "monolith/monolith.cu")) as f:
        mono = f.read()
    with open(os.path.join(nat, "ff/gl64_params.hpp")) as f:
        params = f.read()
    with open(os.path.join(nat, "keccak/keccak.cu")) as f:
        kec = f.read()
    with open(os.path.join(nat, "poseidon/poseidon_bn128_constants.h")) as f:
        bnc = f.read()
    with open(os.path.join(nat, "poseidon/element_bn128.cu")) as f:
        bne = f.read()
    with open(os.path.join(nat, "poseidon/poseidon_bn128.cu")) as f:
        bnp = f.read()

    out = {}
    out["poseidon_rc"] = _numbers(_block(pos, r"ALL_ROUND_CONSTANTS\[[^\]]*\]\s*=\s*{"))
    out["poseidon_circ"] = _numbers(_block(pos, r"MDS_MATRIX_CIRC\[12\]\s*=\s*{"))
    out["poseidon_diag"] = _numbers(_block(pos, r"MDS_MATRIX_DIAG\[12\]\s*=\s*{"))
    out["fast_first"] = _numbers(_block(pos, r"FAST_PARTIAL_FIRST_ROUND_CONSTANT\[12\]\s*=\s*{"))
    out["fast_k"] = _numbers(_block(pos, r"FAST_PARTIAL_ROUND_CONSTANTS\[N_PARTIAL_ROUNDS\]\s*=\s*{"))
    out["fast_v"] = _numbers(_block(pos, r"FAST_PARTIAL_ROUND_VS\[N_PARTIAL_ROUNDS\]\[11\]\s*=\s*{"))
    out["fast_w"] = _numbers(_block(pos, r"FAST_PARTIAL_ROUND_W_HATS\[N_PARTIAL_ROUNDS\]\[11\]\s*=\s*{"))
    out["fast_init"] = _numbers(_block(pos, r"FAST_PARTIAL_ROUND_INITIAL_MATRIX\[11\]\[11\]\s*=\s*{"))
    # the #ifdef'd declarations share one initializer: take the first brace after the CPU name
    diag_start = p2.index("const u64 MATRIX_DIAG_12_GOLDILOCKS[12] = {")
    out["p2_diag"] = _numbers(_block(p2[diag_start:], r"\[12\]\s*=\s*{"))
    rc_start = p2.index("const u64 RC12[360] = {")
    out["p2_rc"] = _numbers(_block(p2[rc_start:], r"\[360\]\s*=\s*{"))
    mrc_start = mono.index("const u64 MONOLITH_ROUND_CONSTANTS[N_ROUNDS + 1][SPONGE_WIDTH] = {")
    mrc = _block(mono[mrc_start:], r"\]\s*=\s*{")
    out["mono_rc"] = _numbers(mrc)
    mm_start = mono.index("const u32 MONOLITH_MAT_12[SPONGE_WIDTH][SPONGE_WIDTH] = {")
    out["mono_mat"] = _numbers(_block(mono[mm_start:], r"\]\s*=\s*{"))
    out["omega"] = _numbers(_block(params, r"OMEGA\[33\]\s*=\s*{"))
    out["omega_inv"] = _numbers(_block(params, r"OMEGA_INV\[33\]\s*=\s*{"))
    out["size_inv"] = _numbers(_block(params, r"DOMAIN_SIZE_INV\[33\]\s*=\s*{"))
    out["k_rndc"] = _numbers(_block(kec, r"keccakf_rndc\)\[24\]\s*=\s*{"))
    out["k_rotc"] = _numbers(_block(kec, r"keccakf_rotc\)\[24\]\s*=\s*{"))
    out["k_piln"] = _numbers(_block(kec, r"keccakf_piln\)\[24\]\s*=\s*{"))
    # Poseidon-BN128 (t = 5): round constants, sparse partial-round matrices,
    # full-round matrix M and the pre-partial matrix P, all 4 x u64 little-endian
    # limbs in Montgomery form (native/poseidon/poseidon_bn128_constants.h:16-737)
    out["bn_c"] = _numbers(_block(bnc, r"C\[100\]\[4\]\s*=\s*{"))
    out["bn_s"] = _numbers(_block(bnc, r"S\[540\]\[4\]\s*=\s*{"))
    out["bn_m"] = _numbers(_block(bnc, r"M\[5\]\[5\]\[4\]\s*=\s*{"))
    out["bn_p"] = _numbers(_block(bnc, r"P\[5\]\[5\]\[4\]\s*=\s*{"))
    out["bn_r2"] = _numbers(_block(bne, r"rSquare\[4\]\s*#endif\s*=\s*{"))
    out["bn_modulus"] = [int(x) for x in re.findall(r"madd3\(m, (\d+)u", bne)[:1]] + \
        [int(x) for x in re.findall(r"madd2\(m, (\d+)u", bne)[:2]]
    out["bn_m0"] = [int(x) for x in re.findall(r"madd0\(m, (\d+)u", bne)[:1]]
    out["bn_np64"] = [int(x) for x in re.findall(r"m = c\[0\] \* (\d+)u", bne)[:1]]
    out["bn_rounds_p"] = _numbers(_block(bnp, r"NROUNDSP\[16\]\s*=\s*{"))
    return out


def _mat_mul(a, b):
    return [[sum(a[i][k] * b[k][j] for k in range(len(b))) % P for j in range(len(b[0]))] for i in range(len(a))]


def _mat_vec(a, v):
    return [sum(a[i][k] * v[k] for k in range(len(v))) % P for i in range(len(a))]


def _mat_inv(a):
    n = len(a)
    m = [list(row) + [int(i == j) for j in range(n)] for i, row in enumerate(a)]
    for c in range(n):
        piv = next(r for r in range(c, n) if m[r][c])
        m[c], m[piv] = m[piv], m[c]
        inv = pow(m[c][c], P - 2, P)
        m[c] = [x * inv % P for x in m[c]]
        for r in range(n):
            if r != c and m[r][c]:
                f = m[r][c]
                m[r] = [(x - f * y) % P for x, y in zip(m[r], m[c])]
    return [row[n:] for row in m]


def poseidon_mds_matrix(circ, diag):
    return [[(circ[(j - r) % 12] + (diag[r] if r == j else 0)) % P for j in range(12)] for r in range(12)]


def derive_poseidon_fast(rc, circ, diag, n_full_half=4, n_partial=22):
    """Partial rounds of Poseidon in the sparse-matrix form of the Poseidon
    paper (Grassi et al., eprint 2019/458, appendix B), derived here from the
    MDS matrix and round constants.

    The 22 partial rounds  x <- M * S0(x + c_r)  (S0: S-box on lane 0 only)
    equal, exactly:
        x <- x + first                       (12 constants)
        x[1..11] <- init * x[1..11]          (11 x 11)
        for r in 0..21:
            x[0] <- S(x[0]) + k[r]            (k[21] = 0)
            x[0], x[i] <- m00 * x[0] + sum_i w[r][i] * x[i],  x[i] + v[r][i] * x[0]
    Derivation: constants are carried backwards through each M (M^-1 c), lane
    0 of the carry stays in its round as k, lanes 1..11 pass through S0; each
    M is factored M = B * D with D = diag(1, N^) acting on lanes 1..11 only
    (commutes with S0 and with k) and B sparse (first row [m00, N^-T w],
    first column v), D merged into the previous round's matrix."""
    M = poseidon_mds_matrix(circ, diag)
    Minv = _mat_inv(M)
    m00 = M[0][0]
    w = M[0][1:]
    v = [M[i][0] for i in range(1, 12)]
    Mh = [row[1:] for row in M[1:]]
    # constants
    base = 12 * n_full_half
    cr = [rc[base + 12 * r: base + 12 * r + 12] for r in range(n_partial)]
    k = [0] * n_partial
    carry = [0] * 12
    for r in range(n_partial - 1, 0, -1):
        d = [(a + b) % P for a, b in zip(cr[r], carry)]
        u = _mat_vec(Minv, d)
        k[r - 1] = u[0]
        carry = [0] + u[1:]
    first = [(a + b) % P for a, b in zip(cr[0], carry)]
    # matrices, last round first: N^_r = Mh^(R - r), v_r = Mh^(R-1-r) v, w_r = N^_r^-T w
    ws, vs = [None] * n_partial, [None] * n_partial
    Nh = Mh
    vr = v
    for r in range(n_partial - 1, -1, -1):
        NhT_inv = _mat_inv([list(col) for col in zip(*Nh)])
        ws[r] = _mat_vec(NhT_inv, w)
        vs[r] = vr
        if r:
            vr = _mat_vec(Nh, v)
            Nh = _mat_mul(Nh, Mh)
    init = Nh

    def sbox(x):
        return pow(x, 7, P)

    def naive(x):
        for r in range(n_partial):
            x = [(a + b) % P for a, b in zip(x, cr[r])]
            x[0] = sbox(x[0])
            x = _mat_vec(M, x)
        return x

    def fast(x):
        x = [(a + b) % P for a, b in zip(x, first)]
        x = [x[0]] + _mat_vec(init, x[1:])
        for r in range(n_partial):
            x[0] = (sbox(x[0]) + k[r]) % P
            x0 = (m00 * x[0] + sum(a * b for a, b in zip(ws[r], x[1:]))) % P
            x = [x0] + [(xi + vi * x[0]) % P for xi, vi in zip(x[1:], vs[r])]
        return x

    import random
    rnd = random.Random(1)
    for _ in range(8):
        x = [rnd.randrange(P) for _ in range(12)]
        assert naive(list(x)) == fast(list(x)), "fast partial rounds disagree with the round-by-round form"
    assert k[-1] == 0
    return {"m00": m00, "first": first, "init": [x for row in init for x in row], "k": k,
            "w": [x for row in ws for x in row], "v": [x for row in vs for x in row]}


def fmt_list(name, vals, per_line=4, hexw=16):
    lines = []
    for i in range(0, len(vals), per_line):
        chunk = vals[i:i + per_line]
        if hexw:
            suffix = "u" if hexw == 8 else "ULL"
            lines.append("    " + ", ".join("0x%0*x%s" % (hexw, v, suffix) for v in chunk))
        else:
            lines.append("    " + ", ".join("%d" % v for v in chunk))
    return "#define %s \\\n" % name + ", \\\n".join(lines) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ZEKNOX_REFERENCE_DIR", os.path.join(REPO_ROOT, "..", "reference")),
                    help="the reference tree (default: $ZEKNOX_REFERENCE_DIR, else ../reference beside this repository)")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "zk_constants.h"))
    args = ap.parse_args()

    omega, omega_inv, size_inv = derive_roots()
    rndc, rotc, piln = derive_keccak()
    ref = read_reference(args.ref)

    # derived tables must agree with the reference's own copies
    assert ref["omega"] == omega, "OMEGA mismatch"
    assert ref["omega_inv"] == omega_inv, "OMEGA_INV mismatch"
    assert ref["size_inv"] == size_inv, "DOMAIN_SIZE_INV mismatch"
    assert ref["k_rndc"] == rndc and ref["k_rotc"] == rotc and ref["k_piln"] == piln, "keccak tables mismatch"

    assert len(ref["poseidon_rc"]) == 360 and all(v < P for v in ref["poseidon_rc"])
    assert ref["poseidon_circ"] == [17, 15, 41, 16, 2, 28, 13, 13, 39, 18, 34, 20]
    assert ref["poseidon_diag"] == [8] + [0] * 11
    assert len(ref["p2_diag"]) == 12 and len(ref["p2_rc"]) == 360
    mono_rc = ref["mono_rc"]
    assert len(mono_rc) == 7 * 12, len(mono_rc)
    mat = ref["mono_mat"]
    assert len(mat) == 144
    row0 = mat[:12]
    for r in range(12):
        for c in range(12):
            assert mat[12 * r + c] == row0[(c - r) % 12], "monolith matrix is not circulant"

    # BN254 Montgomery parameters: derived, checked against the reference's literals
    bn_limbs32, bn_r2, bn_np32 = derive_bn254()
    r64 = _limbs64(BN_R)
    assert ref["bn_m0"] == [r64[0]] and ref["bn_modulus"] == [r64[3], r64[1], r64[2]], "BN254 modulus mismatch"
    assert ref["bn_r2"] == _limbs64(bn_r2), "BN254 R^2 mismatch"
    assert ref["bn_np64"] == [(-pow(BN_R, -1, 1 << 64)) % (1 << 64)], "BN254 -r^-1 mismatch"
    assert ref["bn_rounds_p"][3] == 60, "Poseidon-BN128 t = 5 partial rounds"
    for name, count in (("bn_c", 100), ("bn_s", 540), ("bn_m", 25), ("bn_p", 25)):
        v = ref[name]
        assert len(v) == 4 * count, (name, len(v))
        for i in range(0, len(v), 4):
            assert v[i] | v[i + 1] << 64 | v[i + 2] << 128 | v[i + 3] << 192 < BN_R, name

    hdr = []
    hdr.append("/* Generated by gen_constants.py -- do not edit.\n"
               " * Goldilocks p = 2^64 - 2^32 + 1 parameters for the commit path.\n"
               " * Roots and Keccak tables are derived; hash round constants are Plonky2's\n"
               " * published parameters (see gen_constants.py for provenance). */\n")
    hdr.append("#ifndef ZK_CONSTANTS_H\n#define ZK_CONSTANTS_H\n\n")
    hdr.append("#define ZK_P 0xffffffff00000001ULL\n#define ZK_GENERATOR 7ULL\n\n")
    hdr.append("/* omega[k]: primitive 2^k-th root of unity, omega[k-1] = omega[k]^2 */\n")
    hdr.append(fmt_list("ZK_OMEGA_LIST", omega))
    hdr.append(fmt_list("ZK_OMEGA_INV_LIST", omega_inv))
    hdr.append("/* 2^-k mod p */\n")
    hdr.append(fmt_list("ZK_DOMAIN_SIZE_INV_LIST", size_inv))
    hdr.append("\n/* Poseidon (width 12, 8 full + 22 partial rounds): round constant of lane i in\n"
               " * round r is element 12*r + i. MDS = circulant(row) + diag(8,0,...). */\n")
    hdr.append(fmt_list("ZK_POSEIDON_RC_LIST", ref["poseidon_rc"]))
    hdr.append(fmt_list("ZK_POSEIDON_CIRC_LIST", ref["poseidon_circ"], 12, 0))
    hdr.append("#define ZK_POSEIDON_DIAG0 %d\n" % ref["poseidon_diag"][0])
    fast = derive_poseidon_fast(ref["poseidon_rc"], ref["poseidon_circ"], ref["poseidon_diag"])
    # the derived sparse form agrees with the reference's own tables
    # (native/poseidon/poseidon.hpp:38-801; its initial matrix is stored transposed)
    assert ref["fast_first"] == fast["first"] and ref["fast_k"] == fast["k"], "fast partial constants mismatch"
    assert ref["fast_v"] == fast["v"] and ref["fast_w"] == fast["w"], "fast partial v / w mismatch"
    assert [ref["fast_init"][11 * j + i] for i in range(11) for j in range(11)] == fast["init"], "initial matrix mismatch"
    hdr.append("/* Partial rounds in sparse form (derived by gen_constants.py, checked against\n"
               " * the round-by-round form): x += FIRST; x[1..11] = INIT x[1..11]; per round r:\n"
               " * x0 = S(x0) + K[r]; x0' = M00 x0 + sum W[r][i] x[i+1]; x[i+1] += V[r][i] x0. */\n")
    hdr.append("#define ZK_POSEIDON_FAST_M00 %d\n" % fast["m00"])
    hdr.append(fmt_list("ZK_POSEIDON_FAST_FIRST_LIST", fast["first"]))
    hdr.append(fmt_list("ZK_POSEIDON_FAST_INIT_LIST", fast["init"]))
    hdr.append(fmt_list("ZK_POSEIDON_FAST_K_LIST", fast["k"]))
    hdr.append(fmt_list("ZK_POSEIDON_FAST_W_LIST", fast["w"]))
    hdr.append(fmt_list("ZK_POSEIDON_FAST_V_LIST", fast["v"]))
    hdr.append("\n/* Poseidon2 (width 12, 4+4 external rounds, 22 internal rounds). */\n")
    hdr.append(fmt_list("ZK_POSEIDON2_RC_LIST", ref["p2_rc"]))
    hdr.append(fmt_list("ZK_POSEIDON2_DIAG_LIST", ref["p2_diag"]))
    hdr.append("\n/* Monolith-64 (width 12, 6 rounds): 7 rows of 12 round constants; the\n"
               " * concrete layer is circulant with first row ZK_MONOLITH_CIRC_LIST\n"
               " * (entry [r][c] = row[(c - r) mod 12]). */\n")
    hdr.append(fmt_list("ZK_MONOLITH_RC_LIST", mono_rc))
    hdr.append(fmt_list("ZK_MONOLITH_CIRC_LIST", row0, 12, 0))
    hdr.append("\n/* Poseidon-BN128 over F_r (BN254 scalar field), t = 5, 8 full + 60 partial rounds.\n"
               " * Elements: 8 little-endian 32-bit limbs in Montgomery form (R = 2^256).\n"
               " * C: 100 round constants; S: 60 x 9 sparse partial-round entries; M, P: 5 x 5\n"
               " * matrices stored [j][i] (new_i = sum_j m[j][i] * s_j). */\n")
    hdr.append(fmt_list("ZK_BN254_R_LIST", bn_limbs32, 8, 8))
    hdr.append(fmt_list("ZK_BN254_R2_LIST", [(bn_r2 >> (32 * i)) & 0xFFFFFFFF for i in range(8)], 8, 8))
    hdr.append("#define ZK_BN254_NP 0x%08xu\n" % bn_np32)

    def to32(v64):
        return [(x >> sh) & 0xFFFFFFFF for x in v64 for sh in (0, 32)]

    hdr.append(fmt_list("ZK_BN128_C_LIST", to32(ref["bn_c"]), 8, 8))
    hdr.append(fmt_list("ZK_BN128_S_LIST", to32(ref["bn_s"]), 8, 8))
    hdr.append(fmt_list("ZK_BN128_M_LIST", to32(ref["bn_m"]), 8, 8))
    hdr.append(fmt_list("ZK_BN128_P_LIST", to32(ref["bn_p"]), 8, 8))
    hdr.append("\n/* Keccak-f[1600]: iota constants, rho offsets along the pi walk, pi lanes */\n")
    hdr.append(fmt_list("ZK_KECCAK_RNDC_LIST", rndc))
    hdr.append(fmt_list("ZK_KECCAK_ROTC_LIST", rotc, 12, 0))
    hdr.append(fmt_list("ZK_KECCAK_PILN_LIST", piln, 12, 0))
    hdr.append("\n#endif /* ZK_CONSTANTS_H */\n")
    with open(args.out, "w") as f:
        f.write("".join(hdr))
    print("wrote", args.out)


if __name__ == "__main__":
    sys.exit(main())
