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

    out = {}
    out["poseidon_rc"] = _numbers(_block(pos, r"ALL_ROUND_CONSTANTS\[[^\]]*\]\s*=\s*{"))
    out["poseidon_circ"] = _numbers(_block(pos, r"MDS_MATRIX_CIRC\[12\]\s*=\s*{"))
    out["poseidon_diag"] = _numbers(_block(pos, r"MDS_MATRIX_DIAG\[12\]\s*=\s*{"))
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
    return out


def fmt_list(name, vals, per_line=4, hexw=16):
    lines = []
    for i in range(0, len(vals), per_line):
        chunk = vals[i:i + per_line]
        if hexw:
            lines.append("    " + ", ".join("0x%0*xULL" % (hexw, v) for v in chunk))
        else:
            lines.append("    " + ", ".join("%d" % v for v in chunk))
    return "#define %s \\\n" % name + ", \\\n".join(lines) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
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
    hdr.append("\n/* Poseidon2 (width 12, 4+4 external rounds, 22 internal rounds). */\n")
    hdr.append(fmt_list("ZK_POSEIDON2_RC_LIST", ref["p2_rc"]))
    hdr.append(fmt_list("ZK_POSEIDON2_DIAG_LIST", ref["p2_diag"]))
    hdr.append("\n/* Monolith-64 (width 12, 6 rounds): 7 rows of 12 round constants; the\n"
               " * concrete layer is circulant with first row ZK_MONOLITH_CIRC_LIST\n"
               " * (entry [r][c] = row[(c - r) mod 12]). */\n")
    hdr.append(fmt_list("ZK_MONOLITH_RC_LIST", mono_rc))
    hdr.append(fmt_list("ZK_MONOLITH_CIRC_LIST", row0, 12, 0))
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
