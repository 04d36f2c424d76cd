// hash.cuh -- width-12 Goldilocks permutations and the Plonky2 sponge.
//
// Replaces zeknox's native/poseidon (Plonky2 Poseidon and Poseidon-BN128),
// native/poseidon2, native/monolith and native/keccak hashers.  State is 12
// uint64_t in registers; the work inside a round is unrolled (lane indices are
// constants), the rounds themselves are rolled loops that read their round
// constants from the constant bank, so a permutation's code fits the
// instruction cache.  The same code runs on the host (for the exported CPU
// Merkle builder) and on the device.
#pragma once
#include <stdint.h>
#include <string.h>

#include "bn254.cuh"
#include "gl64.cuh"
#include "zk_constants.h"

namespace zk {

enum HashKind : int { HASH_POSEIDON = 0, HASH_KECCAK = 1, HASH_POSEIDON_BN128 = 2, HASH_POSEIDON2 = 3, HASH_MONOLITH = 4 };

#ifdef __CUDA_ARCH__
#define ZKC(name) d_##name
#else
#define ZKC(name) h_##name
#endif

#ifdef __CUDACC__
#define ZK_CONST_TABLE(type, name, n, list) \
    static __constant__ type d_##name[n] = {list}; \
    static const type h_##name[n] = {list};
#else
#define ZK_CONST_TABLE(type, name, n, list) static const type h_##name[n] = {list};
#endif

ZK_CONST_TABLE(uint64_t, POSEIDON_RC, 360, ZK_POSEIDON_RC_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON_FAST_FIRST, 12, ZK_POSEIDON_FAST_FIRST_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON_FAST_INIT, 121, ZK_POSEIDON_FAST_INIT_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON_FAST_K, 22, ZK_POSEIDON_FAST_K_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON_FAST_W, 242, ZK_POSEIDON_FAST_W_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON_FAST_V, 242, ZK_POSEIDON_FAST_V_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON2_RC, 360, ZK_POSEIDON2_RC_LIST)
ZK_CONST_TABLE(uint64_t, POSEIDON2_DIAG, 12, ZK_POSEIDON2_DIAG_LIST)
ZK_CONST_TABLE(uint64_t, MONOLITH_RC, 84, ZK_MONOLITH_RC_LIST)
ZK_CONST_TABLE(uint64_t, KECCAK_RNDC, 24, ZK_KECCAK_RNDC_LIST)
ZK_CONST_TABLE(uint32_t, BN128_C, 800, ZK_BN128_C_LIST)
ZK_CONST_TABLE(uint32_t, BN128_S, 4320, ZK_BN128_S_LIST)
ZK_CONST_TABLE(uint32_t, BN128_M, 200, ZK_BN128_M_LIST)
ZK_CONST_TABLE(uint32_t, BN128_P, 200, ZK_BN128_P_LIST)

// Small circulant rows and the Keccak lane tables are compile-time constants
// (folded into the code once the loops are unrolled).
#ifdef __CUDACC__
#define ZK_CX __host__ __device__ constexpr
#else
#define ZK_CX constexpr
#endif
ZK_CX uint32_t poseidon_circ(int i)
{
    constexpr uint32_t c[12] = {ZK_POSEIDON_CIRC_LIST};
    return c[i];
}
ZK_CX uint32_t monolith_circ(int i)
{
    constexpr uint32_t c[12] = {ZK_MONOLITH_CIRC_LIST};
    return c[i];
}
ZK_CX int keccak_rot(int t)
{
    constexpr int r[24] = {ZK_KECCAK_ROTC_LIST};
    return r[t];
}
ZK_CX int keccak_pi(int t)
{
    constexpr int p[24] = {ZK_KECCAK_PILN_LIST};
    return p[t];
}

// ------------------------------------------------------------- small dot product
//
// sum_i x_i * c_i with x_i < 2^64 and small c_i, accumulated exactly as two
// 64-bit sums over the 32-bit halves of x (each < 2^32 * 12 * 64 < 2^42), then
// recombined into a < 2^80 value and reduced once.
struct Acc96 {
    uint64_t lo, hi;  // sum of low halves * c, sum of high halves * c
    ZK_HD void zero() { lo = hi = 0; }
    ZK_HD void mac(uint64_t x, uint32_t c)
    {
        lo += (x & 0xFFFFFFFFULL) * c;
        hi += (x >> 32) * c;
    }
    ZK_HD void add(uint64_t x) { lo += x & 0xFFFFFFFFULL; hi += x >> 32; }
    ZK_HD uint64_t reduce() const
    {
        uint64_t l = lo + (hi << 32);
        uint64_t h = (hi >> 32) + (l < lo);
        return gl_reduce96_nc(l, h);
    }
};

// Sum of 64-bit values with the carries counted: lo + 2^64 * c.
struct Sum64 {
    uint64_t lo;
    uint32_t c;
    ZK_HD void set(uint64_t x) { lo = x; c = 0; }
    ZK_HD void add(uint64_t x)
    {
#ifdef __CUDA_ARCH__
        uint32_t l0 = (uint32_t)lo, l1 = (uint32_t)(lo >> 32);
        asm("{\n\t"
            "add.cc.u32   %0, %0, %3;\n\t"
            "addc.cc.u32  %1, %1, %4;\n\t"
            "addc.u32     %2, %2, 0;\n\t"
            "}"
            : "+r"(l0), "+r"(l1), "+r"(c)
            : "r"((uint32_t)x), "r"((uint32_t)(x >> 32)));
        lo = ((uint64_t)l1 << 32) | l0;
#else
        lo += x;
        c += lo < x;
#endif
    }
    // lo + c * EPS, one wrap correction (c * EPS < 2^36)
    ZK_HD uint64_t reduce() const { return gl_add_nc(lo, ((uint64_t)c << 32) - c); }
};

// ----------------------------------------------------------------- Poseidon
//
// Plonky2 Poseidon in the round-by-round ("naive") form of
// native/poseidon/poseidon.cu:771-780 / poseidon.cpp:94-105: 4 full rounds,
// 22 partial rounds (S-box on lane 0 only), 4 full rounds; each round adds the
// 12 round constants of that round, applies the S-box layer, then the MDS
// matrix circ(17,15,41,16,2,28,13,13,39,18,34,20) + diag(8,0,...).
ZK_HD void poseidon_mds(uint64_t s[12])
{
    uint64_t t[12];
#pragma unroll
    for (int r = 0; r < 12; r++) {
        Acc96 a;
        a.zero();
#pragma unroll
        for (int i = 0; i < 12; i++) a.mac(s[(i + r) % 12], poseidon_circ(i));
        if (r == 0) a.mac(s[0], ZK_POSEIDON_DIAG0);
        t[r] = a.reduce();
    }
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = t[i];
}

// The 22 partial rounds in sparse-matrix form (Poseidon paper, eprint
// 2019/458 appendix B; the same rewriting as native/poseidon/poseidon.cpp's
// partial_rounds with its FAST_PARTIAL_* tables, whose values
// gen_constants.py derives from the MDS matrix and round constants and checks
// against the round-by-round form): one dense 11 x 11 layer, then per round
// the S-box on lane 0 and a matrix with one dense row and one dense column --
// 22 full multiplies per round instead of a 144-term MDS product.
ZK_HD void poseidon_partial_rounds(uint64_t s[12])
{
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = gl_add_nc(s[i], ZKC(POSEIDON_FAST_FIRST)[i]);
    uint64_t t[11] = {};
    // One row per iteration (the unrolled 121-product layer missed the
    // instruction cache: rolled, Poseidon forests measured 1.05x); the results
    // shift through t so that every register index stays a compile-time constant.
#pragma unroll 1
    for (int i = 0; i < 11; i++) {
        WideAcc a;
        a.zero();
#pragma unroll
        for (int j = 0; j < 11; j++) a.mac(s[1 + j], ZKC(POSEIDON_FAST_INIT)[11 * i + j]);
#pragma unroll
        for (int k = 0; k < 10; k++) t[k] = t[k + 1];
        t[10] = a.reduce();
    }
#pragma unroll
    for (int i = 0; i < 11; i++) s[1 + i] = t[i];
#pragma unroll 1
    for (int r = 0; r < 22; r++) {
        const uint64_t x0 = gl_add_nc(gl_sbox7_nc(s[0]), ZKC(POSEIDON_FAST_K)[r]);
        WideAcc a;
        a.zero();
        a.mac(x0, ZK_POSEIDON_FAST_M00);
#pragma unroll
        for (int i = 0; i < 11; i++) a.mac(s[1 + i], ZKC(POSEIDON_FAST_W)[11 * r + i]);
        s[0] = a.reduce();
#pragma unroll
        for (int i = 0; i < 11; i++) s[1 + i] = gl_mul_add_nc(x0, ZKC(POSEIDON_FAST_V)[11 * r + i], s[1 + i]);
    }
}

// Lanes hold any 64-bit representative between rounds (round constants are
// < p, so one wrap correction suffices when adding them); the caller
// canonicalises the digest.  One rolled loop over the 8 full rounds, the
// partial rounds after the fourth, so the full-round code exists once.
ZK_HD void poseidon_permute(uint64_t s[12])
{
#pragma unroll 1
    for (int f = 0; f < 8; f++) {
        const int r = f < 4 ? f : f + 22;
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = gl_sbox7_nc(gl_add_nc(s[i], ZKC(POSEIDON_RC)[12 * r + i]));
        poseidon_mds(s);
        if (f == 3) poseidon_partial_rounds(s);
    }
}

// ----------------------------------------------------------------- Poseidon2
//
// native/poseidon2/poseidon2.cu:65-209.  External layer: the 4x4 block
// M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] on each of the three lane
// groups, then every lane adds the sum of its column across the groups -- so
// lane 4g+k ends as  sum_j (1 + [g'==g]) * (M4 x_g')_k.  Internal layer:
// s_i <- s_i * diag_i + sum(s).
//
// The external layer runs on 22-bit pieces of each lane with the M4 addition chain
// of the Poseidon2 paper (eprint 2023/323, appendix B): t0 = x0+x1, t1 = x2+x3,
// t2 = 2x1+t1, t3 = 2x3+t0, t4 = 4t1+t3, t5 = 4t0+t2, M4 x = (t3+t5, t5, t2+t4,
// t4).  Every coefficient of a lane (own block doubled plus the other two)
// sums to 64, so a piece stays below 64 x 2^22 = 2^28.
ZK_HD void p2_m4_pieces(uint32_t *x)
{
    const uint32_t t0 = x[0] + x[1], t1 = x[2] + x[3];
    const uint32_t t2 = 2 * x[1] + t1, t3 = 2 * x[3] + t0;
    const uint32_t t4 = 4 * t1 + t3, t5 = 4 * t0 + t2;
    x[0] = t3 + t5;
    x[1] = t5;
    x[2] = t2 + t4;
    x[3] = t4;
}

// p0 + 2^22 p1 + 2^44 p2 (pieces < 2^28) reduced to a 64-bit representative:
// the sum is lo + 2^64 hi with hi < 2^9, and 2^64 = EPS (mod p).
ZK_HD uint64_t p2_combine_pieces(uint32_t p0, uint32_t p1, uint32_t p2)
{
#ifdef __CUDA_ARCH__
    uint32_t t0, t1, hi, e0, e1;
    asm("{\n\t"
        ".reg .u32 a, b, c, d;\n\t"
        "shl.b32         a, %6, 22;\n\t"
        "shr.b32         b, %6, 10;\n\t"
        "shl.b32         c, %7, 12;\n\t"
        "shr.b32         d, %7, 20;\n\t"
        "add.cc.u32      %0, %5, a;\n\t"     // lo = p0 + 2^22 p1 + 2^44 p2
        "addc.cc.u32     %1, b, c;\n\t"
        "addc.u32        %2, d, 0;\n\t"      // hi
        "sub.cc.u32      %3, 0, %2;\n\t"     // e = hi * EPS = 2^32 hi - hi
        "subc.u32        %4, %2, 0;\n\t"
        "add.cc.u32      %0, %0, %3;\n\t"    // lo + e, one EPS on carry
        "addc.cc.u32     %1, %1, %4;\n\t"
        "addc.u32        %2, 0, 0;\n\t"
        "neg.s32         %2, %2;\n\t"
        "add.cc.u32      %0, %0, %2;\n\t"
        "addc.u32        %1, %1, 0;\n\t"
        "}"
        : "=&r"(t0), "=&r"(t1), "=&r"(hi), "=&r"(e0), "=&r"(e1)
        : "r"(p0), "r"(p1), "r"(p2));
    return ((uint64_t)t1 << 32) | t0;
#else
    const uint64_t l1 = (uint64_t)p0 + ((uint64_t)p1 << 22);
    const uint64_t l2 = (uint64_t)p2 << 44;
    const uint64_t lo = l1 + l2;
    const uint64_t hi = (p2 >> 20) + (lo < l2);
    return gl_reduce96_nc(lo, hi);
#endif
}

ZK_HD void p2_external(uint64_t s[12])
{
    uint32_t p[3][12];
#pragma unroll
    for (int j = 0; j < 12; j++) {
        p[0][j] = (uint32_t)s[j] & 0x3FFFFFu;
        p[1][j] = (uint32_t)(s[j] >> 22) & 0x3FFFFFu;
        p[2][j] = (uint32_t)(s[j] >> 44);
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
#pragma unroll
        for (int g = 0; g < 3; g++) p2_m4_pieces(&p[q][4 * g]);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t col = p[q][k] + p[q][4 + k] + p[q][8 + k];
#pragma unroll
            for (int g = 0; g < 3; g++) p[q][4 * g + k] += col;
        }
    }
#pragma unroll
    for (int j = 0; j < 12; j++) s[j] = p2_combine_pieces(p[0][j], p[1][j], p[2][j]);
}

// Lanes hold any 64-bit representative between layers; digests are
// canonicalised by the sponge.  One rolled loop over the 30 rounds keeps the
// hot code small enough for the instruction cache (measured faster on B200
// than separate loops for the three round groups, and than hashing several
// leaves per thread in lockstep).
ZK_HD void poseidon2_permute(uint64_t s[12])
{
    p2_external(s);
#pragma unroll 1
    for (int r = 0; r < 30; r++) {
        if (r < 4 || r >= 26) {
#pragma unroll
            for (int i = 0; i < 12; i++) s[i] = gl_sbox7_nc<true, true>(gl_add_nc(s[i], ZKC(POSEIDON2_RC)[12 * r + i]));
            p2_external(s);
        } else {
            s[0] = gl_sbox7_nc<true, true>(gl_add_nc(s[0], ZKC(POSEIDON2_RC)[12 * r]));
            Sum64 acc;
            acc.set(s[0]);
#pragma unroll
            for (int i = 1; i < 12; i++) acc.add(s[i]);
            const uint64_t sum = acc.reduce();
            // s_i * d_i + sum as one 128-bit value, reduced once
#pragma unroll
            for (int i = 0; i < 12; i++) s[i] = gl_mul_add_nc(s[i], ZKC(POSEIDON2_DIAG)[i], sum);
        }
    }
}

// ----------------------------------------------------------------- Monolith
//
// Monolith-64 (native/monolith/monolith.cu:114-236): Concrete with round
// constants row 0, then 6 x [Bars on lanes 0..3, Bricks, Concrete(row r)].
//   Bar (per byte b):  rotl1(b ^ (rotl1(~b) & rotl2(b) & rotl3(b)))
//   Bricks: s_i += s_{i-1}^2 for i = 11..1 (old values), with the 65th bit kept
//   Concrete: circulant product of the 65-bit lanes plus the round constant.
ZK_HD uint64_t mono_bar(uint64_t x)
{
    const uint64_t H1 = 0x8080808080808080ULL, L7 = 0x7F7F7F7F7F7F7F7FULL;
    const uint64_t H2 = 0xC0C0C0C0C0C0C0C0ULL, L6 = 0x3F3F3F3F3F3F3F3FULL;
    const uint64_t H3 = 0xE0E0E0E0E0E0E0E0ULL, L5 = 0x1F1F1F1F1F1F1F1FULL;
    uint64_t nx = ~x;
    uint64_t r1 = ((nx & H1) >> 7) | ((nx & L7) << 1);
    uint64_t r2 = ((x & H2) >> 6) | ((x & L6) << 2);
    uint64_t r3 = ((x & H3) >> 5) | ((x & L5) << 3);
    uint64_t t = x ^ (r1 & r2 & r3);
    return ((t & H1) >> 7) | ((t & L7) << 1);
}

ZK_HD void mono_concrete(uint64_t s[12], const uint32_t hi[12], int round)
{
    uint64_t t[12];
#pragma unroll
    for (int r = 0; r < 12; r++) {
        Acc96 a;
        a.zero();
        uint64_t top = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            a.mac(s[c], monolith_circ((c - r + 12) % 12));
            top += (uint64_t)hi[c] * monolith_circ((c - r + 12) % 12);
        }
        a.add(ZKC(MONOLITH_RC)[12 * round + r]);
        // value = lo + 2^32*hi + 2^64*top
        uint64_t l = a.lo + (a.hi << 32);
        uint64_t h = (a.hi >> 32) + (l < a.lo) + top;
        t[r] = gl_reduce96_nc(l, h);
    }
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = t[i];
}

ZK_HD void monolith_permute(uint64_t s[12])
{
    uint32_t hi[12];
#pragma unroll
    for (int i = 0; i < 12; i++) hi[i] = 0;
    mono_concrete(s, hi, 0);
#pragma unroll 1
    for (int r = 1; r <= 6; r++) {
        // Bars act on the bits of the canonical value
#pragma unroll
        for (int i = 0; i < 4; i++) s[i] = mono_bar(gl_canon(s[i]));
        uint64_t sq[11];
#pragma unroll
        for (int i = 0; i < 11; i++) sq[i] = gl_sqr_nc(s[i]);
        hi[0] = 0;
#pragma unroll
        for (int i = 1; i < 12; i++) {
            uint64_t v = s[i] + sq[i - 1];
            hi[i] = v < sq[i - 1];
            s[i] = v;
        }
        mono_concrete(s, hi, r);
    }
}

// ------------------------------------------------------------------- Keccak
//
// Keccak-f[1600] (Keccak reference; zeknox uses Saarinen's formulation,
// native/keccak/keccak.cu:42-79), 24 rounds over 25 lanes.
ZK_HD uint64_t rotl64(uint64_t x, int k) { return k == 0 ? x : (x << k) | (x >> (64 - k)); }

ZK_HD void keccak_f(uint64_t st[25])
{
#pragma unroll 1
    for (int round = 0; round < 24; round++) {
        uint64_t c[5];
#pragma unroll
        for (int x = 0; x < 5; x++) c[x] = st[x] ^ st[x + 5] ^ st[x + 10] ^ st[x + 15] ^ st[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) {
            uint64_t d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
#pragma unroll
            for (int y = 0; y < 25; y += 5) st[y + x] ^= d;
        }
        uint64_t cur = st[1];
#pragma unroll
        for (int t = 0; t < 24; t++) {
            int j = keccak_pi(t);
            uint64_t nxt = st[j];
            st[j] = rotl64(cur, keccak_rot(t));
            cur = nxt;
        }
#pragma unroll
        for (int y = 0; y < 25; y += 5) {
            uint64_t r0 = st[y], r1 = st[y + 1], r2 = st[y + 2], r3 = st[y + 3], r4 = st[y + 4];
            st[y] = r0 ^ (~r1 & r2);
            st[y + 1] = r1 ^ (~r2 & r3);
            st[y + 2] = r2 ^ (~r3 & r4);
            st[y + 3] = r3 ^ (~r4 & r0);
            st[y + 4] = r4 ^ (~r0 & r1);
        }
        st[0] ^= ZKC(KECCAK_RNDC)[round];
    }
}

// ----------------------------------------------------------- Poseidon-BN128
//
// native/poseidon/poseidon_bn128.cu:115-200: the 12 canonical Goldilocks lanes
// become four 192-bit F_r elements (element i = lane 3i * 2^128 + lane 3i+1 *
// 2^64 + lane 3i+2) in state slots 1..4 (slot 0 = 0); round constants before
// every full round but the last, x^5 S-boxes, the full-round matrix M (P
// before the partial rounds), 60 partial rounds in iden3's sparse form (S-box
// on slot 0, + constant, new slot 0 = row . state, slot k += slot0 * column);
// the low 192 bits of slots 0..3 go back to the lanes, each reduced once mod p.
// Constant element idx of a table (read straight from the constant bank on
// the device).
#define ZK_BN_CONST(tab, idx)                                                \
    ([&]() {                                                                 \
        Fr x_;                                                               \
        _Pragma("unroll") for (int k_ = 0; k_ < 8; k_++) x_.w[k_] = ZKC(tab)[8 * (idx) + k_]; \
        return x_;                                                           \
    }())

// The matrix layers' dot products of five terms as one reduction (1) or as
// five fr_mul and four fr_add (0).  Both give the same canonical values.  The
// first, with its product and reduction steps out of line (one copy of their
// code: inlined at the call sites they stalled the leaf kernel on instruction
// fetch), measured 1.20x on a 2^20 x 135 Poseidon-BN128 forest (450 ms against
// 540) and 1.64x on a 2^14 x 135 one (18.0 against 29.5), with 128-thread leaf
// CTAs; it is the default.  The device-resident request loop compiles the
// second: built with the first (inlined), its kernel's register frame grew
// and its transform stages ran 14% slower (2^20 x 256 LDE: 61.0 ms against
// 53.7), because all stages share that kernel's 64-register budget.  Units
// built with different settings hold different bodies of the functions
// below; they are force-inlined (no out-of-line host symbol), the steps they
// call are file-local, and device code is not linked across units.
#ifndef ZK_BN128_DOT_ONE_REDUCTION
#define ZK_BN128_DOT_ONE_REDUCTION 1
#endif

// sum_j c_j * s_j, c_j = constant element c0 + j * cstep of a table
#if ZK_BN128_DOT_ONE_REDUCTION
#define ZK_BN_DOT5(out, tab, c0, cstep, s0, s1, s2, s3, s4)                          \
    do {                                                                               \
        FrWide acc_;                                                                   \
        fr_wide_zero(acc_);                                                            \
        acc_ = fr_mac_wide_ol(acc_, ZK_BN_CONST(tab, (c0)), s0);                       \
        acc_ = fr_mac_wide_ol(acc_, ZK_BN_CONST(tab, (c0) + (cstep)), s1);             \
        acc_ = fr_mac_wide_ol(acc_, ZK_BN_CONST(tab, (c0) + 2 * (cstep)), s2);         \
        acc_ = fr_mac_wide_ol(acc_, ZK_BN_CONST(tab, (c0) + 3 * (cstep)), s3);         \
        acc_ = fr_mac_wide_ol(acc_, ZK_BN_CONST(tab, (c0) + 4 * (cstep)), s4);         \
        out = fr_reduce_wide_ol(acc_);                                                 \
    } while (0)
#else
#define ZK_BN_DOT5(out, tab, c0, cstep, s0, s1, s2, s3, s4)                          \
    do {                                                                               \
        out = fr_mul(ZK_BN_CONST(tab, (c0)), s0);                                      \
        out = fr_add(out, fr_mul(ZK_BN_CONST(tab, (c0) + (cstep)), s1));               \
        out = fr_add(out, fr_mul(ZK_BN_CONST(tab, (c0) + 2 * (cstep)), s2));           \
        out = fr_add(out, fr_mul(ZK_BN_CONST(tab, (c0) + 3 * (cstep)), s3));           \
        out = fr_add(out, fr_mul(ZK_BN_CONST(tab, (c0) + 4 * (cstep)), s4));           \
    } while (0)
#endif

// new_i = sum_j m[j][i] * s_j with m = P (pre = true) or M.  With one
// reduction per output the outputs are computed in a rolled loop (one copy of
// the dot product's code) and shifted into place.
ZK_HD void bn128_mix(Fr st[5], bool pre)
{
    Fr ns[5];
#if ZK_BN128_DOT_ONE_REDUCTION
#pragma unroll 1
    for (int i = 0; i < 5; i++) {
        Fr o;
        if (pre) ZK_BN_DOT5(o, BN128_P, i, 5, st[0], st[1], st[2], st[3], st[4]);
        else ZK_BN_DOT5(o, BN128_M, i, 5, st[0], st[1], st[2], st[3], st[4]);
#pragma unroll
        for (int q = 0; q < 4; q++) ns[q] = ns[q + 1];
        ns[4] = o;
    }
#else
#pragma unroll
    for (int i = 0; i < 5; i++) {
#pragma unroll
        for (int j = 0; j < 5; j++) {
            const Fr m = pre ? ZK_BN_CONST(BN128_P, 5 * j + i) : ZK_BN_CONST(BN128_M, 5 * j + i);
            const Fr t = fr_mul(m, st[j]);
            ns[i] = j == 0 ? t : fr_add(ns[i], t);
        }
    }
#endif
#pragma unroll
    for (int i = 0; i < 5; i++) st[i] = ns[i];
}

ZK_HD void poseidon_bn128_permute(uint64_t s[12])
{
    Fr st[5];
    st[0] = fr_zero();
#pragma unroll
    for (int i = 0; i < 4; i++) {
        Fr x;
        const uint64_t l[3] = {gl_canon(s[3 * i + 2]), gl_canon(s[3 * i + 1]), gl_canon(s[3 * i])};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            x.w[2 * k] = (uint32_t)l[k];
            x.w[2 * k + 1] = (uint32_t)(l[k] >> 32);
        }
        x.w[6] = x.w[7] = 0;
        st[1 + i] = fr_to_mont(x);
    }
#pragma unroll
    for (int i = 0; i < 5; i++) st[i] = fr_add(st[i], ZK_BN_CONST(BN128_C, i));
#pragma unroll 1
    for (int f = 0; f < 8; f++) {
#pragma unroll
        for (int i = 0; i < 5; i++) st[i] = fr_exp5(st[i]);
        if (f != 7) {
            const int c0 = f < 4 ? 5 * (f + 1) : 85 + 5 * (f - 4);
#pragma unroll
            for (int i = 0; i < 5; i++) st[i] = fr_add(st[i], ZK_BN_CONST(BN128_C, c0 + i));
        }
        bn128_mix(st, f == 3);
        if (f == 3) {
#pragma unroll 1
            for (int r = 0; r < 60; r++) {
                const Fr x0 = fr_add(fr_exp5(st[0]), ZK_BN_CONST(BN128_C, 25 + r));
                Fr n0;
                ZK_BN_DOT5(n0, BN128_S, 9 * r, 1, x0, st[1], st[2], st[3], st[4]);
#pragma unroll
                for (int k = 1; k < 5; k++) st[k] = fr_add(st[k], fr_mul(x0, ZK_BN_CONST(BN128_S, 9 * r + 4 + k)));
                st[0] = n0;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const Fr v = fr_from_mont(st[i]);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint64_t limb = ((uint64_t)v.w[2 * k + 1] << 32) | v.w[2 * k];
            s[3 * i + 2 - k] = gl_canon(limb);
        }
    }
}

// ------------------------------------------------------------------ sponges

template <int H>
ZK_HD void permute(uint64_t s[12])
{
    if (H == HASH_POSEIDON) poseidon_permute(s);
    else if (H == HASH_POSEIDON2) poseidon2_permute(s);
    else if (H == HASH_POSEIDON_BN128) poseidon_bn128_permute(s);
    else monolith_permute(s);
}

// Plonky2 overwrite-mode sponge over a strided element source (element i at
// src[i * stride]); rate 8, capacity 4, zero initial state.  Inputs of <= 4
// elements are the digest themselves, zero padded
// (native/poseidon/poseidon_permutation.cuh:84-120).
template <int H>
ZK_HD void sponge_hash_one(const uint64_t *src, uint64_t len, uint64_t out[4])
{
    if (len <= 4) {
#pragma unroll
        for (int i = 0; i < 4; i++) out[i] = (uint64_t)i < len ? src[i] : 0;
        return;
    }
    uint64_t s[12];
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = 0;
    for (uint64_t idx = 0; idx < len; idx += 8) {
        uint64_t k = len - idx;
        if (k >= 8) {
#pragma unroll
            for (int i = 0; i < 8; i++) s[i] = src[idx + i];
        } else {
            // last partial chunk overwrites only its k < 8 lanes
#pragma unroll
            for (int i = 0; i < 8; i++)
                if ((uint64_t)i < k) s[i] = src[idx + i];
        }
        permute<H>(s);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) out[i] = gl_canon(s[i]);
}

template <int H>
ZK_HD void sponge_hash_two(const uint64_t l[4], const uint64_t r[4], uint64_t out[4])
{
    uint64_t s[12];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        s[i] = l[i];
        s[4 + i] = r[i];
        s[8 + i] = 0;
    }
    permute<H>(s);
#pragma unroll
    for (int i = 0; i < 4; i++) out[i] = gl_canon(s[i]);
}

// Keccak-256 (rate 136 bytes, 0x01 ... 0x80 padding) of len 8-byte words, the
// 32-byte digest with limb 3 truncated to one byte (native/keccak/keccak.cu:116-124).
// Fewer than 4 words are copied through (the remaining limbs are not written).
ZK_HD void keccak_hash_one(const uint64_t *src, uint64_t len, uint64_t out[4])
{
    if (len < 4) {
#pragma unroll
        for (int i = 0; i < 3; i++)
            if ((uint64_t)i < len) out[i] = src[i];
        return;
    }
    uint64_t st[25];
#pragma unroll
    for (int i = 0; i < 25; i++) st[i] = 0;
    uint64_t idx = 0;
    for (; len - idx >= 17; idx += 17) {
#pragma unroll
        for (int i = 0; i < 17; i++) st[i] ^= src[idx + i];
        keccak_f(st);
    }
    uint64_t rem = len - idx;
    // tail words, then the pad byte 0x01 right after the message and 0x80 into
    // the last byte of the 136-byte block
#pragma unroll
    for (int i = 0; i < 17; i++) {
        if ((uint64_t)i < rem) st[i] ^= src[idx + i];
        if ((uint64_t)i == rem) st[i] ^= 0x01ULL;
    }
    st[16] ^= 0x8000000000000000ULL;
    keccak_f(st);
    out[0] = st[0];
    out[1] = st[1];
    out[2] = st[2];
    out[3] = st[3] & 0xFF;
}

// Keccak-256 of 25 bytes of l followed by 25 bytes of r (native/keccak/keccak.cu:126-135).
ZK_HD void keccak_hash_two(const uint64_t l[4], const uint64_t r[4], uint64_t out[4])
{
    uint64_t st[25];
#pragma unroll
    for (int i = 0; i < 25; i++) st[i] = 0;
    uint64_t r3 = r[3] & 0xFF;
    st[0] = l[0];
    st[1] = l[1];
    st[2] = l[2];
    st[3] = (l[3] & 0xFF) | (r[0] << 8);
    st[4] = (r[0] >> 56) | (r[1] << 8);
    st[5] = (r[1] >> 56) | (r[2] << 8);
    st[6] = (r[2] >> 56) | (r3 << 8) | (0x01ULL << 16);
    st[16] = 0x8000000000000000ULL;
    keccak_f(st);
    out[0] = st[0];
    out[1] = st[1];
    out[2] = st[2];
    out[3] = st[3] & 0xFF;
}

template <int H>
ZK_HD void hash_one(const uint64_t *src, uint64_t len, uint64_t out[4])
{
    if (H == HASH_KECCAK) keccak_hash_one(src, len, out);
    else sponge_hash_one<H>(src, len, out);
}

template <int H>
ZK_HD void hash_two(const uint64_t l[4], const uint64_t r[4], uint64_t out[4])
{
    if (H == HASH_KECCAK) keccak_hash_two(l, r, out);
    else sponge_hash_two<H>(l, r, out);
}

}  // namespace zk
