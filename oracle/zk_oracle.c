/*
 * zk_oracle.c -- CPU restatement of zeknox's Goldilocks commit path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in zeknox_b200/: the tests, the smoke check and the CPU baseline leg
 * of bench.py call it; the product never does.
 *
 * Everything is exact arithmetic mod p = 2^64 - 2^32 + 1 on unsigned __int128,
 * written from the field's definition and the reference's documented
 * semantics.  Each function names the reference lines it restates (paths are
 * relative to the zeknox repository root).  Values are kept canonical (< p).
 * The reference CPU field (native/ff/goldilocks.hpp:139-177) can return the
 * non-canonical p for x - x, and its reduce128 can leave a value in [p, 2^64)
 * with probability ~2^-32 per operation; both are equal mod p, and every output
 * of the path is compared canonically.
 *
 * Pinning: the hashes and the Merkle builder are checked against the
 * reference's own known-answer vectors (native/tests/tests.cu) and against the
 * reference CPU library compiled from its sources (oracle/Makefile -> _ref/);
 * the NTT family is the O(n^2) DFT definition plus an O(n log n) radix-2
 * restatement that must agree with it.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../zeknox_b200/csrc/zk_constants.h"

typedef uint64_t u64;
typedef uint32_t u32;
typedef unsigned __int128 u128;

#define P ZK_P

static const u64 OMEGA[33] = {ZK_OMEGA_LIST};
static const u64 OMEGA_INV[33] = {ZK_OMEGA_INV_LIST};
static const u64 SIZE_INV[33] = {ZK_DOMAIN_SIZE_INV_LIST};
static const u64 POSEIDON_RC[360] = {ZK_POSEIDON_RC_LIST};
static const u64 POSEIDON_CIRC[12] = {ZK_POSEIDON_CIRC_LIST};
static const u64 P2_RC[360] = {ZK_POSEIDON2_RC_LIST};
static const u64 P2_DIAG[12] = {ZK_POSEIDON2_DIAG_LIST};
static const u64 MONO_RC[7 * 12] = {ZK_MONOLITH_RC_LIST};
static const u64 MONO_CIRC[12] = {ZK_MONOLITH_CIRC_LIST};
static const u64 KECCAK_RNDC[24] = {ZK_KECCAK_RNDC_LIST};
static const int KECCAK_ROTC[24] = {ZK_KECCAK_ROTC_LIST};
static const int KECCAK_PILN[24] = {ZK_KECCAK_PILN_LIST};

/* ------------------------------------------------------------------ field */

static inline u64 f_red(u128 x) { return (u64)(x % P); }
static inline u64 f_add(u64 a, u64 b) { return f_red((u128)a + b); }
static inline u64 f_sub(u64 a, u64 b) { return f_red((u128)a + P - (b % P)); }
static inline u64 f_mul(u64 a, u64 b) { return f_red((u128)a * b); }
static u64 f_pow(u64 a, u64 e)
{
    u64 r = 1;
    a %= P;
    while (e) {
        if (e & 1) r = f_mul(r, a);
        a = f_mul(a, a);
        e >>= 1;
    }
    return r;
}

u64 zko_mul(u64 a, u64 b) { return f_mul(a, b); }
u64 zko_add(u64 a, u64 b) { return f_add(a, b); }
u64 zko_sub(u64 a, u64 b) { return f_sub(a, b); }
u64 zko_pow(u64 a, u64 e) { return f_pow(a, e); }
u64 zko_omega(u32 lg, int inverse) { return inverse ? OMEGA_INV[lg] : OMEGA[lg]; }

static inline u64 rev_bits(u64 x, u32 bits)
{
    u64 r = 0;
    for (u32 i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}

/* ------------------------------------------------------------------- NTT */

/* Definition: X_k = sum_j x_j w^{jk}, w = OMEGA[lg] (or OMEGA_INV[lg]).
 * O(n^2); used to pin the fast form at small sizes. */
void zko_dft_naive(const u64 *in, u64 *out, u32 lg, int inverse)
{
    u64 n = 1ULL << lg;
    u64 w = inverse ? OMEGA_INV[lg] : OMEGA[lg];
    for (u64 k = 0; k < n; k++) {
        u64 wk = f_pow(w, k), acc = 0, t = 1;
        for (u64 j = 0; j < n; j++) {
            acc = f_add(acc, f_mul(in[j], t));
            t = f_mul(t, wk);
        }
        out[k] = acc;
    }
}

/* In-place iterative radix-2 DIT on natural-order input (bit-reverse first),
 * natural-order output, no scaling. */
static void ntt_radix2(u64 *a, u32 lg, int inverse)
{
    u64 n = 1ULL << lg;
    for (u64 i = 0; i < n; i++) {
        u64 r = rev_bits(i, lg);
        if (i < r) {
            u64 t = a[i];
            a[i] = a[r];
            a[r] = t;
        }
    }
    u64 *tw = (u64 *)malloc(sizeof(u64) * (n / 2 + 1));
    for (u32 s = 1; s <= lg; s++) {
        u64 m = 1ULL << s, h = m >> 1;
        u64 wm = inverse ? OMEGA_INV[s] : OMEGA[s];
        tw[0] = 1;
        for (u64 j = 1; j < h; j++) tw[j] = f_mul(tw[j - 1], wm);
        for (u64 k = 0; k < n; k += m)
            for (u64 j = 0; j < h; j++) {
                u64 u = a[k + j], v = f_mul(a[k + j + h], tw[j]);
                a[k + j] = f_add(u, v);
                a[k + j + h] = f_sub(u, v);
            }
    }
    free(tw);
}

/* compute_batched_ntt semantics (native/ntt/ntt.cu:253-309 with
 * ntt_inplace_batch_template :106-158):
 *   forward: x_j *= g^j (with_coset), X = NTT(x), natural order.
 *   inverse: y = iNTT(x) unscaled, then y_i *= g^i (with_coset; forward powers,
 *            applied before normalising, :137-143), then y_i *= n^-1. */
void zko_batched_ntt(u64 *inout, u32 lg, u32 batches, int inverse, int with_coset, u64 coset_gen)
{
    u64 n = 1ULL << lg;
#pragma omp parallel for schedule(dynamic)
    for (long b = 0; b < (long)batches; b++) {
        u64 *a = inout + (u64)b * n;
        if (!inverse) {
            if (with_coset) {
                u64 g = 1;
                for (u64 i = 0; i < n; i++) {
                    a[i] = f_mul(a[i], g);
                    g = f_mul(g, coset_gen);
                }
            }
            ntt_radix2(a, lg, 0);
        } else {
            ntt_radix2(a, lg, 1);
            u64 ninv = SIZE_INV[lg], g = 1;
            for (u64 i = 0; i < n; i++) {
                u64 v = a[i];
                if (with_coset) {
                    v = f_mul(v, g);
                    g = f_mul(g, coset_gen);
                }
                a[i] = f_mul(v, ninv);
            }
        }
    }
}

/* compute_batched_lde semantics (native/ntt/ntt.cu:477-564): zero-extend each
 * column from n = 2^lg to N = 2^(lg+rate) (degree_extension_kernel,
 * native/ntt/kernels.cu:40-60), then the size-N transform of
 * zko_batched_ntt.  Column-major in (batches x n) and out (batches x N). */
void zko_batched_lde(u64 *out, const u64 *in, u32 lg, u32 rate, u32 batches, int inverse, int with_coset,
                     u64 coset_gen)
{
    u64 n = 1ULL << lg, N = n << rate;
    for (u64 b = 0; b < batches; b++) {
        memcpy(out + b * N, in + b * n, n * 8);
        memset(out + b * N + n, 0, (N - n) * 8);
    }
    zko_batched_ntt(out, lg + rate, batches, inverse, with_coset, coset_gen);
}

/* compute_transpose_rev (native/ntt/kernels.cu:94-135):
 * out[rev_lg(i) * batches + b] = in[b * n + i]. */
void zko_transpose_rev(u64 *out, const u64 *in, u32 lg, u32 batches)
{
    u64 n = 1ULL << lg;
#pragma omp parallel for
    for (long i = 0; i < (long)n; i++) {
        u64 r = rev_bits((u64)i, lg);
        for (u64 b = 0; b < batches; b++) out[r * batches + b] = in[b * n + (u64)i];
    }
}

/* --------------------------------------------------------------- Poseidon */

static inline u64 sbox7(u64 x)
{
    u64 x2 = f_mul(x, x), x4 = f_mul(x2, x2), x3 = f_mul(x2, x);
    return f_mul(x3, x4);
}

/* Plonky2 Poseidon, naive round structure (native/poseidon/poseidon.cpp:13-110):
 * 4 full rounds, 22 partial rounds (S-box on lane 0), 4 full rounds; every round
 * adds ALL_ROUND_CONSTANTS[12*r + i] to all lanes before the S-box; MDS row r
 * is sum_i s[(i + r) % 12] * CIRC[i] + 8 * s[r] (diag only on lane 0 -> r=0). */
void zko_poseidon_permute(u64 s[12])
{
    for (u32 r = 0; r < 30; r++) {
        for (int i = 0; i < 12; i++) s[i] = f_add(s[i], POSEIDON_RC[12 * r + i]);
        if (r < 4 || r >= 26) {
            for (int i = 0; i < 12; i++) s[i] = sbox7(s[i]);
        } else {
            s[0] = sbox7(s[0]);
        }
        u64 t[12];
        for (int row = 0; row < 12; row++) {
            u128 acc = 0;
            for (int i = 0; i < 12; i++) acc += (u128)s[(i + row) % 12] * POSEIDON_CIRC[i];
            if (row == 0) acc += (u128)s[0] * ZK_POSEIDON_DIAG0;
            t[row] = f_red(acc);
        }
        memcpy(s, t, sizeof t);
    }
}

/* ---------------------------------------------------------------- Poseidon2 */

/* native/poseidon2/poseidon2.cu:65-82 (4x4 external block) */
static void p2_m4(u64 *x)
{
    u64 t0 = f_add(x[0], x[1]);
    u64 t1 = f_add(x[2], x[3]);
    u64 t2 = f_add(f_add(x[1], x[1]), t1);
    u64 t3 = f_add(f_add(x[3], x[3]), t0);
    u64 t4 = f_add(f_mul(t1, 4), t3);
    u64 t5 = f_add(f_mul(t0, 4), t2);
    u64 t6 = f_add(t3, t5);
    u64 t7 = f_add(t2, t4);
    x[0] = t6;
    x[1] = t5;
    x[2] = t7;
    x[3] = t4;
}

/* native/poseidon2/poseidon2.cu:121-145 */
static void p2_external(u64 *s)
{
    for (int i = 0; i < 12; i += 4) p2_m4(s + i);
    u64 sums[4];
    for (int k = 0; k < 4; k++) sums[k] = f_add(f_add(s[k], s[4 + k]), s[8 + k]);
    for (int i = 0; i < 12; i++) s[i] = f_add(s[i], sums[i % 4]);
}

/* native/poseidon2/poseidon2.cu:167-209 */
void zko_poseidon2_permute(u64 s[12])
{
    p2_external(s);
    for (int r = 0; r < 4; r++) {
        for (int i = 0; i < 12; i++) s[i] = sbox7(f_add(s[i], P2_RC[12 * r + i]));
        p2_external(s);
    }
    for (int r = 4; r < 26; r++) {
        s[0] = sbox7(f_add(s[0], P2_RC[12 * r]));
        u64 sum = 0;
        for (int i = 0; i < 12; i++) sum = f_add(sum, s[i]);
        for (int i = 0; i < 12; i++) s[i] = f_add(f_mul(s[i], P2_DIAG[i]), sum);
    }
    for (int r = 26; r < 30; r++) {
        for (int i = 0; i < 12; i++) s[i] = sbox7(f_add(s[i], P2_RC[12 * r + i]));
        p2_external(s);
    }
}

/* ---------------------------------------------------------------- Monolith */

/* Bar: per byte y = rotl1(x ^ (rotl1(~x) & rotl2(x) & rotl3(x)))
 * (native/monolith/monolith.cu:114-123), applied to the raw bits of lanes 0..3. */
static u64 mono_bar(u64 x)
{
    u64 y = 0;
    for (int i = 0; i < 8; i++) {
        uint8_t b = (uint8_t)(x >> (8 * i));
        uint8_t nb = (uint8_t)~b;
        uint8_t r1 = (uint8_t)((nb << 1) | (nb >> 7));
        uint8_t r2 = (uint8_t)((b << 2) | (b >> 6));
        uint8_t r3 = (uint8_t)((b << 3) | (b >> 5));
        uint8_t t = (uint8_t)(b ^ (r1 & r2 & r3));
        uint8_t o = (uint8_t)((t << 1) | (t >> 7));
        y |= (u64)o << (8 * i);
    }
    return y;
}

/* Monolith-64 (native/monolith/monolith.cu:147-236).  Lanes are handled as the
 * 65-bit integers lo + 2^64 * hi produced by the Bricks layer; Concrete reduces
 * the circulant product plus round constant mod p. */
void zko_monolith_permute(u64 s[12])
{
    u64 hi[12] = {0};
    for (int r = 0; r < 7; r++) {
        if (r > 0) {
            for (int i = 0; i < 4; i++) s[i] = mono_bar(s[i]);
            u64 sq[12];
            for (int i = 0; i < 11; i++) sq[i] = f_mul(s[i], s[i]);
            for (int i = 11; i > 0; i--) {
                u64 v = s[i] + sq[i - 1];
                hi[i] = v < sq[i - 1];
                s[i] = v;
            }
        }
        u64 t[12];
        for (int row = 0; row < 12; row++) {
            u128 acc = MONO_RC[12 * r + row];
            for (int c = 0; c < 12; c++) {
                u64 m = MONO_CIRC[(c - row + 12) % 12];
                acc += ((u128)s[c] + ((u128)hi[c] << 64)) * m;
            }
            t[row] = f_red(acc);
        }
        memcpy(s, t, sizeof t);
        memset(hi, 0, sizeof hi);
    }
}

/* ------------------------------------------------------------------ Keccak */

static inline u64 rotl64(u64 x, int k) { return k ? (x << k) | (x >> (64 - k)) : x; }

/* Keccak-f[1600], 24 rounds (Keccak specification; the reference follows
 * Saarinen's formulation, native/keccak/keccak.cu:42-79). */
static void keccak_f(u64 st[25])
{
    for (int round = 0; round < 24; round++) {
        u64 c[5], d;
        for (int x = 0; x < 5; x++) c[x] = st[x] ^ st[x + 5] ^ st[x + 10] ^ st[x + 15] ^ st[x + 20];
        for (int x = 0; x < 5; x++) {
            d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
            for (int y = 0; y < 25; y += 5) st[y + x] ^= d;
        }
        u64 cur = st[1];
        for (int t = 0; t < 24; t++) {
            int j = KECCAK_PILN[t];
            u64 nxt = st[j];
            st[j] = rotl64(cur, KECCAK_ROTC[t]);
            cur = nxt;
        }
        for (int y = 0; y < 25; y += 5) {
            u64 row[5];
            for (int x = 0; x < 5; x++) row[x] = st[y + x];
            for (int x = 0; x < 5; x++) st[y + x] ^= (~row[(x + 1) % 5]) & row[(x + 2) % 5];
        }
        st[0] ^= KECCAK_RNDC[round];
    }
}

/* Keccak with 32-byte output, rate 136 bytes and the original 0x01..0x80
 * padding (native/keccak/keccak.cu:83-112). */
static void keccak256(const uint8_t *in, u64 len, uint8_t out[32])
{
    u64 st[25] = {0};
    const u64 rate = 136;
    while (len >= rate) {
        for (int i = 0; i < 17; i++) {
            u64 w;
            memcpy(&w, in + 8 * i, 8);
            st[i] ^= w;
        }
        keccak_f(st);
        in += rate;
        len -= rate;
    }
    uint8_t block[136];
    memset(block, 0, sizeof block);
    memcpy(block, in, len);
    block[len] = 0x01;
    block[rate - 1] |= 0x80;
    for (int i = 0; i < 17; i++) {
        u64 w;
        memcpy(&w, block + 8 * i, 8);
        st[i] ^= w;
    }
    keccak_f(st);
    memcpy(out, st, 32);
}

/* --------------------------------------------------------- Poseidon-BN128 */

/* F_r, r the BN254 scalar field order: 4 x 64-bit little-endian limbs in
 * Montgomery form (R = 2^256), as native/poseidon/element_bn128.cu keeps them;
 * multiplication is the textbook CIOS Montgomery product on u128. */
typedef struct {
    u64 v[4];
} fr_t;

static const u32 BN_R32[8] = {ZK_BN254_R_LIST};
static const u32 BN_R2_32[8] = {ZK_BN254_R2_LIST};
static const u32 BN_C32[800] = {ZK_BN128_C_LIST};
static const u32 BN_S32[4320] = {ZK_BN128_S_LIST};
static const u32 BN_M32[200] = {ZK_BN128_M_LIST};
static const u32 BN_P32[200] = {ZK_BN128_P_LIST};

static fr_t fr_load(const u32 *t, int idx)
{
    fr_t x;
    for (int i = 0; i < 4; i++) x.v[i] = (u64)t[8 * idx + 2 * i] | ((u64)t[8 * idx + 2 * i + 1] << 32);
    return x;
}

static int fr_geq(const u64 *a, const u64 *b)
{
    for (int i = 3; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return 1;
}

static void fr_sub_in(u64 *a, const u64 *b)
{
    u64 borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        a[i] = (u64)d;
        borrow = (u64)(d >> 127);
    }
}

static fr_t bn_add(fr_t a, fr_t b)
{
    const fr_t r = fr_load(BN_R32, 0);
    fr_t s;
    u64 c = 0;
    for (int i = 0; i < 4; i++) {
        u128 t = (u128)a.v[i] + b.v[i] + c;
        s.v[i] = (u64)t;
        c = (u64)(t >> 64);
    }
    if (c || fr_geq(s.v, r.v)) fr_sub_in(s.v, r.v);
    return s;
}

static fr_t bn_mul(fr_t a, fr_t b)
{
    const fr_t r = fr_load(BN_R32, 0);
    /* -r^-1 mod 2^64 by Newton's iteration (x <- x (2 - r x)) */
    u64 inv = 1;
    for (int i = 0; i < 6; i++) inv *= 2 - r.v[0] * inv;
    const u64 np = (u64)0 - inv;
    u64 t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u64 c = 0;
        for (int j = 0; j < 4; j++) {
            u128 x = (u128)a.v[i] * b.v[j] + t[j] + c;
            t[j] = (u64)x;
            c = (u64)(x >> 64);
        }
        u128 x = (u128)t[4] + c;
        t[4] = (u64)x;
        t[5] = (u64)(x >> 64);
        const u64 m = t[0] * np;
        x = (u128)m * r.v[0] + t[0];
        c = (u64)(x >> 64);
        for (int j = 1; j < 4; j++) {
            x = (u128)m * r.v[j] + t[j] + c;
            t[j - 1] = (u64)x;
            c = (u64)(x >> 64);
        }
        x = (u128)t[4] + c;
        t[3] = (u64)x;
        t[4] = t[5] + (u64)(x >> 64);
    }
    fr_t z = {{t[0], t[1], t[2], t[3]}};
    if (t[4] || fr_geq(z.v, r.v)) fr_sub_in(z.v, r.v);
    return z;
}

static fr_t bn_exp5(fr_t x)
{
    fr_t x2 = bn_mul(x, x), x4 = bn_mul(x2, x2);
    return bn_mul(x4, x);
}

static void bn_mix(fr_t st[5], const u32 *m)
{
    fr_t ns[5];
    for (int i = 0; i < 5; i++) {
        ns[i] = bn_mul(fr_load(m, i), st[0]);
        for (int j = 1; j < 5; j++) ns[i] = bn_add(ns[i], bn_mul(fr_load(m, 5 * j + i), st[j]));
    }
    memcpy(st, ns, sizeof ns);
}

/* native/poseidon/poseidon_bn128.cu:115-212 (permute_fn + permute): lanes
 * 3i..3i+2 form element i+1 (big-endian lane order, top limb 0), t = 5,
 * 4 full rounds (constants, x^5, M; P for the fourth), 60 sparse partial
 * rounds, 4 full rounds (no constants in the last); slots 0..3 back to the
 * lanes (low 192 bits), each reduced once mod p. */
static void zko_poseidon_bn128_permute(u64 s[12])
{
    fr_t st[5];
    memset(st, 0, sizeof st);
    const fr_t r2 = fr_load(BN_R2_32, 0);
    for (int i = 0; i < 4; i++) {
        fr_t x = {{s[3 * i + 2] % P, s[3 * i + 1] % P, s[3 * i] % P, 0}};
        st[1 + i] = bn_mul(x, r2);
    }
    for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], fr_load(BN_C32, i));
    for (int f = 0; f < 3; f++) {
        for (int i = 0; i < 5; i++) st[i] = bn_exp5(st[i]);
        for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], fr_load(BN_C32, 5 * (f + 1) + i));
        bn_mix(st, BN_M32);
    }
    for (int i = 0; i < 5; i++) st[i] = bn_exp5(st[i]);
    for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], fr_load(BN_C32, 20 + i));
    bn_mix(st, BN_P32);
    for (int r = 0; r < 60; r++) {
        st[0] = bn_add(bn_exp5(st[0]), fr_load(BN_C32, 25 + r));
        fr_t n0 = bn_mul(fr_load(BN_S32, 9 * r), st[0]);
        for (int j = 1; j < 5; j++) n0 = bn_add(n0, bn_mul(fr_load(BN_S32, 9 * r + j), st[j]));
        for (int k = 1; k < 5; k++) st[k] = bn_add(st[k], bn_mul(st[0], fr_load(BN_S32, 9 * r + 4 + k)));
        st[0] = n0;
    }
    for (int f = 0; f < 3; f++) {
        for (int i = 0; i < 5; i++) st[i] = bn_exp5(st[i]);
        for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], fr_load(BN_C32, 85 + 5 * f + i));
        bn_mix(st, BN_M32);
    }
    for (int i = 0; i < 5; i++) st[i] = bn_exp5(st[i]);
    bn_mix(st, BN_M32);
    const fr_t one = {{1, 0, 0, 0}};
    for (int i = 0; i < 4; i++) {
        fr_t v = bn_mul(st[i], one);
        s[3 * i] = v.v[2] % P;
        s[3 * i + 1] = v.v[1] % P;
        s[3 * i + 2] = v.v[0] % P;
    }
}

/* ---------------------------------------------------------------- sponges */

enum { H_POSEIDON = 0, H_KECCAK = 1, H_POSEIDON_BN128 = 2, H_POSEIDON2 = 3, H_MONOLITH = 4 };

static void permute(int h, u64 s[12])
{
    if (h == H_POSEIDON) zko_poseidon_permute(s);
    else if (h == H_POSEIDON2) zko_poseidon2_permute(s);
    else if (h == H_POSEIDON_BN128) zko_poseidon_bn128_permute(s);
    else zko_monolith_permute(s);
}

/* hash_one: Plonky2 overwrite-mode sponge, rate 8, zero initial state
 * (native/poseidon/poseidon_permutation.hpp:84-122); inputs of <= 4 elements
 * are returned zero-padded without hashing.  Keccak
 * (native/keccak/keccak.cu:139-147): < 4 elements are copied (remaining
 * output limbs untouched), otherwise keccak256 of the bytes with limb 3
 * truncated to its low byte. */
int zko_hash_one(int h, const u64 *in, u64 n, u64 out[4])
{
    if (h == H_KECCAK) {
        if (n < 4) {
            memcpy(out, in, n * 8);
            return 0;
        }
        keccak256((const uint8_t *)in, n * 8, (uint8_t *)out);
        out[3] &= 0xFF;
        return 0;
    }
    if (h != H_POSEIDON && h != H_POSEIDON2 && h != H_MONOLITH && h != H_POSEIDON_BN128) return -1;
    if (n <= 4) {
        for (u64 i = 0; i < 4; i++) out[i] = i < n ? in[i] : 0;
        return 0;
    }
    u64 s[12] = {0};
    for (u64 idx = 0; idx < n; idx += 8) {
        u64 k = n - idx < 8 ? n - idx : 8;
        for (u64 i = 0; i < k; i++) s[i] = in[idx + i];
        permute(h, s);
    }
    for (int i = 0; i < 4; i++) out[i] = s[i] % P;
    return 0;
}

/* hash_two: state = left || right || 0^4, one permutation
 * (poseidon_permutation.hpp:125-139); Keccak: keccak256(25 bytes of left ||
 * 25 bytes of right) (keccak.cu:149-156). */
int zko_hash_two(int h, const u64 l[4], const u64 r[4], u64 out[4])
{
    if (h == H_KECCAK) {
        uint8_t buf[50];
        memcpy(buf, l, 25);
        memcpy(buf + 25, r, 25);
        keccak256(buf, 50, (uint8_t *)out);
        out[3] &= 0xFF;
        return 0;
    }
    if (h != H_POSEIDON && h != H_POSEIDON2 && h != H_MONOLITH && h != H_POSEIDON_BN128) return -1;
    u64 s[12] = {0};
    memcpy(s, l, 32);
    memcpy(s + 4, r, 32);
    permute(h, s);
    for (int i = 0; i < 4; i++) out[i] = s[i] % P;
    return 0;
}

/* Keccak-f[1600] alone, 25 lanes in place (the permutation of keccak256 above). */
void zko_keccak_f(u64 st[25]) { keccak_f(st); }

int zko_permute(int h, u64 s[12])
{
    if (h != H_POSEIDON && h != H_POSEIDON2 && h != H_MONOLITH && h != H_POSEIDON_BN128) return -1;
    permute(h, s);
    return 0;
}

/* ----------------------------------------------------------------- Merkle */

/* Linear Merkle forest (native/merkle/merkle.cpp:20-124, same layout as the GPU
 * builder native/merkle/merkle.cu:166-244).  2^cap_height subtrees of L leaves
 * each; subtree k owns digests [k*(2L-2), (k+1)*(2L-2)); inside it the level of
 * 2^r nodes starts at 2^r - 2, node i's children are 2(i+1) and 2(i+1)+1 of
 * the level below, leaf digests start at L - 2, and the subtree root H2(d[0],
 * d[1]) goes to cap[k].  Special cases: caps == leaves -> caps are the leaf
 * hashes and digests are untouched; L == 2 -> digests are the leaf hashes. */
int zko_merkle(u64 *digests, u64 *caps, const u64 *leaves, u64 n_digests, u64 n_caps, u64 n_leaves,
               u64 leaf_size, u64 cap_height, int h)
{
    if (n_caps == n_leaves) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n_leaves; i++) zko_hash_one(h, leaves + (u64)i * leaf_size, leaf_size, caps + 4 * (u64)i);
        return 0;
    }
    u64 sub_dig = n_digests >> cap_height, sub_leaves = n_leaves >> cap_height;
    if (sub_dig * n_caps != n_digests || sub_leaves * n_caps != n_leaves || n_caps != (1ULL << cap_height))
        return -1;
    for (u64 k = 0; k < n_caps; k++) {
        const u64 *lv = leaves + k * sub_leaves * leaf_size;
        u64 *dg = digests + k * sub_dig * 4;
        u64 *cp = caps + k * 4;
        if (sub_leaves == 1) {
            zko_hash_one(h, lv, leaf_size, dg);
            memcpy(cp, dg, 32);
            continue;
        }
        if (sub_leaves == 2) {
            zko_hash_one(h, lv, leaf_size, dg);
            zko_hash_one(h, lv + leaf_size, leaf_size, dg + 4);
            zko_hash_two(h, dg, dg + 4, cp);
            continue;
        }
        u64 *leaf_dig = dg + (sub_dig - sub_leaves) * 4;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)sub_leaves; i++) zko_hash_one(h, lv + (u64)i * leaf_size, leaf_size, leaf_dig + 4 * (u64)i);
        u64 level = sub_leaves / 2;
        while (level >= 2) {
            u64 start = level - 2, child = 2 * level - 2;
#pragma omp parallel for schedule(static)
            for (long i = 0; i < (long)level; i++)
                zko_hash_two(h, dg + 4 * (child + 2 * (u64)i), dg + 4 * (child + 2 * (u64)i + 1), dg + 4 * (start + (u64)i));
            level /= 2;
        }
        zko_hash_two(h, dg, dg + 4, cp);
    }
    return 0;
}

int zko_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void zko_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* Horner evaluation sum_j c_j x^j (spot checks of large LDEs). */
u64 zko_eval_poly(const u64 *c, u64 n, u64 x)
{
    u64 acc = 0;
    for (u64 j = n; j-- > 0;) acc = f_add(f_mul(acc, x), c[j]);
    return acc;
}
