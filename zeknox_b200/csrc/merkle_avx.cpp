// merkle_avx.cpp -- Poseidon Merkle forests on the host's vector units.
//
// The reference's optional AVX2 / AVX-512 host builder
// (native/merkle/merkle_avx.cpp, exported as fill_digests_buf_linear_cpu_avx and
// fill_digests_buf_linear_cpu_avx512 when built with USE_AVX / USE_AVX512;
// Poseidon only) vectorises one state across the lanes of a register.  Here
// every vector lane is a different state: W = 8 (AVX-512) or 4 (AVX2)
// leaves or nodes are hashed together, lane i of vector k holding lane k of
// state i, so the permutation is the scalar one with every operation made W
// wide -- no shuffles.  The Goldilocks product is built from four 32x32->64
// lane products (vpmuludq) and the same reduction as gl_reduce128; the full-
// round MDS is the exact small-constant product over 32-bit halves (as Acc96);
// the partial rounds use the sparse form of hash.cuh.  Values stay canonical.
//
// This file is compiled twice, with -mavx512f -DZK_SIMD_W=8 and with -mavx2
// -DZK_SIMD_W=4, into zk_merkle_poseidon_avx512 / zk_merkle_poseidon_avx2.
// It includes no C++ headers and everything but the entry point has internal
// linkage, so no inline function compiled for those ISAs can be picked by the
// linker for code that runs on other CPUs; the callers (abi.cu) check the CPU
// before calling.
#include <immintrin.h>
#include <stdint.h>
#include <string.h>

#include "zk_constants.h"

#ifndef ZK_SIMD_W
#error "ZK_SIMD_W must be 8 (AVX-512) or 4 (AVX2)"
#endif

namespace {

constexpr int W = ZK_SIMD_W;
constexpr uint64_t P = 0xFFFFFFFF00000001ULL;
constexpr uint64_t EPS = 0xFFFFFFFFULL;

#define ZK_INL static inline __attribute__((always_inline))

#if ZK_SIMD_W == 8
typedef __m512i V;
typedef __mmask8 M;
ZK_INL V vset1(uint64_t x) { return _mm512_set1_epi64((long long)x); }
ZK_INL V vload(const uint64_t *p) { return _mm512_loadu_si512((const void *)p); }
ZK_INL void vstore(uint64_t *p, V v) { _mm512_storeu_si512((void *)p, v); }
ZK_INL V vadd(V a, V b) { return _mm512_add_epi64(a, b); }
ZK_INL V vsub(V a, V b) { return _mm512_sub_epi64(a, b); }
ZK_INL V vand(V a, V b) { return _mm512_and_si512(a, b); }
ZK_INL V vsrl32(V a) { return _mm512_srli_epi64(a, 32); }
ZK_INL V vsll32(V a) { return _mm512_slli_epi64(a, 32); }
ZK_INL V vmul32(V a, V b) { return _mm512_mul_epu32(a, b); }
ZK_INL M vltu(V a, V b) { return _mm512_cmplt_epu64_mask(a, b); }
ZK_INL M vgeu(V a, V b) { return _mm512_cmpge_epu64_mask(a, b); }
ZK_INL M mor(M a, M b) { return (M)(a | b); }
ZK_INL V vsel(M m, V a, V b) { return _mm512_mask_blend_epi64(m, a, b); }  // m ? b : a
#define ZK_SIMD_ENTRY zk_merkle_poseidon_avx512
#elif ZK_SIMD_W == 4
typedef __m256i V;
typedef __m256i M;  // all-ones lanes
ZK_INL V vset1(uint64_t x) { return _mm256_set1_epi64x((long long)x); }
ZK_INL V vload(const uint64_t *p) { return _mm256_loadu_si256((const __m256i *)p); }
ZK_INL void vstore(uint64_t *p, V v) { _mm256_storeu_si256((__m256i *)p, v); }
ZK_INL V vadd(V a, V b) { return _mm256_add_epi64(a, b); }
ZK_INL V vsub(V a, V b) { return _mm256_sub_epi64(a, b); }
ZK_INL V vand(V a, V b) { return _mm256_and_si256(a, b); }
ZK_INL V vsrl32(V a) { return _mm256_srli_epi64(a, 32); }
ZK_INL V vsll32(V a) { return _mm256_slli_epi64(a, 32); }
ZK_INL V vmul32(V a, V b) { return _mm256_mul_epu32(a, b); }
// unsigned compare by flipping the sign bits (AVX2 has only the signed one)
ZK_INL M vltu(V a, V b)
{
    const V s = _mm256_set1_epi64x((long long)0x8000000000000000ULL);
    return _mm256_cmpgt_epi64(_mm256_xor_si256(b, s), _mm256_xor_si256(a, s));
}
ZK_INL M vgeu(V a, V b) { return _mm256_xor_si256(vltu(a, b), _mm256_set1_epi64x(-1)); }
ZK_INL M mor(M a, M b) { return _mm256_or_si256(a, b); }
ZK_INL V vsel(M m, V a, V b) { return _mm256_blendv_epi8(a, b, m); }  // m ? b : a
#define ZK_SIMD_ENTRY zk_merkle_poseidon_avx2
#else
#error "ZK_SIMD_W must be 8 or 4"
#endif

// ------------------------------------------------------------ field, W wide

ZK_INL V canon(V x) { return vsel(vgeu(x, vset1(P)), x, vsub(x, vset1(P))); }

// a + b for canonical a, b (the scalar gl_add)
ZK_INL V gadd(V a, V b)
{
    const V s = vadd(a, b);
    const V t = vadd(s, vset1(EPS));
    return vsel(mor(vltu(s, a), vltu(t, s)), s, t);
}

// lo + 2^64 hi reduced to a canonical value (the scalar gl_reduce128)
ZK_INL V reduce128(V lo, V hi)
{
    const V h1 = vsrl32(hi), h0 = vand(hi, vset1(EPS));
    V t0 = vsub(lo, h1);
    t0 = vsel(vltu(lo, h1), t0, vsub(t0, vset1(EPS)));
    const V t1 = vsub(vsll32(h0), h0);
    V t2 = vadd(t0, t1);
    t2 = vsel(vltu(t2, t1), t2, vadd(t2, vset1(EPS)));
    return canon(t2);
}

// a * b: four 32x32->64 lane products, the 128-bit sum with its carries, reduced
ZK_INL V gmul(V a, V b)
{
    const V ah = vsrl32(a), bh = vsrl32(b);
    const V p00 = vmul32(a, b), p01 = vmul32(a, bh), p10 = vmul32(ah, b), p11 = vmul32(ah, bh);
    const V mid = vadd(p01, p10);          // may wrap: then 2^96 is missing
    const V lo = vadd(p00, vsll32(mid));   // may wrap: then 2^64 is missing
    V hi = vadd(p11, vsrl32(mid));
    hi = vsel(vltu(mid, p01), hi, vadd(hi, vset1(1ULL << 32)));
    hi = vsel(vltu(lo, p00), hi, vadd(hi, vset1(1)));
    return reduce128(lo, hi);
}

ZK_INL V sbox7(V x)
{
    const V x2 = gmul(x, x);
    const V x4 = gmul(x2, x2);
    const V x3 = gmul(x2, x);
    return gmul(x3, x4);
}

// ----------------------------------------------------------------- Poseidon

const uint64_t RC[360] = {ZK_POSEIDON_RC_LIST};
const uint32_t CIRC[12] = {ZK_POSEIDON_CIRC_LIST};
const uint64_t FIRST[12] = {ZK_POSEIDON_FAST_FIRST_LIST};
const uint64_t INIT[121] = {ZK_POSEIDON_FAST_INIT_LIST};
const uint64_t K[22] = {ZK_POSEIDON_FAST_K_LIST};
const uint64_t FW[242] = {ZK_POSEIDON_FAST_W_LIST};
const uint64_t FV[242] = {ZK_POSEIDON_FAST_V_LIST};

// circ(17,15,41,16,2,28,13,13,39,18,34,20) + diag(8,0,...): exact sums of the
// 32-bit halves times the constants (< 2^32 * 264 < 2^41), recombined, reduced.
ZK_INL void mds(V s[12])
{
    V lo[12], hi[12];
    for (int i = 0; i < 12; i++) {
        lo[i] = vand(s[i], vset1(EPS));
        hi[i] = vsrl32(s[i]);
    }
    V t[12];
    for (int r = 0; r < 12; r++) {
        V al = vset1(0), ah = vset1(0);
        for (int i = 0; i < 12; i++) {
            const V c = vset1(CIRC[i] + (r == 0 && i == 0 ? ZK_POSEIDON_DIAG0 : 0));
            al = vadd(al, vmul32(lo[(i + r) % 12], c));
            ah = vadd(ah, vmul32(hi[(i + r) % 12], c));
        }
        // al + 2^32 ah = l + 2^64 h, h < 2^9
        const V l = vadd(al, vsll32(ah));
        V h = vsrl32(ah);
        h = vsel(vltu(l, al), h, vadd(h, vset1(1)));
        V x = vadd(l, vsub(vsll32(h), h));  // + h * EPS (< 2^41)
        x = vsel(vltu(x, l), x, vadd(x, vset1(EPS)));
        t[r] = canon(x);
    }
    for (int i = 0; i < 12; i++) s[i] = t[i];
}

void permute(V s[12])
{
    for (int f = 0; f < 8; f++) {
        const int r = f < 4 ? f : f + 22;
        for (int i = 0; i < 12; i++) s[i] = sbox7(gadd(s[i], vset1(RC[12 * r + i])));
        mds(s);
        if (f != 3) continue;
        // partial rounds, sparse form
        for (int i = 0; i < 12; i++) s[i] = gadd(s[i], vset1(FIRST[i]));
        V t[11];
        for (int i = 0; i < 11; i++) {
            V a = gmul(s[1], vset1(INIT[11 * i]));
            for (int j = 1; j < 11; j++) a = gadd(a, gmul(s[1 + j], vset1(INIT[11 * i + j])));
            t[i] = a;
        }
        for (int i = 0; i < 11; i++) s[1 + i] = t[i];
        for (int q = 0; q < 22; q++) {
            const V x0 = gadd(sbox7(s[0]), vset1(K[q]));
            V a = gmul(x0, vset1(ZK_POSEIDON_FAST_M00));
            for (int i = 0; i < 11; i++) a = gadd(a, gmul(s[1 + i], vset1(FW[11 * q + i])));
            s[0] = a;
            for (int i = 0; i < 11; i++) s[1 + i] = gadd(s[1 + i], gmul(x0, vset1(FV[11 * q + i])));
        }
    }
}

// Digests of `count` inputs of `len` words, input j at src + j * stride:
// the Plonky2 overwrite sponge (rate 8, zero initial state; <= 4 words are the
// digest themselves, zero padded), W inputs per permutation.
void hash_many(const uint64_t *src, uint64_t stride, uint64_t len, uint64_t count, uint64_t *out)
{
    if (len <= 4) {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < (int64_t)count; j++)
            for (uint64_t q = 0; q < 4; q++) out[4 * j + q] = q < len ? src[j * stride + q] : 0;
        return;
    }
    const int64_t blocks = (int64_t)((count + W - 1) / W);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < blocks; b++) {
        const uint64_t *row[W];
        for (int l = 0; l < W; l++) {
            uint64_t j = (uint64_t)b * W + l;
            row[l] = src + (j < count ? j : count - 1) * stride;  // a short block repeats its last input
        }
        V s[12];
        for (int i = 0; i < 12; i++) s[i] = vset1(0);
        alignas(64) uint64_t buf[W];
        for (uint64_t idx = 0; idx < len; idx += 8) {
            const uint64_t k = len - idx < 8 ? len - idx : 8;
            for (uint64_t i = 0; i < k; i++) {
                for (int l = 0; l < W; l++) buf[l] = row[l][idx + i];
                s[i] = vload(buf);
            }
            permute(s);
        }
        alignas(64) uint64_t d[4][W];
        for (int q = 0; q < 4; q++) vstore(d[q], s[q]);
        for (int l = 0; l < W; l++) {
            const uint64_t j = (uint64_t)b * W + l;
            if (j >= count) break;
            for (int q = 0; q < 4; q++) out[4 * j + q] = d[q][l];
        }
    }
}

}  // namespace

// The linear forest of native/merkle/merkle.cpp:20-124 with Poseidon, for
// arguments the caller has checked (merkle_geometry_check).
extern "C" void ZK_SIMD_ENTRY(uint64_t *dig, uint64_t *cap, const uint64_t *leaves, uint64_t n_dig, uint64_t n_cap,
                              uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height)
{
    if (n_cap == n_leaves) {
        hash_many(leaves, leaf_size, leaf_size, n_leaves, cap);
        return;
    }
    const uint64_t L = n_leaves >> cap_height, D = n_dig >> cap_height;
    for (uint64_t k = 0; k < n_cap; k++) {
        const uint64_t *lv = leaves + k * L * leaf_size;
        uint64_t *dg = dig + k * D * 4;
        // leaf digests at [L - 2, 2L - 2), each level of m nodes at [m - 2, 2m - 2),
        // node i's children the 8 consecutive words at 2(i + 1) + start of the level below
        hash_many(lv, leaf_size, leaf_size, L, dg + (D - L) * 4);
        for (uint64_t m = L / 2; m >= 2; m /= 2) hash_many(dg + 4 * (2 * m - 2), 8, 8, m, dg + 4 * (m - 2));
        hash_many(dg, 8, 8, 1, cap + 4 * k);
    }
}
