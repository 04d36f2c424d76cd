// coop.cuh -- Poseidon and Poseidon2 permutations held by a group of threads.
//
// The leaf kernel hashes one leaf per thread, the throughput form.  On one
// thread a width-12 permutation is ~20 K instructions with long dependent
// carry chains: about 26 us on B200 when its warp runs alone, and that latency
// is what the narrow levels of a Merkle tree and forests of a few thousand
// leaves wait on (one permutation per level, a leaf's permutations in
// sequence).  Here an aligned group of four threads of a warp holds one state:
// thread q < 3 owns lanes 4q..4q+3, thread 3 computes on a copy of thread 0's
// constants and writes nothing.  The linear layers exchange lanes with warp
// shuffles; during the partial rounds every thread keeps its own copy of lane
// 0, so the S-box chain -- the critical path -- needs no exchange, and the
// products of the other lanes are taken while it runs.
//
// Same permutations, same constants and the same sponge as hash.cuh
// (native/poseidon/poseidon.cu, native/poseidon2/poseidon2.cu,
// native/poseidon/poseidon_permutation.cuh:84-135); lanes hold any 64-bit
// representative between layers and digests are canonicalised, so the results
// are identical to the one-thread form.  Every thread of a warp must call these
// functions together (full-warp shuffles).
#pragma once
#include <stdint.h>

#include "hash.cuh"

namespace zk {

#ifndef ZK_COOP_UNROLL
#define ZK_COOP_UNROLL 2
#endif
static constexpr int COOP_UNROLL = ZK_COOP_UNROLL;  // partial rounds per loop iteration

#ifdef __CUDACC__

struct CoopGroup {
    uint32_t q;   // thread of the group, 0..3 (3 computes on a copy)
    uint32_t qc;  // q for constant lookups (thread 3 reads thread 0's)
    uint32_t l0;  // warp lane of thread 0 of the group
    uint32_t la;  // warp lane of thread (q + 1) mod 3
    uint32_t lb;  // warp lane of thread (q + 2) mod 3
    __device__ __forceinline__ void init()
    {
        const uint32_t lane = threadIdx.x & 31u;
        q = lane & 3u;
        qc = q < 3 ? q : 0;
        l0 = lane & ~3u;
        la = l0 + (q + 1) % 3;
        lb = l0 + (q + 2) % 3;
    }
};

// Tables the threads of a group read at different indices (their own lanes'
// constants): constant-bank reads of distinct addresses serialise, so these are
// global copies read through L1.
#define ZK_COOP_TABLE(name, n, list) static __device__ const uint64_t g_##name[n] = {list};
ZK_COOP_TABLE(POSEIDON2_RC, 360, ZK_POSEIDON2_RC_LIST)
ZK_COOP_TABLE(POSEIDON2_DIAG, 12, ZK_POSEIDON2_DIAG_LIST)
ZK_COOP_TABLE(POSEIDON_RC, 360, ZK_POSEIDON_RC_LIST)
ZK_COOP_TABLE(POSEIDON_FAST_FIRST, 12, ZK_POSEIDON_FAST_FIRST_LIST)
ZK_COOP_TABLE(POSEIDON_FAST_INIT, 121, ZK_POSEIDON_FAST_INIT_LIST)
ZK_COOP_TABLE(POSEIDON_FAST_W, 242, ZK_POSEIDON_FAST_W_LIST)
ZK_COOP_TABLE(POSEIDON_FAST_V, 242, ZK_POSEIDON_FAST_V_LIST)
#define ZKG(name, i) __ldg(&g_##name[i])

__device__ __forceinline__ uint32_t coop_shfl(uint32_t v, uint32_t src) { return __shfl_sync(0xFFFFFFFFu, v, src); }
__device__ __forceinline__ uint64_t coop_shfl(uint64_t v, uint32_t src)
{
    return ((uint64_t)coop_shfl((uint32_t)(v >> 32), src) << 32) | coop_shfl((uint32_t)v, src);
}

// t[m] = lane (4q + m) mod 12 of the state: own lanes, then thread (q+1)'s, then (q+2)'s.
__device__ __forceinline__ void coop_gather(const uint64_t s[4], uint64_t t[12], const CoopGroup &c)
{
#pragma unroll
    for (int j = 0; j < 4; j++) {
        t[j] = s[j];
        t[4 + j] = coop_shfl(s[j], c.la);
        t[8 + j] = coop_shfl(s[j], c.lb);
    }
}

// Sum over the three state threads of a 64-bit partial value: any 64-bit
// representative of the total.
__device__ __forceinline__ uint64_t coop_sum3(uint64_t part, const CoopGroup &c)
{
    Sum64 acc;
    acc.set(part);
    acc.add(coop_shfl(part, c.la));
    acc.add(coop_shfl(part, c.lb));
    return acc.reduce();
}

// (r3:r2:r1:r0) + x, x < 2^64, reduced (the 128-bit sum cannot wrap: r < (2^64 - 1)^2 + 1).
__device__ __forceinline__ uint64_t coop_wide_add_reduce(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3, uint64_t x)
{
    asm("{\n\t"
        "add.cc.u32   %0, %0, %4;\n\t"
        "addc.cc.u32  %1, %1, %5;\n\t"
        "addc.cc.u32  %2, %2, 0;\n\t"
        "addc.u32     %3, %3, 0;\n\t"
        "}"
        : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3)
        : "r"((uint32_t)x), "r"((uint32_t)(x >> 32)));
    return reduce_nc(r0, r1, r2, r3);
}

// ---------------------------------------------------------------- Poseidon2

// External layer: M4 on the thread's own block (22-bit pieces, as in
// p2_external), then every lane adds its column's sum over the three blocks.
__device__ __forceinline__ void p2_external_coop(uint64_t s[4], const CoopGroup &c)
{
    uint32_t p[3][4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        p[0][j] = (uint32_t)s[j] & 0x3FFFFFu;
        p[1][j] = (uint32_t)(s[j] >> 22) & 0x3FFFFFu;
        p[2][j] = (uint32_t)(s[j] >> 44);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) p2_m4_pieces(p[k]);
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 4; j++) p[k][j] += p[k][j] + coop_shfl(p[k][j], c.la) + coop_shfl(p[k][j], c.lb);
#pragma unroll
    for (int j = 0; j < 4; j++) s[j] = p2_combine_pieces(p[0][j], p[1][j], p[2][j]);
}

__device__ __forceinline__ void p2_full_round_coop(uint64_t s[4], int r, const CoopGroup &c)
{
#pragma unroll
    for (int j = 0; j < 4; j++) s[j] = gl_sbox7_nc(gl_add_nc(s[j], ZKG(POSEIDON2_RC, 12 * r + 4 * c.qc + j)));
    p2_external_coop(s, c);
}

__device__ __forceinline__ void poseidon2_permute_coop(uint64_t s[4], const CoopGroup &c)
{
    p2_external_coop(s, c);
#pragma unroll 1
    for (int r = 0; r < 4; r++) p2_full_round_coop(s, r, c);
    // Partial rounds.  x = lane 0 in every thread; lane 0's new value is
    // d0 x' + (x' + rest) = (d0 + 1) x' + rest with rest = sum of lanes 1..11.
    uint64_t d[4];
#pragma unroll
    for (int j = 0; j < 4; j++) d[j] = ZKG(POSEIDON2_DIAG, 4 * c.qc + j);
    const uint64_t d0p1 = ZKC(POSEIDON2_DIAG)[0] + 1;
    uint64_t x = coop_shfl(s[0], c.l0);
    uint64_t rc = ZKC(POSEIDON2_RC)[12 * 4];  // lane 0's round constant, loaded a round ahead
#pragma unroll COOP_UNROLL
    for (int r = 4; r < 26; r++) {
        const uint64_t rc_next = ZKC(POSEIDON2_RC)[12 * (r + 1)];
        uint32_t pr[4][4];
#pragma unroll
        for (int j = 0; j < 4; j++) mul_wide(s[j], d[j], pr[j][0], pr[j][1], pr[j][2], pr[j][3]);
        Sum64 own;
        own.set(c.q == 0 ? 0 : s[0]);  // thread 0's s[0] is lane 0, carried in x
        own.add(s[1]);
        own.add(s[2]);
        own.add(s[3]);
        const uint64_t rest = coop_sum3(own.reduce(), c);
        x = gl_sbox7_nc(gl_add_nc(x, rc));
        rc = rc_next;
        Sum64 tot;
        tot.set(rest);
        tot.add(x);
        const uint64_t sum = tot.reduce();
#pragma unroll
        for (int j = 0; j < 4; j++) s[j] = coop_wide_add_reduce(pr[j][0], pr[j][1], pr[j][2], pr[j][3], sum);
        x = gl_mul_add_nc(x, d0p1, rest);
    }
    if (c.q == 0) s[0] = x;
#pragma unroll 1
    for (int r = 26; r < 30; r++) p2_full_round_coop(s, r, c);
}

// ----------------------------------------------------------------- Poseidon

// Full-round MDS: output lane r = sum_i circ(i) s[(i + r) mod 12] (+ 8 s[0]
// for r = 0); with t[m] = s[(m + 4q) mod 12], lane 4q + j is
// sum_i circ(i) t[(i + j) mod 12] -- the same compile-time constants in every thread.
__device__ __forceinline__ void poseidon_mds_coop(uint64_t s[4], const CoopGroup &c)
{
    uint64_t t[12];
    coop_gather(s, t, c);
    const uint32_t diag = c.q == 0 ? ZK_POSEIDON_DIAG0 : 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        Acc96 a;
        a.zero();
#pragma unroll
        for (int i = 0; i < 12; i++) a.mac(t[(i + j) % 12], poseidon_circ(i));
        if (j == 0) a.mac(t[0], diag);
        s[j] = a.reduce();
    }
}

// Sparse partial rounds of poseidon_partial_rounds with lane 0 in every thread.
__device__ __forceinline__ void poseidon_partial_rounds_coop(uint64_t s[4], const CoopGroup &c)
{
#pragma unroll
    for (int j = 0; j < 4; j++) s[j] = gl_add_nc(s[j], ZKG(POSEIDON_FAST_FIRST, 4 * c.qc + j));
    // dense 11 x 11 layer on lanes 1..11: lane L = 4q + j >= 1 takes row L - 1
    {
        uint64_t t[12];
        coop_gather(s, t, c);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t L = 4 * c.qc + j;
            const uint32_t row = L == 0 ? 0 : L - 1;  // lane 0 keeps its value
            WideAcc a;
            a.zero();
#pragma unroll
            for (int m = 0; m < 12; m++) {
                const uint32_t lam = (m + 4 * c.qc) % 12;  // lane of t[m]; lane 0 is not an input
                const uint64_t w = ZKG(POSEIDON_FAST_INIT, 11 * row + (lam == 0 ? 0 : lam - 1));
                a.mac(t[m], lam == 0 ? 0 : w);
            }
            if (L != 0) s[j] = a.reduce();
        }
    }
    uint64_t x = coop_shfl(s[0], c.l0);
#pragma unroll COOP_UNROLL
    for (int r = 0; r < 22; r++) {
        // dot product of lanes 1..11 with row r of W, from the old lanes
        WideAcc a;
        a.zero();
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t L = 4 * c.qc + j;
            a.mac(s[j], (c.q == 0 && j == 0) ? 0 : ZKG(POSEIDON_FAST_W, 11 * r + (L == 0 ? 0 : L - 1)));
        }
        const uint64_t rest = coop_sum3(a.reduce(), c);
        const uint64_t x0 = gl_add_nc(gl_sbox7_nc(x), ZKC(POSEIDON_FAST_K)[r]);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t L = 4 * c.qc + j;
            s[j] = gl_mul_add_nc(x0, ZKG(POSEIDON_FAST_V, 11 * r + (L == 0 ? 0 : L - 1)), s[j]);
        }
        x = gl_mul_add_nc(x0, (uint64_t)ZK_POSEIDON_FAST_M00, rest);
    }
    if (c.q == 0) s[0] = x;
}

__device__ __forceinline__ void poseidon_permute_coop(uint64_t s[4], const CoopGroup &c)
{
#pragma unroll 1
    for (int f = 0; f < 8; f++) {
        const int r = f < 4 ? f : f + 22;
#pragma unroll
        for (int j = 0; j < 4; j++) s[j] = gl_sbox7_nc(gl_add_nc(s[j], ZKG(POSEIDON_RC, 12 * r + 4 * c.qc + j)));
        poseidon_mds_coop(s, c);
        if (f == 3) poseidon_partial_rounds_coop(s, c);
    }
}

// ------------------------------------------------------------------ sponges

template <int H>
struct HasCoop {
    static constexpr bool value = H == HASH_POSEIDON || H == HASH_POSEIDON2;
};

template <int H>
__device__ __forceinline__ void permute_coop(uint64_t s[4], const CoopGroup &c)
{
    if constexpr (H == HASH_POSEIDON) poseidon_permute_coop(s, c);
    else poseidon2_permute_coop(s, c);
}

// sponge_hash_one with the state in the group; every thread of the group
// passes the same src and len, the digest is valid in thread 0.
template <int H>
__device__ __forceinline__ void sponge_hash_one_coop(const uint64_t *src, uint64_t len, uint64_t out[4],
                                                     const CoopGroup &c)
{
    if (len <= 4) {
#pragma unroll
        for (int i = 0; i < 4; i++) out[i] = (uint64_t)i < len ? src[i] : 0;
        return;
    }
    uint64_t s[4] = {0, 0, 0, 0};
    const uint32_t off = 4 * c.q;  // rate lanes 0..7 belong to threads 0 and 1
    for (uint64_t idx = 0; idx < len; idx += 8) {
        if (c.q < 2) {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (idx + off + j < len) s[j] = src[idx + off + j];
        }
        permute_coop<H>(s, c);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) out[i] = gl_canon(s[i]);
}

// sponge_hash_two: state [l, r, 0]; the digest is valid in thread 0.
template <int H>
__device__ __forceinline__ void sponge_hash_two_coop(const uint64_t *l, const uint64_t *r, uint64_t out[4],
                                                     const CoopGroup &c)
{
    const uint64_t *src = c.q == 0 ? l : r;
    uint64_t s[4];
#pragma unroll
    for (int i = 0; i < 4; i++) s[i] = c.q < 2 ? src[i] : 0;
    permute_coop<H>(s, c);
#pragma unroll
    for (int i = 0; i < 4; i++) out[i] = gl_canon(s[i]);
}

#endif  // __CUDACC__

}  // namespace zk
