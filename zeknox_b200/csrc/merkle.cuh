// merkle.cuh -- linear-layout Merkle forest builder (device side).
//
// Replaces native/merkle/merkle.cu:24-280 of zeknox.  Layout (unchanged, it is
// the ABI): 2^cap_height subtrees of L leaves; subtree k owns digests
// [k(2L-2), (k+1)(2L-2)); in it the level with 2^r nodes starts at 2^r - 2,
// node i of a level has children 2(i+1)+start and 2(i+1)+1+start of the level
// below, leaf digests start at L-2, and the subtree root H2(d[0], d[1]) is
// cap[k].
//
// Kernel structure (B200-first instead of one launch per level):
//   * leaf kernel: one thread per leaf runs the sponge with the state in
//     registers (nothing else, so no warp idles on a barrier);
//   * level kernel: one thread per node of one level, for the wide levels
//     just above the leaves (and for levels a tail CTA cannot hold);
//   * fold kernel: each CTA folds T consecutive nodes log2(T) levels up in
//     shared memory, writing every node, and the caps of subtrees that fit;
//   * tail kernel: one CTA per subtree folds the remaining levels in shared
//     memory and writes the cap.
#pragma once
#include <stdint.h>

#include "bounds.cuh"
#include "coop.cuh"
#include "hash.cuh"

namespace zk {

struct MerkleGeom {
    uint64_t n_leaves;
    uint64_t leaf_size;
    uint64_t sub_leaves;   // L
    uint64_t sub_digests;  // 2L - 2
    uint32_t log_sub;      // log2 L
    uint32_t n_caps;
};

__device__ __forceinline__ uint64_t merkle_node_index(const MerkleGeom &g, uint64_t first_leaf, uint32_t level_u)
{
    // node at height level_u (leaves are height 0) covering leaves starting at first_leaf
    uint64_t k = first_leaf >> g.log_sub;
    uint64_t in_sub = first_leaf & (g.sub_leaves - 1);
    uint64_t level_nodes = g.sub_leaves >> level_u;
    return k * g.sub_digests + (level_nodes - 2) + (in_sub >> level_u);
}

// Words of the digest buffer and of the leaves (the extents the checked build
// tests accesses against).
__device__ __forceinline__ uint64_t merkle_digest_words(const MerkleGeom &g) { return 4 * (uint64_t)g.n_caps * g.sub_digests; }
__device__ __forceinline__ uint64_t merkle_leaf_words(const MerkleGeom &g) { return g.n_leaves * g.leaf_size; }

template <int H>
__device__ __forceinline__ void leaf_hash(const uint64_t *__restrict__ row, uint64_t len, uint64_t out[4])
{
    hash_one<H>(row, len, out);
}

// Leaf digests only: one thread per leaf, no shared memory, no barriers, so
// every warp stays on the hash for the whole kernel.
template <int H, int T>
__device__ __forceinline__ void merkle_leaf_body(const uint64_t *__restrict__ leaves, uint64_t *__restrict__ digests,
                                                 uint64_t *__restrict__ caps, const MerkleGeom &g)
{
    const uint64_t i = (uint64_t)blockIdx.x * T + threadIdx.x;
    if (i >= g.n_leaves) return;
    // caps == leaves: the leaf hashes are the caps, digests untouched
    uint64_t *dst = g.sub_leaves == 1 ? caps + 4 * i : digests + 4 * merkle_node_index(g, i, 0);
    if (g.sub_leaves == 1 ? !ZK_IN_BOUNDS(4 * i + 3, 4 * (uint64_t)g.n_caps, OOB_MERKLE_CAP)
                          : !ZK_IN_BOUNDS(4 * merkle_node_index(g, i, 0) + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST))
        return;
    if (g.leaf_size && !ZK_IN_BOUNDS((i + 1) * g.leaf_size - 1, merkle_leaf_words(g), OOB_MERKLE_LEAF)) return;
    uint64_t d[4];
    if (H == HASH_KECCAK && g.leaf_size < 4) {
        // Keccak copies a < 4-word leaf and leaves the other digest words as
        // they are in the output buffer (native/keccak/keccak.cu:118-121)
#pragma unroll
        for (int q = 0; q < 4; q++) d[q] = dst[q];
    }
    leaf_hash<H>(leaves + i * g.leaf_size, g.leaf_size, d);
#pragma unroll
    for (int q = 0; q < 4; q++) dst[q] = d[q];
}

template <int H, int T>
__global__ void __launch_bounds__(T)
    merkle_leaf_kernel(const uint64_t *__restrict__ leaves, uint64_t *__restrict__ digests, uint64_t *__restrict__ caps,
                       MerkleGeom g)
{
    merkle_leaf_body<H, T>(leaves, digests, caps, g);
}

// The same, held to 1024 threads per SM (64 registers): measured 1.02-1.03x
// for Poseidon and Poseidon2 leaves on B200, and slower for the other hashes,
// which keep the unconstrained kernel above.
template <int H, int T>
__global__ void __launch_bounds__(T, 1024 / T)
    merkle_leaf_kernel_1k(const uint64_t *__restrict__ leaves, uint64_t *__restrict__ digests,
                          uint64_t *__restrict__ caps, MerkleGeom g)
{
    merkle_leaf_body<H, T>(leaves, digests, caps, g);
}

// Leaf digests plus the LV tree levels above them inside the CTA (sponge
// hashes only; needs T leaves per CTA inside one subtree and LV < log2 T,
// LV <= the subtree's top height).  A node is the sponge hash of its two
// children's 8 consecutive words, so leaves and nodes go through the same
// call site and the permutation's code exists once.
template <int H, int T, int LV>
__global__ void __launch_bounds__(T, 1024 / T)
    merkle_leaf_levels_kernel(const uint64_t *__restrict__ leaves, uint64_t *__restrict__ digests, MerkleGeom g)
{
    __shared__ uint64_t nd[T][4];
    const uint64_t i0 = (uint64_t)blockIdx.x * T;
    const uint32_t t = threadIdx.x;
#pragma unroll 1
    for (int v = 0; v <= LV; v++) {
        const uint32_t nodes = T >> v;
        uint64_t h[4];
        if (t < nodes) {
            const uint64_t *src = v == 0 ? leaves + (i0 + t) * g.leaf_size : &nd[2 * t][0];
            const bool row_ok =
                v != 0 || ZK_IN_BOUNDS((i0 + t + 1) * g.leaf_size - 1, merkle_leaf_words(g), OOB_MERKLE_LEAF);
            if (row_ok) sponge_hash_one<H>(src, v == 0 ? g.leaf_size : 8, h);
            const uint64_t di = merkle_node_index(g, i0 + ((uint64_t)t << v), (uint32_t)v);
            if (row_ok && ZK_IN_BOUNDS(4 * di + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST)) {
#pragma unroll
                for (int q = 0; q < 4; q++) digests[4 * di + q] = h[q];
            }
        }
        __syncthreads();
        if (t < nodes) {
#pragma unroll
            for (int q = 0; q < 4; q++) nd[t][q] = h[q];
        }
        __syncthreads();
    }
}

// Leaf kernel of hash H with CTAs of T threads.
template <int H, int T>
constexpr auto merkle_leaf_kernel_for()
{
    if constexpr (H == HASH_POSEIDON || H == HASH_POSEIDON2) return merkle_leaf_kernel_1k<H, T>;
    else return merkle_leaf_kernel<H, T>;
}

// Folds stored digests upwards from height u0 (0 = leaf digests): each CTA
// takes T consecutive nodes of that height and computes every node above them
// whose subtree lies in the CTA (up to log2 T levels, or up to the subtree's
// two top nodes), writing each node; when whole subtrees fit in the CTA it
// also writes their caps.
template <int H, int T>
__global__ void __launch_bounds__(T) merkle_fold_kernel(uint64_t *__restrict__ digests, uint64_t *__restrict__ caps,
                                                        MerkleGeom g, uint32_t u0)
{
    __shared__ uint64_t node[T][4];
    const uint64_t count = g.n_leaves >> u0;     // nodes at height u0
    const uint64_t i0 = (uint64_t)blockIdx.x * T;  // first node of this CTA (height u0)
    const uint32_t t = threadIdx.x;
    const uint64_t cta_nodes = count - i0 < (uint64_t)T ? count - i0 : (uint64_t)T;
    if (t < cta_nodes) {
        const uint64_t di = merkle_node_index(g, (i0 + t) << u0, u0);
        const bool ok = ZK_IN_BOUNDS(4 * di + 3, merkle_digest_words(g), OOB_MERKLE_NODE);
#pragma unroll
        for (int q = 0; q < 4; q++) node[t][q] = ok ? digests[4 * di + q] : 0;
    }
    const uint32_t top = g.log_sub - 1;  // highest stored height
    uint32_t U = 0;
    while ((1u << (U + 1)) <= T && u0 + U + 1 <= top) U++;
    for (uint32_t v = 1; v <= U; v++) {
        __syncthreads();
        const uint32_t nodes = T >> v;
        uint64_t h[4];
        const bool act = t < nodes && ((uint64_t)t << v) < cta_nodes;
        if (act) {
            hash_two<H>(node[2 * t], node[2 * t + 1], h);
            const uint64_t di = merkle_node_index(g, (i0 + ((uint64_t)t << v)) << u0, u0 + v);
            if (ZK_IN_BOUNDS(4 * di + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST)) {
#pragma unroll
                for (int q = 0; q < 4; q++) digests[4 * di + q] = h[q];
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int q = 0; q < 4; q++) node[t][q] = h[q];
        }
    }
    const uint64_t sub_nodes = g.sub_leaves >> u0;  // height-u0 nodes per subtree
    if (u0 + U == top && sub_nodes <= (uint64_t)T) {
        __syncthreads();
        const uint32_t subs = (uint32_t)(cta_nodes / sub_nodes);
        if (t < subs) {
            uint64_t h[4];
            hash_two<H>(node[2 * t], node[2 * t + 1], h);
            const uint64_t k = ((i0 << u0) >> g.log_sub) + t;
            if (ZK_IN_BOUNDS(4 * k + 3, 4 * (uint64_t)g.n_caps, OOB_MERKLE_CAP)) {
#pragma unroll
                for (int q = 0; q < 4; q++) caps[4 * k + q] = h[q];
            }
        }
    }
}

// One CTA per subtree: starting from the stored level of height u0 (m nodes per
// subtree, 2 < m <= MAXM), fold to 2 nodes and write the cap.  Two shared
// buffers (MAXM and MAXM/2 digests) alternate between levels.
template <int H, int MAXM>
__global__ void __launch_bounds__(256) merkle_tail_kernel(uint64_t *__restrict__ digests, uint64_t *__restrict__ caps,
                                                          MerkleGeom g, uint32_t u0)
{
    __shared__ uint64_t bufa[MAXM][4];
    __shared__ uint64_t bufb[MAXM / 2][4];
    const uint64_t k = blockIdx.x;
    uint64_t *sub = digests + k * g.sub_digests * 4;
    const uint64_t sub0 = k * g.sub_digests * 4;  // sub's first word in the digest buffer
    uint32_t m = (uint32_t)(g.sub_leaves >> u0);
    for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
        const bool ok = ZK_IN_BOUNDS(sub0 + 4 * (m - 2 + j) + 3, merkle_digest_words(g), OOB_MERKLE_NODE);
#pragma unroll
        for (int q = 0; q < 4; q++) bufa[j][q] = ok ? sub[4 * (m - 2 + j) + q] : 0;
    }
    uint64_t(*src)[4] = bufa;
    uint64_t(*dst)[4] = bufb;
    while (m > 2) {
        __syncthreads();
        uint32_t half = m / 2;
        for (uint32_t j = threadIdx.x; j < half; j += blockDim.x) {
            uint64_t h[4];
            hash_two<H>(src[2 * j], src[2 * j + 1], h);
            const bool ok = ZK_IN_BOUNDS(sub0 + 4 * (half - 2 + j) + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (ok) sub[4 * (half - 2 + j) + q] = h[q];
                dst[j][q] = h[q];
            }
        }
        uint64_t(*tmp)[4] = src;
        src = dst;
        dst = tmp;
        m = half;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t h[4];
        hash_two<H>(src[0], src[1], h);
        if (ZK_IN_BOUNDS(4 * k + 3, 4 * (uint64_t)g.n_caps, OOB_MERKLE_CAP)) {
#pragma unroll
            for (int q = 0; q < 4; q++) caps[4 * k + q] = h[q];
        }
    }
}

// One level, node-parallel, for very large subtrees (m > tail capacity).
template <int H>
__global__ void merkle_level_kernel(uint64_t *__restrict__ digests, MerkleGeom g, uint32_t u)
{
    uint64_t per_sub = g.sub_leaves >> u;
    uint64_t total = per_sub * g.n_caps;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = x / per_sub, j = x % per_sub;
        uint64_t *sub = digests + k * g.sub_digests * 4;
        uint64_t start = per_sub - 2, child = 2 * per_sub - 2;
        const uint64_t sub0 = k * g.sub_digests * 4;
        if (!ZK_IN_BOUNDS(sub0 + 4 * (child + 2 * j + 1) + 3, merkle_digest_words(g), OOB_MERKLE_NODE) ||
            !ZK_IN_BOUNDS(sub0 + 4 * (start + j) + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST))
            continue;
        uint64_t h[4];
        hash_two<H>(sub + 4 * (child + 2 * j), sub + 4 * (child + 2 * j + 1), h);
#pragma unroll
        for (int q = 0; q < 4; q++) sub[4 * (start + j) + q] = h[q];
    }
}

// ------------------------------------------------------ cooperative kernels
//
// Poseidon and Poseidon2 with one permutation per group of four threads
// (coop.cuh): the leaves of forests too small to fill the GPU with one leaf
// per thread, and the tree levels below the wide ones, whose time is the
// latency of one permutation per level.  A warp holds eight groups; a group
// with nothing to do hashes a copy of its warp's first task and writes
// nothing, and a warp with nothing to do skips the level, so the full-warp
// shuffles always see all 32 threads.

// Leaf digests, one leaf per group.
template <int H, int T>
__global__ void __launch_bounds__(T)
    merkle_leaf_coop_kernel(const uint64_t *__restrict__ leaves, uint64_t *__restrict__ digests,
                            uint64_t *__restrict__ caps, MerkleGeom g)
{
    CoopGroup c;
    c.init();
    const uint64_t gi = ((uint64_t)blockIdx.x * T + threadIdx.x) >> 2;
    if ((gi & ~7ULL) >= g.n_leaves) return;  // the whole warp is past the end
    const uint64_t i = gi < g.n_leaves ? gi : g.n_leaves - 1;
    uint64_t d[4];
    // (every thread of the warp runs the permutation: a row out of range is
    // hashed from row 0 and its digest not written)
    const bool row_ok = !g.leaf_size || ZK_IN_BOUNDS((i + 1) * g.leaf_size - 1, merkle_leaf_words(g), OOB_MERKLE_LEAF);
    sponge_hash_one_coop<H>(leaves + (row_ok ? i : 0) * g.leaf_size, g.leaf_size, d, c);
    const bool dst_ok = g.sub_leaves == 1
                            ? ZK_IN_BOUNDS(4 * gi + 3, 4 * (uint64_t)g.n_caps, OOB_MERKLE_CAP)
                            : ZK_IN_BOUNDS(4 * merkle_node_index(g, gi, 0) + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST);
    if (c.q == 0 && gi < g.n_leaves && row_ok && dst_ok) {
        uint64_t *dst = g.sub_leaves == 1 ? caps + 4 * gi : digests + 4 * merkle_node_index(g, gi, 0);
#pragma unroll
        for (int q = 0; q < 4; q++) dst[q] = d[q];
    }
}

// merkle_fold_kernel with T / 4 nodes of height u0 per CTA.
template <int H, int T>
__global__ void __launch_bounds__(T) merkle_fold_coop_kernel(uint64_t *__restrict__ digests, uint64_t *__restrict__ caps,
                                                             MerkleGeom g, uint32_t u0)
{
    constexpr uint32_t NG = T / 4;
    __shared__ uint64_t node[NG][4];
    CoopGroup c;
    c.init();
    const uint32_t grp = threadIdx.x >> 2;
    const uint32_t wg = grp & ~7u;  // first group of this warp
    const uint64_t count = g.n_leaves >> u0;
    const uint64_t i0 = (uint64_t)blockIdx.x * NG;
    const uint64_t cta_nodes = count - i0 < (uint64_t)NG ? count - i0 : (uint64_t)NG;
    for (uint32_t t = threadIdx.x; t < 4 * cta_nodes; t += T) {
        const uint64_t wi = 4 * merkle_node_index(g, (i0 + (t >> 2)) << u0, u0) + (t & 3);
        node[t >> 2][t & 3] = ZK_IN_BOUNDS(wi, merkle_digest_words(g), OOB_MERKLE_NODE) ? digests[wi] : 0;
    }
    const uint32_t top = g.log_sub - 1;
    uint32_t U = 0;
    while ((1u << (U + 1)) <= NG && u0 + U + 1 <= top) U++;
    for (uint32_t v = 1; v <= U; v++) {
        __syncthreads();
        const uint32_t nodes = NG >> v;
        const bool act = grp < nodes && ((uint64_t)grp << v) < cta_nodes;
        const bool wact = wg < nodes && ((uint64_t)wg << v) < cta_nodes;
        uint64_t h[4];
        if (wact) {
            const uint32_t src = act ? grp : wg;
            sponge_hash_two_coop<H>(node[2 * src], node[2 * src + 1], h, c);
            if (act && c.q == 0) {
                const uint64_t di = merkle_node_index(g, (i0 + ((uint64_t)grp << v)) << u0, u0 + v);
                if (ZK_IN_BOUNDS(4 * di + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST)) {
#pragma unroll
                    for (int q = 0; q < 4; q++) digests[4 * di + q] = h[q];
                }
            }
        }
        __syncthreads();
        if (act && c.q == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) node[grp][q] = h[q];
        }
    }
    const uint64_t sub_nodes = g.sub_leaves >> u0;
    if (u0 + U == top && sub_nodes <= (uint64_t)NG) {
        __syncthreads();
        const uint32_t subs = (uint32_t)(cta_nodes / sub_nodes);
        if (wg < subs) {
            const bool act = grp < subs;
            const uint32_t src = act ? grp : wg;
            uint64_t h[4];
            sponge_hash_two_coop<H>(node[2 * src], node[2 * src + 1], h, c);
            if (act && c.q == 0) {
                const uint64_t k = ((i0 << u0) >> g.log_sub) + grp;
                if (ZK_IN_BOUNDS(4 * k + 3, 4 * (uint64_t)g.n_caps, OOB_MERKLE_CAP)) {
#pragma unroll
                    for (int q = 0; q < 4; q++) caps[4 * k + q] = h[q];
                }
            }
        }
    }
}

// merkle_tail_kernel with one permutation per group: one CTA of 256 threads
// (64 groups) per subtree.
template <int H, int MAXM>
__global__ void __launch_bounds__(256) merkle_tail_coop_kernel(uint64_t *__restrict__ digests, uint64_t *__restrict__ caps,
                                                               MerkleGeom g, uint32_t u0)
{
    constexpr uint32_t NG = 256 / 4;
    __shared__ uint64_t bufa[MAXM][4];
    __shared__ uint64_t bufb[MAXM / 2][4];
    CoopGroup c;
    c.init();
    const uint32_t grp = threadIdx.x >> 2;
    const uint64_t k = blockIdx.x;
    uint64_t *sub = digests + k * g.sub_digests * 4;
    const uint64_t sub0 = k * g.sub_digests * 4;
    uint32_t m = (uint32_t)(g.sub_leaves >> u0);
    for (uint32_t j = threadIdx.x; j < 4 * m; j += 256)
        bufa[j >> 2][j & 3] =
            ZK_IN_BOUNDS(sub0 + 4 * (m - 2) + j, merkle_digest_words(g), OOB_MERKLE_NODE) ? sub[4 * (m - 2) + j] : 0;
    uint64_t(*src)[4] = bufa;
    uint64_t(*dst)[4] = bufb;
    while (m > 2) {
        __syncthreads();
        const uint32_t half = m / 2;
        for (uint32_t base = grp & ~7u; base < half; base += NG) {
            const uint32_t j = base + (grp & 7u);
            const bool act = j < half;
            const uint32_t jj = act ? j : base;
            uint64_t h[4];
            sponge_hash_two_coop<H>(src[2 * jj], src[2 * jj + 1], h, c);
            if (act && c.q == 0) {
                const bool ok = ZK_IN_BOUNDS(sub0 + 4 * (half - 2 + j) + 3, merkle_digest_words(g), OOB_MERKLE_DIGEST);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (ok) sub[4 * (half - 2 + j) + q] = h[q];
                    dst[j][q] = h[q];
                }
            }
        }
        uint64_t(*tmp)[4] = src;
        src = dst;
        dst = tmp;
        m = half;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t h[4];
        sponge_hash_two_coop<H>(src[0], src[1], h, c);
        if (threadIdx.x == 0 && ZK_IN_BOUNDS(4 * k + 3, 4 * (uint64_t)g.n_caps, OOB_MERKLE_CAP)) {
#pragma unroll
            for (int q = 0; q < 4; q++) caps[4 * k + q] = h[q];
        }
    }
}

}  // namespace zk
