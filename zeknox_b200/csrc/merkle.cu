// merkle.cu -- host driver of the Merkle forest builder.
//
// Follows native/merkle/merkle.cu:166-280 of zeknox for the layout and the
// special cases (caps == leaves; subtrees of 1 or 2 leaves).  Launches: the
// leaf kernel; one node-parallel level kernel per level while a level still
// has >= wide_level_nodes nodes; the fold kernel (the next 8 levels inside
// CTAs, and the caps when whole subtrees fit); for subtrees still above 1024
// nodes, level kernels, then one tail CTA per subtree -- 2 to 6 launches where
// the reference launches one per level.  Poseidon2's leaf kernel also builds
// the first three levels above the leaves in its CTAs.  For Poseidon and Poseidon2 the fold
// and tail kernels (and the leaf kernel of forests of at most coop_leaves
// leaves) run one permutation per group of four threads (coop.cuh): the fold
// kernel then takes 6 levels per launch.
#include <cstdio>
#include <string>

#include "geom.h"
#include "merkle.cuh"
#include "ntt_api.cuh"
#include "runtime.cuh"

namespace zk {

static constexpr int LEAF_T = 256;     // default leaves (threads) per CTA of the leaf kernel ("leaf_threads.<hash>")
// Poseidon-BN128's leaf kernel holds 136 registers a thread: three 128-thread
// CTAs fit an SM (12 warps) where one 256-thread CTA does (measured on 2^20 x
// 135 forests: 450 against 491 ms; 2^14 x 135: 18.0 against 23.9 ms)
template <int H>
constexpr int leaf_t_default()
{
    return H == HASH_POSEIDON_BN128 ? 128 : LEAF_T;
}
// Threads per CTA of the node-parallel level kernel: 128 for Poseidon-BN128
// (158 registers: three CTAs per SM instead of one), 256 otherwise.  The wide
// levels are ~6% of a forest's permutations: 2^20 x 135 Poseidon-BN128
// forest 449.0 against 450.2 ms.
template <int H>
constexpr unsigned level_t()
{
    return H == HASH_POSEIDON_BN128 ? 128u : 256u;
}
static constexpr int FOLD_T = 256;     // leaf digests per CTA of the fold kernel
static constexpr int TAIL_MAXM = 1024; // nodes a tail CTA can take
static constexpr int LEAF_LEVELS = 3;  // tree levels the Poseidon2 leaf kernel folds in its CTAs
static constexpr int COOP_T = 256;     // threads (64 groups of four) per CTA of the cooperative kernels
static constexpr uint64_t COOP_LEAVES = 1ULL << 13;  // default: forests up to this many leaves hash their leaves
                                                     // with the cooperative kernel ("coop_leaves.<hash>")
static constexpr uint64_t WIDE_LEVEL_NODES = 1ULL << 15;  // default: levels at least this wide run node-parallel
                                                          // ("wide_level_nodes.<hash>")

bool merkle_geometry_ok(uint64_t n_digests, uint64_t n_caps, uint64_t n_leaves, uint64_t cap_height, std::string &err)
{
    return merkle_geometry_check(n_digests, n_caps, n_leaves, cap_height, err);
}

template <int H>
static void merkle_launch(uint64_t *digests, uint64_t *caps, const uint64_t *leaves, const MerkleGeom &g, cudaStream_t s)
{
    constexpr bool COOP = HasCoop<H>::value;
    const uint32_t lg_leaves = ilog2_exact(g.n_leaves);
    const uint64_t lt = tune_get("leaf_threads." + std::to_string(H), lg_leaves, leaf_t_default<H>());
    uint64_t blocks;
    bool coop_leaf = false;
    if constexpr (COOP) coop_leaf = g.n_leaves <= tune_get("coop_leaves." + std::to_string(H), lg_leaves, COOP_LEAVES);
    uint32_t u0 = 0;
    // Poseidon2: the first LEAF_LEVELS tree levels inside the leaf kernel's
    // CTAs (measured 1.006x on Poseidon2 forests, 0.97x on Poseidon's)
    const bool fused = H == HASH_POSEIDON2 && !coop_leaf && lt == (uint64_t)LEAF_T &&
                       g.sub_leaves >= (uint64_t)LEAF_T && g.log_sub > (uint32_t)LEAF_LEVELS;
    if (fused) {
        if constexpr (H == HASH_POSEIDON2) {
            blocks = g.n_leaves / LEAF_T;
            merkle_leaf_levels_kernel<H, LEAF_T, LEAF_LEVELS><<<(unsigned)blocks, LEAF_T, 0, s>>>(leaves, digests, g);
            u0 = LEAF_LEVELS;
        }
    } else if (coop_leaf) {
        if constexpr (COOP) {
            blocks = (g.n_leaves + COOP_T / 4 - 1) / (COOP_T / 4);
            merkle_leaf_coop_kernel<H, COOP_T><<<(unsigned)blocks, COOP_T, 0, s>>>(leaves, digests, caps, g);
        }
    } else if (lt == 64) {
        blocks = (g.n_leaves + 63) / 64;
        merkle_leaf_kernel_for<H, 64>()<<<(unsigned)blocks, 64, 0, s>>>(leaves, digests, caps, g);
    } else if (lt == 128) {
        blocks = (g.n_leaves + 127) / 128;
        merkle_leaf_kernel_for<H, 128>()<<<(unsigned)blocks, 128, 0, s>>>(leaves, digests, caps, g);
    } else {
        blocks = (g.n_leaves + LEAF_T - 1) / LEAF_T;
        merkle_leaf_kernel_for<H, LEAF_T>()<<<(unsigned)blocks, LEAF_T, 0, s>>>(leaves, digests, caps, g);
    }
    note_launch();
    const uint64_t wide = tune_get("wide_level_nodes." + std::to_string(H), lg_leaves, WIDE_LEVEL_NODES);
    if (g.sub_leaves == 1) return;  // caps == leaves
    // Wide levels: one node per thread while a level still fills the GPU.
    const uint32_t top = g.log_sub - 1;
    while (u0 + 1 <= top && (g.n_leaves >> (u0 + 1)) >= wide) {
        u0++;
        const uint64_t total = g.n_leaves >> u0;
        merkle_level_kernel<H><<<(unsigned)((total + level_t<H>() - 1) / level_t<H>()), level_t<H>(), 0, s>>>(digests, g,
                                                                                                          u0);
        note_launch();
    }
    // Narrow levels: folded inside CTAs of fold_nodes nodes.
    const uint32_t fold_nodes = COOP ? COOP_T / 4 : FOLD_T;
    const uint64_t count = g.n_leaves >> u0;
    blocks = (count + fold_nodes - 1) / fold_nodes;
    if constexpr (COOP) merkle_fold_coop_kernel<H, COOP_T><<<(unsigned)blocks, COOP_T, 0, s>>>(digests, caps, g, u0);
    else merkle_fold_kernel<H, FOLD_T><<<(unsigned)blocks, FOLD_T, 0, s>>>(digests, caps, g, u0);
    note_launch();
    const uint64_t sub_nodes = g.sub_leaves >> u0;
    if (sub_nodes <= (uint64_t)fold_nodes) return;  // caps written by the fold kernel
    // heights folded by the fold kernel
    uint32_t U = 0;
    while ((1u << (U + 1)) <= fold_nodes && u0 + U + 1 <= top) U++;
    u0 += U;
    while ((g.sub_leaves >> u0) > (uint64_t)TAIL_MAXM) {
        u0++;
        uint64_t total = (g.sub_leaves >> u0) * g.n_caps;
        uint64_t nb = (total + level_t<H>() - 1) / level_t<H>();
        if (nb > 65535) nb = 65535;
        merkle_level_kernel<H><<<(unsigned)nb, level_t<H>(), 0, s>>>(digests, g, u0);
        note_launch();
    }
    if constexpr (COOP) merkle_tail_coop_kernel<H, TAIL_MAXM><<<g.n_caps, 256, 0, s>>>(digests, caps, g, u0);
    else merkle_tail_kernel<H, TAIL_MAXM><<<g.n_caps, 256, 0, s>>>(digests, caps, g, u0);
    note_launch();
}

bool merkle_device(uint64_t *digests, uint64_t *caps, const uint64_t *leaves, uint64_t n_digests, uint64_t n_caps,
                   uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height, uint64_t hash_type, cudaStream_t stream,
                   std::string &err)
{
    NvtxRange range("zeknox merkle");
    if (!merkle_geometry_ok(n_digests, n_caps, n_leaves, cap_height, err)) return false;
    if (n_caps > 0xFFFFFFFFULL) {
        err = "too many caps";
        return false;
    }
    MerkleGeom g;
    g.n_leaves = n_leaves;
    g.leaf_size = leaf_size;
    g.sub_leaves = n_leaves / n_caps;
    g.sub_digests = 2 * g.sub_leaves - 2;
    g.log_sub = ilog2_exact(g.sub_leaves);
    g.n_caps = (uint32_t)n_caps;
    switch (hash_type) {
    case HASH_POSEIDON: merkle_launch<HASH_POSEIDON>(digests, caps, leaves, g, stream); break;
    case HASH_KECCAK: merkle_launch<HASH_KECCAK>(digests, caps, leaves, g, stream); break;
    case HASH_POSEIDON_BN128: merkle_launch<HASH_POSEIDON_BN128>(digests, caps, leaves, g, stream); break;
    case HASH_POSEIDON2: merkle_launch<HASH_POSEIDON2>(digests, caps, leaves, g, stream); break;
    case HASH_MONOLITH: merkle_launch<HASH_MONOLITH>(digests, caps, leaves, g, stream); break;
    default:
        err = "unsupported hash_type " + std::to_string(hash_type);
        return false;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return false;
    }
    return true;
}

cudaError_t oob_take_merkle(uint64_t r[4]) { return oob_take_local(r); }

}  // namespace zk
