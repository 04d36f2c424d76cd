// serve_loop.cuh -- the device-resident request loop of the commit server.
//
// One cooperative, persistent kernel (every CTA resident at once) takes
// requests from a ring in mapped host memory and runs their stages itself,
// across the whole GPU: the fused LDE's passes (ntt_pass_body, every tile of
// a pass handed out to the CTAs in turn), then the Merkle forest of any of
// the five hashes (leaf hashes, node-parallel levels, the fold and the tail;
// four threads per permutation for Poseidon and Poseidon2, one for the
// others).  A grid barrier separates the stages.  The host admits requests against the arena
// budget, plans their stages (long ones split into pieces of a few
// milliseconds), copies the plan into device memory and posts the entry.
//
// Scheduling: up to LOOP_RING entries are active at once; before every stage
// the leader picks the active entry with the least estimated work left and
// runs its next stage (shortest remaining work first, preemptive at stage
// boundaries), so a small request that arrives behind a large one is not
// held up by all of it.  A finished entry is marked done in host memory; the
// kernel exits after an idle period (the host relaunches it when the next
// entry arrives).
//
// Every wait is bounded by %globaltimer: the ring poll (idle_ns: then the
// kernel exits), an entry's start gate (ready_ns: the entry fails with
// LOOP_DONE_TIMEOUT and the loop goes on) and the grid barrier (barrier_ns:
// the CTA that runs out raises `abort`, every CTA leaves, and the entry fails).
//
// Memory ordering: the host posts an entry with a release store after the
// plan's copy has completed; the leader reads `head` with ld.acquire.sys and
// every CTA acquires the barrier's generation at gpu scope before it reads the
// plan or data, so weak loads after a barrier see the stores before it.  Data
// that changes while the kernel runs (plans, leaves, digests, scratch) is
// never read through the non-coherent load path; tables (twiddles, coset
// powers) are built before a launch and never change under it.
#pragma once
#include <stdint.h>

#include "bulk.cuh"
#include "coop.cuh"
#include "hash.cuh"
#include "merkle.cuh"
#include "ntt.cuh"

namespace zk {

constexpr uint32_t LOOP_RING = 16;        // ring entries (requests posted and not yet retired)
constexpr uint32_t LOOP_MAX_STAGES = 384;  // stages (pieces) of one request
constexpr uint32_t LOOP_THREADS = 256;
constexpr uint32_t LOOP_TAIL_MAXM = 512;   // nodes a tail CTA takes (half of merkle.cu's: 24 KiB)
constexpr uint32_t LOOP_PASS_TILE = 4096;  // words of an NTT pass tile (as ntt.cu)
// shared memory of a CTA: the pass tile (32 KiB; measured 1.6% faster on a
// 2^20 x 256 request than 48 KiB for 1024-node tails: passes 57.5 against 64.1 ms)
constexpr uint32_t LOOP_SMEM_BYTES = LOOP_PASS_TILE * 8;
static_assert(LOOP_SMEM_BYTES >= (LOOP_TAIL_MAXM + LOOP_TAIL_MAXM / 2) * 32, "tail buffers");

enum LoopStageKind : uint32_t {
    LS_PASS = 1,       // one NTT pass: a.grid tiles
    LS_LEAF = 2,       // leaf digests, one leaf per thread
    LS_LEAF_COOP = 3,  // leaf digests, one leaf per group of four threads
    LS_LEVEL = 4,      // one tree level (height u), one node per thread
    LS_FOLD_COOP = 5,  // 64 nodes of height u per CTA folded upwards in shared memory
    LS_TAIL_COOP = 6,  // one subtree per CTA from height u to its cap
    LS_FOLD = 7,       // 256 nodes of height u per CTA, one permutation per thread
    LS_TAIL = 8,       // one subtree per CTA, one permutation per thread
    LS_COPY = 9,       // a.n_src words from a.src to a.dst, 4096 per CTA
    LS_REORDER = 10,   // the bit-reversal reorder of a column-output transform (fields below)
};

enum LoopDone : uint32_t { LOOP_DONE_NONE = 0, LOOP_DONE_OK = 1, LOOP_DONE_TIMEOUT = 2, LOOP_DONE_ABORT = 3 };

// LS_REORDER keeps its arguments in `a`: src, dst, src_stride, dst_stride,
// L (log2 of the transform), rate, vcols (columns), n_src (the factor), tab
// (a per-position table or null), src_len, dst_len.
struct LoopStage {
    uint32_t kind, hash;                 // LoopStageKind; hash type of Merkle stages
    uint32_t logr, load, store, u;       // LS_PASS kernel shape; Merkle height
    uint32_t inv, direct;                // LS_PASS: inverse roots; first sub-step straight from global memory
    uint64_t blocks;                     // CTA-sized work items of this piece
    uint64_t first;                      // index of its first work item
    uint64_t cost_ns;                    // estimated device time (the scheduler's measure of work)
    NttPassArgs a;                       // LS_PASS
    const uint64_t *leaves;              // Merkle stages
    uint64_t *digests, *caps;
    MerkleGeom g;
};
static_assert(sizeof(LoopStage) % 8 == 0, "stages are copied as 8-byte words");

// One ring entry (mapped host memory; the plan itself is in device memory).
struct LoopSlot {
    uint32_t ready;      // host: the entry may start (the test hook leaves it 0)
    uint32_t done;       // device: LoopDone
    uint32_t n_stages;
    uint32_t pad;
    uint64_t ready_ns;   // limit of the start-gate wait
    const LoopStage *stages;  // device memory
    // device: the device time of each stage, barrier to barrier (the
    // per-stage trace zeknox_server_trace returns)
    uint64_t t_stage[LOOP_MAX_STAGES];
};

struct LoopRing {  // mapped host memory
    uint64_t head;       // host: entries posted
    uint64_t taken;      // device: entries taken (activated, or failed at the start gate)
    uint64_t tail;       // device: entries finished (done set), in any order
    uint32_t close;      // host: exit as soon as nothing is active or posted
    uint32_t status;     // device: bit 0 an entry's gate ran out, bit 1 a barrier ran out
    uint64_t idle_ns, barrier_ns;
    uint32_t order[LOOP_RING];  // host: the slot of entry number e is order[e mod LOOP_RING]
    LoopSlot slot[LOOP_RING];
};

constexpr uint32_t LOOP_MAX_CTAS = 2048;

struct LoopActive {  // an entry being run
    uint32_t slot, cursor, n, pad;
    const LoopStage *plan;
    uint64_t remaining_ns;
};

struct LoopCtl {  // device memory, zeroed (but for taken / finished) before each launch
    unsigned arrive, gen, abort;
    int cur;                 // slot whose stage runs next; -1 exit
    uint32_t pick;           // its index in active[]
    uint32_t rank_bad;       // the CTAs are not spread evenly over SMs: ranks = block indices
    uint64_t taken, finished;
    const LoopStage *stage;  // the stage that runs next
    uint32_t n_active, pad;
    unsigned long long next_item;  // work items of the running stage handed out past the first round
    LoopActive active[LOOP_RING];
    uint32_t cta_sm[LOOP_MAX_CTAS];  // %smid of every CTA
};

__device__ __forceinline__ uint64_t ld_acquire_sys_u64(const uint64_t *p)
{
    uint64_t v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_acquire_sys_u32(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_sys_u32(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_sys_u64(uint64_t *p, uint64_t v)
{
    asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned *p) { return *(const volatile unsigned *)p; }

// Grid barrier of the cooperative launch, bounded by limit_ns; false when this
// or another CTA gave up (every CTA then leaves the loop).
__device__ __forceinline__ bool loop_grid_sync(LoopCtl *ctl, uint64_t limit_ns)
{
    __shared__ unsigned s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned ok = 1;
        const unsigned gen = ld_volatile_u32(&ctl->gen);
        __threadfence();
        if (atomicAdd(&ctl->arrive, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->arrive, 0u);
            __threadfence();
            atomicAdd(&ctl->gen, 1u);
        } else {
            // poll the generation word sparingly (every waiting CTA polls the
            // same L2 line); the abort flag and the clock every 64th poll
            const uint64_t t0 = globaltimer_ns();
            for (uint32_t it = 1; ld_volatile_u32(&ctl->gen) == gen; it++) {
                __nanosleep(512);
                if (it % 64) continue;
                if (ld_volatile_u32(&ctl->abort)) {
                    ok = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > limit_ns) {
                    atomicExch(&ctl->abort, 1u);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok && !ld_volatile_u32(&ctl->abort);
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------------- stages

// Stage bodies are separate (not inlined) functions, so each gets the
// register allocation of its own code, as its standalone kernel does, instead
// of one allocation over every stage of the loop.  A pass copies its
// arguments out of shared memory first: shared stores to the tile could
// otherwise alias them and force a reload at every use.
// Where a CTA takes its work items: its first by rank (spread over SMs),
// the rest from the stage's counter in turn (a CTA that finishes early takes
// more), as a hardware grid scheduler would.  Measured on a 2^20 x 256
// request: LDE passes 53.8 against 57.8 ms with every item by rank, wide
// levels 10.5 against 11.1 ms.  The leaf stages keep the rank stride: the
// barrier of each hand-out lines a CTA's warps up again, where by rank they
// run ahead into the next item (leaf hashes 354.0 against 352.1 ms with the
// counter, 11.38 against 10.97 ms at 2^16 x 128).
struct LoopWork {
    uint32_t rank;
    unsigned long long *next;
};

__device__ __forceinline__ uint64_t loop_grab(const LoopWork &w)
{
    __shared__ uint64_t s_b;
    __syncthreads();
    if (threadIdx.x == 0) s_b = gridDim.x + atomicAdd(w.next, 1ULL);
    __syncthreads();
    return s_b;
}

template <int LOGR, int LOADM, int STOREM>
__device__ __noinline__ void loop_pass(const NttPassArgs *pa, uint64_t first, uint64_t blocks, uint64_t *sm, LoopWork w)
{
    const NttPassArgs a = *pa;
    for (uint64_t b = w.rank; b < blocks; b = loop_grab(w)) {
        ntt_pass_body<LOGR, 0, LOOP_THREADS, LOOP_PASS_TILE, LOADM, STOREM, 1>(a, (uint32_t)(first + b), sm);
        __syncthreads();
    }
}

// Inverse column passes (the inverse transform of an evaluation-form input).
template <int LOGR, int DIRECT>
__device__ __noinline__ void loop_pass_inv(const NttPassArgs *pa, uint64_t first, uint64_t blocks, uint64_t *sm,
                                           LoopWork w)
{
    const NttPassArgs a = *pa;
    for (uint64_t b = w.rank; b < blocks; b = loop_grab(w)) {
        ntt_pass_body<LOGR, 1, LOOP_THREADS, LOOP_PASS_TILE, LOAD_PLAIN, STORE_SAME, DIRECT>(a, (uint32_t)(first + b),
                                                                                         sm);
        __syncthreads();
    }
}

__device__ __noinline__ void loop_copy(const LoopStage *pst, LoopWork w)
{
    const uint64_t *src = pst->a.src;
    uint64_t *dst = pst->a.dst;
    const uint64_t count = pst->a.n_src, first = pst->first, blocks = pst->blocks;
    for (uint64_t b = w.rank; b < blocks; b = loop_grab(w)) {
        const uint64_t base = (first + b) * (16 * LOOP_THREADS);
#pragma unroll 4
        for (uint32_t k = 0; k < 16; k++) {
            const uint64_t i = base + k * LOOP_THREADS + threadIdx.x;
            if (i < count) dst[i] = src[i];
        }
    }
}

__device__ __noinline__ void loop_reorder(const LoopStage *pst, uint64_t (*tile)[33], LoopWork w)
{
    const NttPassArgs a = pst->a;
    const uint64_t first = pst->first, blocks = pst->blocks;
    for (uint64_t b = w.rank; b < blocks; b = loop_grab(w)) {
        bitrev_reorder_body(a.src, a.dst, a.src_stride, a.dst_stride, a.L, a.rate, a.vcols, a.n_src, a.tab,
                            a.src_len, a.dst_len, first + b, tile);
        __syncthreads();
    }
}

// The pass shapes a planned fused LDE of 2^9 .. 2^22-point columns uses with
// the row-output radix 2^8, and the inverse column passes of the same sizes
// (the host rejects any other before posting).
__device__ __forceinline__ void loop_run_pass(const LoopStage &st, const NttPassArgs *a, uint64_t *sm, LoopWork w)
{
    if (st.inv) {
        if (st.direct) {
            switch (st.logr) {
            case 6: loop_pass_inv<6, 1>(a, st.first, st.blocks, sm, w); break;
            case 7: loop_pass_inv<7, 1>(a, st.first, st.blocks, sm, w); break;
            case 8: loop_pass_inv<8, 1>(a, st.first, st.blocks, sm, w); break;
            default: loop_pass_inv<9, 1>(a, st.first, st.blocks, sm, w); break;
            }
        } else {
            switch (st.logr) {
            case 6: loop_pass_inv<6, 0>(a, st.first, st.blocks, sm, w); break;
            case 7: loop_pass_inv<7, 0>(a, st.first, st.blocks, sm, w); break;
            case 8: loop_pass_inv<8, 0>(a, st.first, st.blocks, sm, w); break;
            case 9: loop_pass_inv<9, 0>(a, st.first, st.blocks, sm, w); break;
            case 10: loop_pass_inv<10, 0>(a, st.first, st.blocks, sm, w); break;
            case 11: loop_pass_inv<11, 0>(a, st.first, st.blocks, sm, w); break;
            default: loop_pass_inv<12, 0>(a, st.first, st.blocks, sm, w); break;
            }
        }
        return;
    }
    if (st.load == LOAD_COSETS && st.store == STORE_SAME) {
        switch (st.logr) {
        case 1: loop_pass<1, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 2: loop_pass<2, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 3: loop_pass<3, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 4: loop_pass<4, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 5: loop_pass<5, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 6: loop_pass<6, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 7: loop_pass<7, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 8: loop_pass<8, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 9: loop_pass<9, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        default: loop_pass<10, LOAD_COSETS, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        }
    } else if (st.store == STORE_SAME) {
        switch (st.logr) {
        case 5: loop_pass<5, LOAD_PLAIN, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        case 6: loop_pass<6, LOAD_PLAIN, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        default: loop_pass<7, LOAD_PLAIN, STORE_SAME>(a, st.first, st.blocks, sm, w); break;
        }
    } else {
        loop_pass<8, LOAD_PLAIN, STORE_ROWS>(a, st.first, st.blocks, sm, w);
    }
}

template <int H>
__device__ __noinline__ void loop_leaf(const LoopStage *pst, LoopWork w)
{
    // only the loop bounds and the row address stay live across the
    // permutation; the destination's geometry is read again from shared
    // memory after it (fewer registers held: 0.8% faster leaf stage)
    const uint64_t blocks = pst->blocks, first = pst->first;
    const uint64_t n_leaves = pst->g.n_leaves, leaf_size = pst->g.leaf_size;
    const uint64_t *leaves = pst->leaves;
    for (uint64_t b = w.rank; b < blocks; b += gridDim.x) {
        const uint64_t i = (first + b) * LOOP_THREADS + threadIdx.x;
        if (i >= n_leaves) continue;
        uint64_t d[4];
        if (H == HASH_KECCAK && leaf_size < 4) {
            const MerkleGeom g = pst->g;
            uint64_t *dst = g.sub_leaves == 1 ? pst->caps + 4 * i : pst->digests + 4 * merkle_node_index(g, i, 0);
#pragma unroll
            for (int q = 0; q < 4; q++) d[q] = dst[q];
        }
        leaf_hash<H>(leaves + i * leaf_size, leaf_size, d);
        const volatile LoopStage *v = pst;
        const uint64_t sub_leaves = v->g.sub_leaves;
        uint64_t *dst;
        if (sub_leaves == 1) {
            dst = v->caps + 4 * i;
        } else {
            const uint32_t log_sub = v->g.log_sub;
            const uint64_t k = i >> log_sub, in_sub = i & (sub_leaves - 1);
            dst = v->digests + 4 * (k * v->g.sub_digests + (sub_leaves - 2) + in_sub);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) dst[q] = d[q];
    }
}

template <int H>
__device__ __noinline__ void loop_leaf_coop(const LoopStage *pst, LoopWork w)
{
    const LoopStage st = *pst;
    const MerkleGeom &g = st.g;
    CoopGroup c;
    c.init();
    for (uint64_t b = w.rank; b < st.blocks; b += gridDim.x) {
        const uint64_t gi = ((st.first + b) * LOOP_THREADS + threadIdx.x) >> 2;
        if ((gi & ~7ULL) >= g.n_leaves) continue;  // the whole warp is past the end
        const uint64_t i = gi < g.n_leaves ? gi : g.n_leaves - 1;
        uint64_t d[4];
        sponge_hash_one_coop<H>(st.leaves + i * g.leaf_size, g.leaf_size, d, c);
        if (c.q == 0 && gi < g.n_leaves) {
            uint64_t *dst = g.sub_leaves == 1 ? st.caps + 4 * gi : st.digests + 4 * merkle_node_index(g, gi, 0);
#pragma unroll
            for (int q = 0; q < 4; q++) dst[q] = d[q];
        }
    }
}

template <int H>
__device__ __noinline__ void loop_level(const LoopStage *pst, LoopWork w)
{
    const LoopStage st = *pst;
    const MerkleGeom &g = st.g;
    const uint64_t per_sub = g.sub_leaves >> st.u, total = per_sub * g.n_caps;
    for (uint64_t b = w.rank; b < st.blocks; b = loop_grab(w)) {
        const uint64_t x = (st.first + b) * LOOP_THREADS + threadIdx.x;
        if (x >= total) continue;
        const uint64_t k = x / per_sub, j = x % per_sub;
        uint64_t *sub = st.digests + k * g.sub_digests * 4;
        const uint64_t start = per_sub - 2, child = 2 * per_sub - 2;
        uint64_t h[4];
        hash_two<H>(sub + 4 * (child + 2 * j), sub + 4 * (child + 2 * j + 1), h);
#pragma unroll
        for (int q = 0; q < 4; q++) sub[4 * (start + j) + q] = h[q];
    }
}

// 64 consecutive nodes of height u per work item, folded upwards inside the
// CTA (the cooperative fold of merkle.cuh, with the caps of whole subtrees).
template <int H>
__device__ __noinline__ void loop_fold_coop(const LoopStage *pst, uint64_t (*node)[4], LoopWork w)
{
    const LoopStage st = *pst;
    constexpr uint32_t NG = LOOP_THREADS / 4;
    const MerkleGeom &g = st.g;
    const uint32_t u0 = st.u;
    CoopGroup c;
    c.init();
    const uint32_t grp = threadIdx.x >> 2;
    const uint32_t wg = grp & ~7u;
    const uint64_t count = g.n_leaves >> u0;
    const uint32_t top = g.log_sub - 1;
    uint32_t U = 0;
    while ((1u << (U + 1)) <= NG && u0 + U + 1 <= top) U++;
    for (uint64_t b = w.rank; b < st.blocks; b = loop_grab(w)) {
        const uint64_t i0 = (st.first + b) * NG;
        const uint64_t cta_nodes = count - i0 < (uint64_t)NG ? count - i0 : (uint64_t)NG;
        for (uint32_t t = threadIdx.x; t < 4 * cta_nodes; t += LOOP_THREADS)
            node[t >> 2][t & 3] = st.digests[4 * merkle_node_index(g, (i0 + (t >> 2)) << u0, u0) + (t & 3)];
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
#pragma unroll
                    for (int q = 0; q < 4; q++) st.digests[4 * di + q] = h[q];
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
#pragma unroll
                    for (int q = 0; q < 4; q++) st.caps[4 * k + q] = h[q];
                }
            }
        }
        __syncthreads();
    }
}

// One subtree per work item, from height u to its cap (the cooperative tail
// of merkle.cuh).
template <int H>
__device__ __noinline__ void loop_tail_coop(const LoopStage *pst, uint64_t (*bufa)[4], uint64_t (*bufb)[4], LoopWork w)
{
    const LoopStage st = *pst;
    constexpr uint32_t NG = LOOP_THREADS / 4;
    const MerkleGeom &g = st.g;
    CoopGroup c;
    c.init();
    const uint32_t grp = threadIdx.x >> 2;
    for (uint64_t kb = w.rank; kb < st.blocks; kb = loop_grab(w)) {
        const uint64_t k = st.first + kb;
        uint64_t *sub = st.digests + k * g.sub_digests * 4;
        uint32_t m = (uint32_t)(g.sub_leaves >> st.u);
        for (uint32_t j = threadIdx.x; j < 4 * m; j += LOOP_THREADS) bufa[j >> 2][j & 3] = sub[4 * (m - 2) + j];
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
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        sub[4 * (half - 2 + j) + q] = h[q];
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
            if (threadIdx.x == 0) {
#pragma unroll
                for (int q = 0; q < 4; q++) st.caps[4 * k + q] = h[q];
            }
        }
        __syncthreads();
    }
}

// 256 consecutive nodes of height u per work item, one permutation per
// thread (merkle.cuh's merkle_fold_kernel: the hashes without a cooperative
// form).
template <int H>
__device__ __noinline__ void loop_fold(const LoopStage *pst, uint64_t (*node)[4], LoopWork w)
{
    constexpr uint32_t T = LOOP_THREADS;
    const LoopStage st = *pst;
    const MerkleGeom &g = st.g;
    const uint32_t u0 = st.u, t = threadIdx.x;
    const uint64_t count = g.n_leaves >> u0;
    const uint32_t top = g.log_sub - 1;
    uint32_t U = 0;
    while ((1u << (U + 1)) <= T && u0 + U + 1 <= top) U++;
    for (uint64_t b = w.rank; b < st.blocks; b = loop_grab(w)) {
        const uint64_t i0 = (st.first + b) * T;
        const uint64_t cta_nodes = count - i0 < (uint64_t)T ? count - i0 : (uint64_t)T;
        if (t < cta_nodes) {
            const uint64_t di = merkle_node_index(g, (i0 + t) << u0, u0);
#pragma unroll
            for (int q = 0; q < 4; q++) node[t][q] = st.digests[4 * di + q];
        }
        for (uint32_t v = 1; v <= U; v++) {
            __syncthreads();
            const uint32_t nodes = T >> v;
            uint64_t h[4];
            const bool act = t < nodes && ((uint64_t)t << v) < cta_nodes;
            if (act) {
                hash_two<H>(node[2 * t], node[2 * t + 1], h);
                const uint64_t di = merkle_node_index(g, (i0 + ((uint64_t)t << v)) << u0, u0 + v);
#pragma unroll
                for (int q = 0; q < 4; q++) st.digests[4 * di + q] = h[q];
            }
            __syncthreads();
            if (act) {
#pragma unroll
                for (int q = 0; q < 4; q++) node[t][q] = h[q];
            }
        }
        const uint64_t sub_nodes = g.sub_leaves >> u0;
        if (u0 + U == top && sub_nodes <= (uint64_t)T) {
            __syncthreads();
            const uint32_t subs = (uint32_t)(cta_nodes / sub_nodes);
            if (t < subs) {
                uint64_t h[4];
                hash_two<H>(node[2 * t], node[2 * t + 1], h);
                const uint64_t k = ((i0 << u0) >> g.log_sub) + t;
#pragma unroll
                for (int q = 0; q < 4; q++) st.caps[4 * k + q] = h[q];
            }
        }
        __syncthreads();
    }
}

// One subtree per work item from height u to its cap, one permutation per
// thread (merkle.cuh's merkle_tail_kernel).
template <int H>
__device__ __noinline__ void loop_tail(const LoopStage *pst, uint64_t (*bufa)[4], uint64_t (*bufb)[4], LoopWork w)
{
    const LoopStage st = *pst;
    const MerkleGeom &g = st.g;
    for (uint64_t kb = w.rank; kb < st.blocks; kb = loop_grab(w)) {
        const uint64_t k = st.first + kb;
        uint64_t *sub = st.digests + k * g.sub_digests * 4;
        uint32_t m = (uint32_t)(g.sub_leaves >> st.u);
        for (uint32_t j = threadIdx.x; j < m; j += LOOP_THREADS) {
#pragma unroll
            for (int q = 0; q < 4; q++) bufa[j][q] = sub[4 * (m - 2 + j) + q];
        }
        uint64_t(*src)[4] = bufa;
        uint64_t(*dst)[4] = bufb;
        while (m > 2) {
            __syncthreads();
            const uint32_t half = m / 2;
            for (uint32_t j = threadIdx.x; j < half; j += LOOP_THREADS) {
                uint64_t h[4];
                hash_two<H>(src[2 * j], src[2 * j + 1], h);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    sub[4 * (half - 2 + j) + q] = h[q];
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
#pragma unroll
            for (int q = 0; q < 4; q++) st.caps[4 * k + q] = h[q];
        }
        __syncthreads();
    }
}

template <int H>
__device__ __forceinline__ void loop_run_merkle(const LoopStage &st, uint64_t *sm, LoopWork w)
{
    switch (st.kind) {
    case LS_LEAF: loop_leaf<H>(&st, w); break;
    case LS_LEVEL: loop_level<H>(&st, w); break;
    case LS_FOLD: loop_fold<H>(&st, (uint64_t(*)[4])sm, w); break;
    case LS_TAIL: loop_tail<H>(&st, (uint64_t(*)[4])sm, (uint64_t(*)[4])(sm + 4 * LOOP_TAIL_MAXM), w); break;
    default:
        if constexpr (HasCoop<H>::value) {
            if (st.kind == LS_LEAF_COOP) loop_leaf_coop<H>(&st, w);
            else if (st.kind == LS_FOLD_COOP) loop_fold_coop<H>(&st, (uint64_t(*)[4])sm, w);
            else loop_tail_coop<H>(&st, (uint64_t(*)[4])sm, (uint64_t(*)[4])(sm + 4 * LOOP_TAIL_MAXM), w);
        }
        break;
    }
}

// A CTA's rank: work item b of a stage goes to the CTA of rank b mod the
// grid.  The cooperative grid places consecutive block indices on the same
// SM, so a stage with fewer items than CTAs would crowd onto a few SMs;
// ranked as (its place among the CTAs of its SM) x (SMs) + (its SM's place
// among the SMs), the first items land on distinct SMs.  When the CTAs are not
// spread evenly over SMs the ranks fall back to the block indices.
__device__ uint32_t loop_rank(LoopCtl *ctl, uint64_t barrier_ns)
{
    __shared__ uint32_t s_sm_bits[8], s_slot, s_rank;
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if (threadIdx.x < 8) s_sm_bits[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        s_slot = 0;
        if (blockIdx.x < LOOP_MAX_CTAS) ctl->cta_sm[blockIdx.x] = smid;
        if (smid >= 256 || gridDim.x > LOOP_MAX_CTAS) atomicExch(&ctl->rank_bad, 1u);
    }
    if (!loop_grid_sync(ctl, barrier_ns)) return blockIdx.x;
    if (gridDim.x > LOOP_MAX_CTAS) return blockIdx.x;  // ranks = block indices (rank_bad is set)
    for (uint32_t j = threadIdx.x; j < gridDim.x; j += LOOP_THREADS) {
        const uint32_t sm_j = *(volatile uint32_t *)&ctl->cta_sm[j];
        if (sm_j < 256) atomicOr(&s_sm_bits[sm_j >> 5], 1u << (sm_j & 31));
        if (j < blockIdx.x && sm_j == smid) atomicAdd(&s_slot, 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t n_sm = 0, below = 0;
        for (int w = 0; w < 8; w++) {
            n_sm += __popc(s_sm_bits[w]);
            if (smid < 256) {
                const uint32_t lim = smid >> 5;
                if ((uint32_t)w < lim) below += __popc(s_sm_bits[w]);
                else if ((uint32_t)w == lim) below += __popc(s_sm_bits[w] & ((1u << (smid & 31)) - 1));
            }
        }
        const uint32_t per_sm = n_sm ? gridDim.x / n_sm : 0;
        if (!n_sm || per_sm * n_sm != gridDim.x || s_slot >= per_sm) atomicExch(&ctl->rank_bad, 1u);
        s_rank = s_slot * n_sm + below;
    }
    if (!loop_grid_sync(ctl, barrier_ns)) return blockIdx.x;
    return ld_volatile_u32(&ctl->rank_bad) ? blockIdx.x : s_rank;
}

// The loop.  Launched cooperatively with LOOP_THREADS threads and
// LOOP_SMEM_BYTES of dynamic shared memory per CTA.
#ifndef ZK_LOOP_MIN_CTAS
#define ZK_LOOP_MIN_CTAS 4  // CTAs of the loop per SM (64 registers a thread)
#endif
__global__ void __launch_bounds__(LOOP_THREADS, ZK_LOOP_MIN_CTAS) serve_loop_kernel(LoopRing *ring, LoopCtl *ctl)
{
    extern __shared__ __align__(16) uint64_t loop_sm[];
    __shared__ LoopStage s_stage;
    __shared__ int s_cur;
    __shared__ const LoopStage *s_next;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    const uint64_t barrier_ns = ring->barrier_ns;
    const uint32_t rank = loop_rank(ctl, barrier_ns);
    const LoopWork w{rank, &ctl->next_item};
    for (;;) {
        if (leader) {
            // take posted entries (waiting, bounded, only when nothing is active)
            const uint64_t t0 = globaltimer_ns();
            for (;;) {
                const uint64_t head = ld_acquire_sys_u64(&ring->head);
                while (ctl->taken < head && ctl->n_active < LOOP_RING) {
                    const uint32_t k = *(volatile uint32_t *)&ring->order[ctl->taken % LOOP_RING] % LOOP_RING;
                    LoopSlot *sl = &ring->slot[k];
                    const uint64_t t1 = globaltimer_ns();
                    bool ready = false;
                    for (;;) {
                        if (ld_acquire_sys_u32(&sl->ready)) {
                            ready = true;
                            break;
                        }
                        if (globaltimer_ns() - t1 > sl->ready_ns) break;
                        __nanosleep(1000);
                    }
                    if (ready) {
                        LoopActive &e = ctl->active[ctl->n_active++];
                        e.slot = k;
                        e.cursor = 0;
                        const uint32_t n = *(volatile uint32_t *)&sl->n_stages;
                        e.n = n < LOOP_MAX_STAGES ? n : LOOP_MAX_STAGES;
                        e.plan = *(const LoopStage *const volatile *)&sl->stages;
                        uint64_t rem = 0;
                        for (uint32_t q = 0; q < e.n; q++) rem += *(const volatile uint64_t *)&e.plan[q].cost_ns;
                        e.remaining_ns = rem;
                    } else {
                        // only the leader writes status: no atomics on host memory
                        st_release_sys_u32(&ring->status, *(volatile uint32_t *)&ring->status | 1u);
                        st_release_sys_u32(&sl->done, LOOP_DONE_TIMEOUT);
                        st_release_sys_u64(&ring->tail, ++ctl->finished);
                    }
                    st_release_sys_u64(&ring->taken, ++ctl->taken);
                }
                if (ctl->n_active) break;
                if (ld_acquire_sys_u32(&ring->close) || globaltimer_ns() - t0 > ring->idle_ns) break;
                __nanosleep(1000);
            }
            // the active entry with the least estimated work left runs its next stage
            int cur = -1;
            if (ctl->n_active) {
                uint32_t best = 0;
                for (uint32_t q = 1; q < ctl->n_active; q++)
                    if (ctl->active[q].remaining_ns < ctl->active[best].remaining_ns) best = q;
                const LoopActive &e = ctl->active[best];
                ctl->pick = best;
                ctl->stage = e.plan + e.cursor;
                ctl->next_item = 0;
                cur = (int)e.slot;
            }
            ctl->cur = cur;
        }
        if (!loop_grid_sync(ctl, barrier_ns)) break;
        if (threadIdx.x == 0) {
            s_cur = *(volatile int *)&ctl->cur;
            s_next = *(const LoopStage *const volatile *)&ctl->stage;
        }
        __syncthreads();
        if (s_cur < 0) break;
        const uint64_t t_begin = leader ? globaltimer_ns() : 0;
        // the stage description into shared memory (volatile loads: the plan
        // buffers are rewritten between requests)
        for (uint32_t w = threadIdx.x; w < sizeof(LoopStage) / 8; w += LOOP_THREADS)
            ((uint64_t *)&s_stage)[w] = ((const volatile uint64_t *)s_next)[w];
        __syncthreads();
        const LoopStage &st = s_stage;
        if (st.kind == LS_PASS) loop_run_pass(st, &st.a, loop_sm, w);
        else if (st.kind == LS_COPY) loop_copy(&st, w);
        else if (st.kind == LS_REORDER) loop_reorder(&st, (uint64_t(*)[33])loop_sm, w);
        else if (st.hash == HASH_POSEIDON2) loop_run_merkle<HASH_POSEIDON2>(st, loop_sm, w);
        else if (st.hash == HASH_KECCAK) loop_run_merkle<HASH_KECCAK>(st, loop_sm, w);
        else if (st.hash == HASH_MONOLITH) loop_run_merkle<HASH_MONOLITH>(st, loop_sm, w);
        else if (st.hash == HASH_POSEIDON_BN128) loop_run_merkle<HASH_POSEIDON_BN128>(st, loop_sm, w);
        else loop_run_merkle<HASH_POSEIDON>(st, loop_sm, w);
        const bool ok = loop_grid_sync(ctl, barrier_ns);
        if (leader) {
            LoopActive &e = ctl->active[ctl->pick];
            LoopSlot *sl = &ring->slot[e.slot];
            *(volatile uint64_t *)&sl->t_stage[e.cursor] = globaltimer_ns() - t_begin;
            e.remaining_ns = e.remaining_ns > st.cost_ns ? e.remaining_ns - st.cost_ns : 0;
            e.cursor++;
            if (!ok) {
                // every active entry fails: the loop leaves
                st_release_sys_u32(&ring->status, *(volatile uint32_t *)&ring->status | 2u);
                __threadfence_system();
                for (uint32_t q = 0; q < ctl->n_active; q++) {
                    st_release_sys_u32(&ring->slot[ctl->active[q].slot].done, LOOP_DONE_ABORT);
                    ++ctl->finished;
                }
                ctl->n_active = 0;
                st_release_sys_u64(&ring->tail, ctl->finished);
            } else if (e.cursor >= e.n) {
                __threadfence_system();
                st_release_sys_u32(&sl->done, LOOP_DONE_OK);
                st_release_sys_u64(&ring->tail, ++ctl->finished);
                ctl->active[ctl->pick] = ctl->active[--ctl->n_active];
            }
        }
        if (!ok) break;
    }
}

}  // namespace zk
