// serve.cu -- continuous-batching commit server (include/zeknox_b200.h).
//
// Host side: any thread submits requests into a FIFO; one server thread per
// server admits the head of the queue whenever a slot stream is idle and the
// job's device memory fits, enqueues the whole commit (LDE, Merkle, caps
// copy-out) on that slot's stream, and polls the slot events to retire
// finished jobs.  While the head waits for memory (not for a slot), small
// requests behind it (at most 1/8 of the budget each) that fit now may start
// ahead of it, at most `slots` of them per waiting head: a large request then
// holds up no small one, and waits for at most `slots` small ones itself.
//
// Memory: the budget is one device allocation made when the server is
// created (an arena), and every job takes one contiguous range of it
// (first fit, freed ranges merged with their neighbours).  Jobs therefore
// never call the driver's allocator, and a job the budget admits always has
// the memory: per-job stream-ordered allocations of multi-GB buffers measured
// out-of-memory failures and long allocation stalls at this size mix.
//
// Device side: jobs on different slots overlap; twiddle, coset and
// round-constant tables stay resident in the device context across requests
// (zeknox_server_prepare builds them ahead of the stream).
//
// Device-loop mode (zeknox_server_create_ex with ZK_SERVE_DEVICE_LOOP): the
// same admission, but an admitted job is not launched from the host.  Its
// stages are planned on the host, copied to device memory and posted to a
// ring in mapped host memory, and a persistent cooperative kernel
// (serve_loop.cuh) runs them, one request at a time across the whole GPU.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

// the loop kernel's Poseidon-BN128 matrix layers as five reductions per dot
// product (the register budget the loop's stages share; hash.cuh)
#define ZK_BN128_DOT_ONE_REDUCTION 0
#include "../../include/zeknox_b200.h"
#include "batch.cuh"
#include "ntt_api.cuh"
#include "runtime.cuh"
#include "serve_loop.cuh"
#include "zk_constants.h"

namespace zk {
namespace {

using Clock = std::chrono::steady_clock;

constexpr uint64_t ARENA_ALIGN = 256;
constexpr uint64_t NO_RANGE = ~0ULL;

uint64_t align_up(uint64_t x) { return (x + ARENA_ALIGN - 1) / ARENA_ALIGN * ARENA_ALIGN; }

// First-fit allocator over the byte offsets of the arena.
struct RangeAlloc {
    std::map<uint64_t, uint64_t> free_;  // offset -> size
    void init(uint64_t size)
    {
        free_.clear();
        if (size) free_[0] = size;
    }
    uint64_t take(uint64_t size)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < size) continue;
            const uint64_t off = it->first, rest = it->second - size;
            free_.erase(it);
            if (rest) free_[off + size] = rest;
            return off;
        }
        return NO_RANGE;
    }
    bool fits(uint64_t size) const
    {
        for (const auto &kv : free_)
            if (kv.second >= size) return true;
        return false;
    }
    void give(uint64_t off, uint64_t size)
    {
        auto it = free_.emplace(off, size).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Ticket {
    zk_serve_request req;
    Clock::time_point t_submit, t_admit, t_done;
    int status = 0;  // 0 queued, 1 running, 2 done, < 0 failed or cancelled
    int slot = -1;
    uint64_t bytes = 0;        // arena bytes of the job (aligned pieces)
    uint64_t off = NO_RANGE;   // its range in the arena while admitted
    uint64_t *leaves = nullptr, *digests = nullptr, *caps = nullptr, *scratch = nullptr;
    cudaEvent_t done_ev = nullptr;
    // device-loop mode: each stage's kind and its duration on the device
    std::vector<uint32_t> trace_kind;
    std::vector<uint64_t> trace_ns;
};

struct Server {
    DeviceCtx *ctx = nullptr;
    uint64_t budget = 0, in_use = 0, peak = 0, completed = 0;
    uint8_t *arena = nullptr;
    RangeAlloc ranges;
    std::vector<cudaStream_t> slot_stream;
    std::vector<uint64_t> slot_ticket;  // 0 = idle
    cudaEvent_t tables_ready = nullptr; // recorded on the context stream after a start's table builds
    std::mutex mu;
    std::condition_variable cv;  // signalled on submit, completion, release, stop
    std::deque<uint64_t> queue;
    std::map<uint64_t, Ticket> tickets;
    uint64_t next_id = 1;
    uint64_t blocked_head = 0;  // head of the queue that waits for memory
    uint32_t bypassed = 0;      // small requests started ahead of it
    int inject_next = 0;        // test hook: the next start fails at this stage (ZK_SERVE_FAIL_*)
    bool stop = false;
    std::thread worker;

    // device-loop mode
    bool device_loop = false;
    LoopRing *ring = nullptr, *ring_dev = nullptr;  // mapped host memory, and its device address
    LoopCtl *ctl = nullptr;                         // device
    LoopStage *plans = nullptr;                     // device: LOOP_RING x LOOP_MAX_STAGES
    LoopStage *plans_host = nullptr;                // pinned staging of the same shape
    cudaStream_t loop_stream = nullptr, copy_stream = nullptr;
    cudaEvent_t loop_exit = nullptr;
    bool loop_live = false;
    int loop_grid = 0;
    uint64_t posted = 0, retired = 0;               // ring entries posted / retired by this host
    uint64_t ring_ticket[LOOP_RING] = {};           // ticket of each slot (0: free)
    uint64_t ring_seq[LOOP_RING] = {};              // entry number posted in each slot
    uint32_t loop_depth = 1;                        // entries in flight at most

    // Arena bytes of a job: leaves, digests, caps and LDE scratch, each
    // starting on an ARENA_ALIGN boundary.
    static uint64_t job_bytes(const zk_serve_request &r)
    {
        const uint64_t N = 1ULL << (r.lg_n + r.rate_bits);
        const uint64_t caps = 1ULL << r.cap_height;
        return align_up(8 * N * r.cols) + align_up(64 * (N - caps)) + align_up(32 * caps) +
               align_up(8 * commit_scratch_words(r.lg_n, r.rate_bits, r.cols, r.input_is_values != 0));
    }

    void place(Ticket &t)
    {
        const zk_serve_request &r = t.req;
        const uint64_t N = 1ULL << (r.lg_n + r.rate_bits);
        const uint64_t n_caps = 1ULL << r.cap_height;
        const uint64_t sw = commit_scratch_words(r.lg_n, r.rate_bits, r.cols, r.input_is_values != 0);
        uint8_t *p = arena + t.off;
        t.leaves = (uint64_t *)p;
        p += align_up(8 * N * r.cols);
        t.digests = N > n_caps ? (uint64_t *)p : nullptr;
        p += align_up(64 * (N - n_caps));
        t.caps = (uint64_t *)p;
        p += align_up(32 * n_caps);
        t.scratch = sw ? (uint64_t *)p : nullptr;
    }

    // Give an admitted job's range back (caller holds mu; nothing on the GPU
    // may still use it).
    void unadmit(Ticket &t)
    {
        if (t.off != NO_RANGE) {
            ranges.give(t.off, t.bytes);
            in_use -= t.bytes;
            t.off = NO_RANGE;
        }
        t.leaves = t.digests = t.caps = t.scratch = nullptr;
    }

    // Queue an admitted job's whole commit on its slot stream.  Runs on the
    // server thread without `mu` (client threads keep submitting, waiting and
    // releasing meanwhile): a starting ticket can be neither released nor
    // cancelled, and only this thread starts jobs.  Returns 1 when the work is
    // queued, else a negative status (the slot stream has then finished
    // whatever this start queued, so the range may be reused at once).
    int start(Ticket &t, int slot, int inject)
    {
        const zk_serve_request &r = t.req;
        cudaStream_t s = slot_stream[slot];
        const uint64_t n_caps = 1ULL << r.cap_height;
        NvtxRange range("zeknox serve start");
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        try {
            zk_commit_job j{};
            j.lg_n = r.lg_n;
            j.rate_bits = r.rate_bits;
            j.cols = r.cols;
            j.cap_height = r.cap_height;
            j.hash_type = r.hash_type;
            j.input_is_values = r.input_is_values;
            j.coset_gen = r.coset_gen;
            j.input = r.input;
            j.leaves = t.leaves;
            j.digests = t.digests;
            j.caps = t.caps;
            if (inject == ZK_SERVE_FAIL_SHAPE) j.cap_height = j.lg_n + j.rate_bits + 1;  // a shape that cannot commit
            if (inject == ZK_SERVE_FAIL_ALLOC)
                throw cuda_failure(-(int)cudaErrorMemoryAllocation, "device allocation refused (injected)");
            check_job(j);
            // tables this shape reads that are not resident yet are built on
            // the context stream; the slot stream waits for them on the
            // device, not the server thread on the host
            prepare_job(*ctx, j);
            ZK_CUDA(cudaEventRecord(tables_ready, ctx->stream));
            ZK_CUDA(cudaStreamWaitEvent(s, tables_ready, 0));
            if (inject == ZK_SERVE_FAIL_LAUNCH)
                throw cuda_failure(-(int)cudaErrorLaunchFailure, "kernel launch refused (injected)");
            commit_enqueue(*ctx, j, s, t.scratch);
            if (r.caps_host) ZK_CUDA(cudaMemcpyAsync(r.caps_host, t.caps, n_caps * 32, cudaMemcpyDeviceToHost, s));
            ZK_CUDA(cudaEventCreateWithFlags(&t.done_ev, cudaEventDisableTiming));
            ZK_CUDA(cudaEventRecord(t.done_ev, s));
            return 1;
        } catch (const std::exception &e) {
            const cuda_failure *cf = dynamic_cast<const cuda_failure *>(&e);
            const arg_failure *af = dynamic_cast<const arg_failure *>(&e);
            (void)cudaStreamSynchronize(s);  // whatever was queued finishes before the range is reused
            (void)cudaGetLastError();
            if (t.done_ev) {
                cudaEventDestroy(t.done_ev);
                t.done_ev = nullptr;
            }
            return cf ? (cf->code < 0 ? cf->code : -1) : af ? -af->code : -1;
        }
    }

    // ---------------------------------------------------- device-loop mode

    // The loop kernel is running (it exits after an idle period).
    bool loop_running()
    {
        if (!loop_live) return false;
        const cudaError_t q = cudaEventQuery(loop_exit);
        if (q == cudaErrorNotReady) return true;
        loop_live = false;
        if (q != cudaSuccess) (void)cudaGetLastError();
        return false;
    }

    // Launch the loop if entries wait and it is not running.
    void loop_ensure()
    {
        if (loop_running()) return;
        const uint64_t taken = __atomic_load_n(&ring->taken, __ATOMIC_ACQUIRE);
        if (taken >= posted) return;
        LoopCtl init{};
        init.taken = taken;
        init.finished = __atomic_load_n(&ring->tail, __ATOMIC_ACQUIRE);
        ZK_CUDA(cudaMemcpyAsync(ctl, &init, sizeof init, cudaMemcpyHostToDevice, loop_stream));
        void *args[] = {(void *)&ring_dev, (void *)&ctl};
        ZK_CUDA(cudaLaunchCooperativeKernel((const void *)serve_loop_kernel, dim3(loop_grid), dim3(LOOP_THREADS), args,
                                            LOOP_SMEM_BYTES, loop_stream));
        note_launch();
        ZK_CUDA(cudaEventRecord(loop_exit, loop_stream));
        loop_live = true;
    }

    // Let the loop finish what is posted and exit (so kernels on other streams
    // get the SMs: table builds).
    void loop_stop()
    {
        if (!loop_running()) return;
        __atomic_store_n(&ring->close, 1u, __ATOMIC_RELEASE);
        (void)cudaEventSynchronize(loop_exit);
        __atomic_store_n(&ring->close, 0u, __ATOMIC_RELEASE);
        loop_live = false;
    }

    // Stages of the forest, as merkle.cu launches them (for Poseidon and
    // Poseidon2 cooperative leaves up to coop_leaves; node-parallel wide
    // levels; the fold; levels beyond the tail's capacity; the tail; the fold
    // and tail cooperative for Poseidon and Poseidon2); every stage gives the
    // same digests as its kernel.
    // Device time estimates of the scheduler (only their ratios matter): one
    // width-12 permutation and one LDE element of the whole GPU's throughput.
    static constexpr double PERM_NS = 1.27, LDE_ELEM_NS = 0.016;
    static constexpr uint64_t PIECE_NS = 4000000;  // stages longer than this are split
    static constexpr uint64_t MAX_PIECES = 64;     // into at most this many pieces

    // Append a stage, split into pieces of whole multiples of the loop's grid
    // when it is estimated above PIECE_NS, so the scheduler can switch entries
    // between the pieces.
    static void push_split(std::vector<LoopStage> &out, LoopStage st, double ns_per_block, uint64_t grid)
    {
        const uint64_t total = st.blocks;
        st.cost_ns = (uint64_t)(ns_per_block * (double)total);
        uint64_t piece = total;
        if (st.cost_ns > PIECE_NS && grid) {
            const double piece_ns = std::max((double)PIECE_NS, (double)st.cost_ns / MAX_PIECES);
            piece = (uint64_t)(piece_ns / ns_per_block + grid - 1) / grid * grid;
            if (piece < grid) piece = grid;
        }
        for (uint64_t f = 0; f < total; f += piece) {
            LoopStage p = st;
            p.first = f;
            p.blocks = total - f < piece ? total - f : piece;
            p.cost_ns = (uint64_t)(ns_per_block * (double)p.blocks);
            out.push_back(p);
        }
    }

    // Device time of one permutation at the whole GPU's throughput, per hash
    // (measured forests of 2^20 x 135 leaves: Poseidon 788, Keccak 3300,
    // Poseidon-BN128 35, Poseidon2 1190, Monolith 2060 M/s).
    static double perm_ns(uint32_t hash)
    {
        switch (hash) {
        case HASH_KECCAK: return 0.30;
        case HASH_POSEIDON_BN128: return 28.6;
        case HASH_POSEIDON2: return 0.84;
        case HASH_MONOLITH: return 0.49;
        default: return 1.27;
        }
    }

    static void merkle_stages(std::vector<LoopStage> &out, uint64_t *digests, uint64_t *caps, const uint64_t *leaves,
                              uint64_t n_leaves, uint64_t leaf_size, uint32_t cap_height, uint32_t hash, uint64_t grid)
    {
        MerkleGeom g{};
        g.n_leaves = n_leaves;
        g.leaf_size = leaf_size;
        g.n_caps = 1u << cap_height;
        g.sub_leaves = n_leaves >> cap_height;
        g.sub_digests = 2 * g.sub_leaves - 2;
        g.log_sub = ilog2_exact(g.sub_leaves);
        const bool coop = hash == HASH_POSEIDON || hash == HASH_POSEIDON2;
        const double leaf_perms = hash == HASH_KECCAK ? (double)(leaf_size * 8 / 136 + 1)
                                  : leaf_size > 4    ? (double)((leaf_size + 7) / 8)
                                                     : 0.0;
        const double pns = perm_ns(hash);
        auto stage = [&](uint32_t kind, uint32_t u, uint64_t blocks) {
            LoopStage st{};
            st.kind = kind;
            st.hash = hash;
            st.u = u;
            st.blocks = blocks;
            st.leaves = leaves;
            st.digests = digests;
            st.caps = caps;
            st.g = g;
            // permutations per work item: a leaf CTA hashes 256 leaves (64 in
            // the cooperative form), a level CTA 256 nodes, a fold CTA 64 nodes
            // and the levels above them, a tail CTA one subtree
            double per = 0;
            switch (kind) {
            case LS_LEAF: per = LOOP_THREADS * leaf_perms; break;
            case LS_LEAF_COOP: per = LOOP_THREADS / 4 * leaf_perms; break;
            case LS_LEVEL: per = LOOP_THREADS; break;
            case LS_FOLD_COOP: per = 2.0 * LOOP_THREADS / 4; break;
            case LS_FOLD: per = 2.0 * LOOP_THREADS; break;
            default: per = 2.0 * (double)(g.sub_leaves >> u); break;
            }
            push_split(out, st, per * pns, grid);
        };
        const uint32_t lg_leaves = ilog2_exact(n_leaves);
        const std::string h = std::to_string(hash);
        if (coop && n_leaves <= tune_get("coop_leaves." + h, lg_leaves, 1ULL << 13))
            stage(LS_LEAF_COOP, 0, (n_leaves + LOOP_THREADS / 4 - 1) / (LOOP_THREADS / 4));
        else
            stage(LS_LEAF, 0, (n_leaves + LOOP_THREADS - 1) / LOOP_THREADS);
        if (g.sub_leaves == 1) return;
        const uint64_t wide = tune_get("wide_level_nodes." + h, lg_leaves, 1ULL << 15);
        const uint32_t top = g.log_sub - 1;
        uint32_t u0 = 0;
        while (u0 + 1 <= top && (n_leaves >> (u0 + 1)) >= wide) {
            u0++;
            stage(LS_LEVEL, u0, ((n_leaves >> u0) + LOOP_THREADS - 1) / LOOP_THREADS);
        }
        // the fold takes 64 nodes per CTA (cooperative) or 256 (one permutation
        // per thread), as merkle.cu's fold kernels do
        const uint32_t NG = coop ? LOOP_THREADS / 4 : LOOP_THREADS;
        stage(coop ? LS_FOLD_COOP : LS_FOLD, u0, ((n_leaves >> u0) + NG - 1) / NG);
        if ((g.sub_leaves >> u0) <= NG) return;  // caps written by the fold
        uint32_t U = 0;
        while ((1u << (U + 1)) <= NG && u0 + U + 1 <= top) U++;
        u0 += U;
        while ((g.sub_leaves >> u0) > LOOP_TAIL_MAXM) {
            u0++;
            stage(LS_LEVEL, u0, (((g.sub_leaves >> u0) * g.n_caps) + LOOP_THREADS - 1) / LOOP_THREADS);
        }
        stage(coop ? LS_TAIL_COOP : LS_TAIL, u0, g.n_caps);
    }

    // Plan an admitted job, copy the plan to the device and post it to the
    // ring.  Server thread, without `mu`; returns 1 or a negative status.
    int loop_start(Ticket &t, uint64_t id, int inject)
    {
        const zk_serve_request &r = t.req;
        NvtxRange range("zeknox serve post");
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        try {
            const uint64_t N = 1ULL << (r.lg_n + r.rate_bits);
            if (inject == ZK_SERVE_FAIL_ALLOC)
                throw cuda_failure(-(int)cudaErrorMemoryAllocation, "device allocation refused (injected)");
            if (inject == ZK_SERVE_FAIL_SHAPE) throw arg_failure("shape rejected (injected)");
            const uint64_t gen = (r.coset_gen ? r.coset_gen : ZK_GENERATOR) % GL_P;
            const bool values = r.input_is_values != 0;
            if (!lde_rows_plan_tables_resident(*ctx, r.lg_n, r.rate_bits, gen) ||
                (values && !ntt_inverse_plan_tables_resident(*ctx, r.lg_n))) {
                // the table kernels need SMs the loop occupies
                loop_stop();
                lde_rows_plan_tables(*ctx, r.lg_n, r.rate_bits, gen);
                if (values) ntt_inverse_plan_tables(*ctx, r.lg_n);
                ctx->sync();
            }
            std::vector<LoopStage> plan;
            const uint64_t *coeffs = r.input;
            if (values) {
                // evaluations on H -> coefficients, in the job's scratch after the
                // LDE's (as commit_enqueue): copy, inverse transform, reorder
                const uint64_t n = 1ULL << r.lg_n, words = n * r.cols;
                uint64_t *cf = t.scratch + lde_rows_scratch_elems(r.lg_n, r.rate_bits, r.cols);
                LoopStage cp{};
                cp.kind = LS_COPY;
                cp.blocks = (words + 16 * LOOP_THREADS - 1) / (16 * LOOP_THREADS);
                cp.a.src = r.input;
                cp.a.dst = cf;
                cp.a.n_src = words;
                push_split(plan, cp, 16.0 * LOOP_THREADS * 0.002, (uint64_t)loop_grid);
                PlannedReorder ro{};
                for (const PlannedPass &pp : ntt_inverse_plan(*ctx, cf, r.lg_n, r.cols, cf + words, ro)) {
                    const bool ok = pp.inv && pp.load == LOAD_PLAIN && pp.store == STORE_SAME &&
                                    ((pp.direct && pp.logr >= 6 && pp.logr <= 9) ||
                                     (!pp.direct && pp.logr >= 6 && pp.logr <= 12));
                    if (!ok) throw arg_failure("an inverse pass shape the device loop does not run");
                    LoopStage st{};
                    st.kind = LS_PASS;
                    st.logr = pp.logr;
                    st.load = (uint32_t)pp.load;
                    st.store = (uint32_t)pp.store;
                    st.inv = 1;
                    st.direct = (uint32_t)pp.direct;
                    st.blocks = pp.grid;
                    st.a = pp.a;
                    push_split(plan, st, LOOP_PASS_TILE * LDE_ELEM_NS, (uint64_t)loop_grid);
                }
                LoopStage rs{};
                rs.kind = LS_REORDER;
                rs.blocks = ro.blocks;
                rs.a.src = ro.src;
                rs.a.dst = ro.dst;
                rs.a.src_stride = ro.src_stride;
                rs.a.dst_stride = ro.dst_stride;
                rs.a.L = ro.lg_t;
                rs.a.rate = ro.rate;
                rs.a.vcols = ro.cols;
                rs.a.n_src = ro.mul;
                rs.a.src_len = ro.src_len;
                rs.a.dst_len = ro.dst_len;
                push_split(plan, rs, (double)words / (double)ro.blocks * 0.004, (uint64_t)loop_grid);
                coeffs = cf;
            }
            for (const PlannedPass &pp :
                 lde_rows_plan(*ctx, t.leaves, coeffs, r.lg_n, r.rate_bits, r.cols, gen, t.scratch)) {
                const bool ok = pp.direct && ((pp.load == LOAD_COSETS && pp.store == STORE_SAME && pp.logr >= 1 &&
                                               pp.logr <= 10) ||
                                              (pp.load == LOAD_PLAIN && pp.store == STORE_SAME && pp.logr >= 5 &&
                                               pp.logr <= 7) ||
                                              (pp.load == LOAD_PLAIN && pp.store == STORE_ROWS && pp.logr == 8));
                if (!ok) throw arg_failure("a pass shape the device loop does not run");
                LoopStage st{};
                st.kind = LS_PASS;
                st.logr = pp.logr;
                st.load = (uint32_t)pp.load;
                st.store = (uint32_t)pp.store;
                st.direct = 1;
                st.blocks = pp.grid;
                st.a = pp.a;
                push_split(plan, st, LOOP_PASS_TILE * LDE_ELEM_NS, (uint64_t)loop_grid);
            }
            merkle_stages(plan, t.digests, t.caps, t.leaves, N, r.cols, r.cap_height, r.hash_type, (uint64_t)loop_grid);
            if (plan.size() > LOOP_MAX_STAGES) throw arg_failure("request needs more stages than a ring entry holds");
            if (inject == ZK_SERVE_FAIL_LAUNCH)
                throw cuda_failure(-(int)cudaErrorLaunchFailure, "kernel launch refused (injected)");
            uint32_t k = 0;
            while (k < LOOP_RING && ring_ticket[k]) k++;
            if (k == LOOP_RING) throw arg_failure("no free ring entry");  // admission keeps one free
            LoopStage *host = plans_host + (uint64_t)k * LOOP_MAX_STAGES;
            LoopStage *dev = plans + (uint64_t)k * LOOP_MAX_STAGES;
            memcpy(host, plan.data(), plan.size() * sizeof(LoopStage));
            ZK_CUDA(cudaMemcpyAsync(dev, host, plan.size() * sizeof(LoopStage), cudaMemcpyHostToDevice, copy_stream));
            ZK_CUDA(cudaStreamSynchronize(copy_stream));
            LoopSlot &sl = ring->slot[k];
            sl.n_stages = (uint32_t)plan.size();
            sl.stages = dev;
            const bool gate_shut = inject == ZK_SERVE_FAIL_GATE;
            sl.ready_ns = gate_shut ? 20000000ULL : 10000000000ULL;
            __atomic_store_n(&sl.done, (uint32_t)LOOP_DONE_NONE, __ATOMIC_RELAXED);
            __atomic_store_n(&sl.ready, gate_shut ? 0u : 1u, __ATOMIC_RELEASE);
            ring_ticket[k] = id;
            ring_seq[k] = posted;
            __atomic_store_n(&ring->order[posted % LOOP_RING], k, __ATOMIC_RELAXED);
            posted++;
            __atomic_store_n(&ring->head, posted, __ATOMIC_RELEASE);
            loop_ensure();
            return 1;
        } catch (const std::exception &e) {
            const cuda_failure *cf = dynamic_cast<const cuda_failure *>(&e);
            const arg_failure *af = dynamic_cast<const arg_failure *>(&e);
            (void)cudaGetLastError();
            return cf ? (cf->code < 0 ? cf->code : -1) : af ? -af->code : -1;
        }
    }

    // Retire finished ring entries, in any order (caller holds mu); true if
    // any finished.  Relaunches the loop when entries wait and it has exited.
    bool loop_retire()
    {
        bool progressed = false;
        bool pending = false;
        for (uint32_t k = 0; k < LOOP_RING; k++) {
            if (!ring_ticket[k]) continue;
            LoopSlot &sl = ring->slot[k];
            const uint32_t d = __atomic_load_n(&sl.done, __ATOMIC_ACQUIRE);
            if (d == LOOP_DONE_NONE) {
                pending = true;
                continue;
            }
            Ticket &t = tickets[ring_ticket[k]];
            int status = 2;
            if (d == LOOP_DONE_OK) {
                // per-stage trace: the stage kinds from the plan, the device
                // times from the loop
                const LoopStage *plan = plans_host + (uint64_t)k * LOOP_MAX_STAGES;
                const uint32_t n = sl.n_stages < LOOP_MAX_STAGES ? sl.n_stages : LOOP_MAX_STAGES;
                t.trace_kind.resize(n);
                t.trace_ns.resize(n);
                for (uint32_t q = 0; q < n; q++) {
                    t.trace_kind[q] = plan[q].kind == LS_PASS ? 16 + plan[q].logr : plan[q].kind;
                    t.trace_ns[q] = sl.t_stage[q];
                }
                if (t.req.caps_host) {
                    const uint64_t n_caps = 1ULL << t.req.cap_height;
                    cudaError_t e = cudaMemcpyAsync(t.req.caps_host, t.caps, n_caps * 32, cudaMemcpyDeviceToHost,
                                                    copy_stream);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(copy_stream);
                    if (e != cudaSuccess) status = -(int)e;
                }
            } else {
                status = -(int)cudaErrorLaunchTimeout;  // a bounded wait of the loop ran out
            }
            t.status = status;
            t.t_done = Clock::now();
            __atomic_store_n(&sl.done, (uint32_t)LOOP_DONE_NONE, __ATOMIC_RELAXED);
            ring_ticket[k] = 0;
            retired++;
            completed++;
            progressed = true;
        }
        if (pending) {
            std::lock_guard<std::recursive_mutex> dl(ctx->mu);
            if (!loop_running()) {
                // entries the exited loop had taken and not finished (a CTA
                // gave up on a barrier after the leader passed it) fail
                const uint64_t taken = __atomic_load_n(&ring->taken, __ATOMIC_ACQUIRE);
                for (uint32_t k = 0; k < LOOP_RING; k++)
                    if (ring_ticket[k] && ring_seq[k] < taken &&
                        __atomic_load_n(&ring->slot[k].done, __ATOMIC_ACQUIRE) == LOOP_DONE_NONE)
                        __atomic_store_n(&ring->slot[k].done, (uint32_t)LOOP_DONE_ABORT, __ATOMIC_RELEASE);
                try {
                    loop_ensure();
                } catch (const std::exception &) {
                    (void)cudaGetLastError();
                }
            }
        }
        return progressed;
    }

    void loop_device_mode()
    {
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            if (loop_retire()) cv.notify_all();
            while (!queue.empty() && posted - retired < loop_depth) {
                auto pick = queue.begin();
                if (!ranges.fits(tickets[*pick].bytes)) {
                    if (blocked_head != *pick) {
                        blocked_head = *pick;
                        bypassed = 0;
                    }
                    if (bypassed >= loop_depth) break;
                    for (++pick; pick != queue.end(); ++pick) {
                        const uint64_t b = tickets[*pick].bytes;
                        if (b <= budget / 8 && ranges.fits(b)) break;
                    }
                    if (pick == queue.end()) break;
                    bypassed++;
                }
                const uint64_t id = *pick;
                Ticket &t = tickets[id];
                queue.erase(pick);
                t.off = ranges.take(t.bytes);
                in_use += t.bytes;
                peak = in_use > peak ? in_use : peak;
                place(t);
                t.t_admit = Clock::now();
                t.status = 1;
                const int inject = inject_next;
                inject_next = 0;
                lk.unlock();
                const int st = loop_start(t, id, inject);
                lk.lock();
                if (st < 0) {
                    t.status = st;
                    t.t_done = Clock::now();
                    unadmit(t);
                }
                cv.notify_all();
            }
            const bool busy = retired < posted;
            if (stop && !busy && queue.empty()) break;
            if (busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                lk.lock();
            } else {
                cv.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
        std::lock_guard<std::recursive_mutex> dl(ctx->mu);
        loop_stop();
    }

    void loop()
    {
        if (device_loop) {
            loop_device_mode();
            return;
        }
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            // retire finished jobs
            bool progressed = false;
            for (size_t k = 0; k < slot_ticket.size(); k++) {
                uint64_t id = slot_ticket[k];
                if (!id) continue;
                Ticket &t = tickets[id];
                cudaError_t q = cudaEventQuery(t.done_ev);
                if (q == cudaErrorNotReady) continue;
                t.t_done = Clock::now();
                t.status = q == cudaSuccess ? 2 : -(int)q;
                if (q != cudaSuccess) (void)cudaGetLastError();
                cudaEventDestroy(t.done_ev);
                t.done_ev = nullptr;
                slot_ticket[k] = 0;
                completed++;
                progressed = true;
            }
            if (progressed) cv.notify_all();
            // admit in arrival order, small requests past a head that waits for memory
            while (!queue.empty()) {
                int slot = -1;
                for (size_t k = 0; k < slot_ticket.size(); k++)
                    if (!slot_ticket[k]) {
                        slot = (int)k;
                        break;
                    }
                if (slot < 0) break;
                auto pick = queue.begin();
                if (!ranges.fits(tickets[*pick].bytes)) {
                    if (blocked_head != *pick) {
                        blocked_head = *pick;
                        bypassed = 0;
                    }
                    if (bypassed >= slot_ticket.size()) break;
                    for (++pick; pick != queue.end(); ++pick) {
                        const uint64_t b = tickets[*pick].bytes;
                        if (b <= budget / 8 && ranges.fits(b)) break;
                    }
                    if (pick == queue.end()) break;
                    bypassed++;
                }
                const uint64_t id = *pick;
                Ticket &t = tickets[id];
                queue.erase(pick);
                t.off = ranges.take(t.bytes);
                in_use += t.bytes;
                peak = in_use > peak ? in_use : peak;
                place(t);
                t.slot = slot;
                t.t_admit = Clock::now();
                t.status = 1;
                slot_ticket[slot] = id;
                const int inject = inject_next;
                inject_next = 0;
                lk.unlock();
                const int st = start(t, slot, inject);
                lk.lock();
                if (st < 0) {
                    // could not start: the slot and the range are free again
                    t.status = st;
                    t.t_done = Clock::now();
                    unadmit(t);
                    slot_ticket[slot] = 0;
                }
                cv.notify_all();
            }
            bool busy = false;
            for (uint64_t id : slot_ticket) busy |= id != 0;
            if (stop && !busy && queue.empty()) break;
            if (busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                lk.lock();
            } else {
                cv.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
    }
};

Server *as_server(void *p)
{
    if (!p) throw arg_failure("null server");
    return (Server *)p;
}

RustError to_error(int code, const std::string &msg)
{
    RustError e;
    e.code = code;
    e.message = msg.empty() ? nullptr : strdup(msg.c_str());
    return e;
}

template <class F>
RustError guard(F &&f)
{
    try {
        f();
        return RustError{0, nullptr};
    } catch (const arg_failure &e) {
        return to_error(e.code, e.what());
    } catch (const cuda_failure &e) {
        return to_error(e.code, e.what());
    } catch (const std::exception &e) {
        return to_error(-(int)cudaErrorUnknown, e.what());
    }
}

}  // namespace
}  // namespace zk

using zk::Server;

namespace zk {
namespace {

// The device-loop resources of a server: the ring, the loop's control block,
// the plan buffers, two streams and the launch shape (every CTA resident).
void create_device_loop(Server *s, uint32_t slots)
{
    DeviceCtx &c = *s->ctx;
    int coop = 0;
    ZK_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.id));
    if (!coop) throw arg_failure("the device does not support cooperative launches");
    ZK_CUDA(cudaFuncSetAttribute(serve_loop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LOOP_SMEM_BYTES));
    int per_sm = 0;
    ZK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_loop_kernel, LOOP_THREADS, LOOP_SMEM_BYTES));
    if (per_sm < 1) throw arg_failure("the device loop does not fit on an SM");
    s->loop_grid = per_sm * c.sm_count;
    if (s->loop_grid > (int)LOOP_MAX_CTAS) s->loop_grid = (int)LOOP_MAX_CTAS / c.sm_count * c.sm_count;
    void *h = nullptr;
    ZK_CUDA(cudaHostAlloc(&h, sizeof(LoopRing), cudaHostAllocMapped | cudaHostAllocPortable));
    memset(h, 0, sizeof(LoopRing));
    s->ring = (LoopRing *)h;
    void *d = nullptr;
    ZK_CUDA(cudaHostGetDevicePointer(&d, h, 0));
    s->ring_dev = (LoopRing *)d;
    s->ring->idle_ns = 20000000ULL;      // 20 ms without a request: the kernel exits
    s->ring->barrier_ns = 10000000000ULL;  // 10 s: the longest stage (2^25 leaves x 32 permutations) takes ~1.3 s
    ZK_CUDA(cudaMalloc((void **)&s->ctl, sizeof(LoopCtl)));
    ZK_CUDA(cudaMalloc((void **)&s->plans, sizeof(LoopStage) * LOOP_RING * LOOP_MAX_STAGES));
    ZK_CUDA(cudaHostAlloc((void **)&s->plans_host, sizeof(LoopStage) * LOOP_RING * LOOP_MAX_STAGES,
                          cudaHostAllocDefault));
    ZK_CUDA(cudaStreamCreateWithFlags(&s->loop_stream, cudaStreamNonBlocking));
    ZK_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    ZK_CUDA(cudaEventCreateWithFlags(&s->loop_exit, cudaEventDisableTiming));
    s->loop_depth = slots < LOOP_RING ? slots : LOOP_RING;
    s->device_loop = true;
}

void free_device_loop(Server *s)
{
    if (s->loop_stream) {
        cudaStreamSynchronize(s->loop_stream);
        cudaStreamDestroy(s->loop_stream);
    }
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->loop_exit) cudaEventDestroy(s->loop_exit);
    if (s->ctl) cudaFree(s->ctl);
    if (s->plans) cudaFree(s->plans);
    if (s->plans_host) cudaFreeHost(s->plans_host);
    if (s->ring) cudaFreeHost(s->ring);
}

}  // namespace
}  // namespace zk

extern "C" RustError zeknox_server_create(size_t device_id, uint64_t budget_bytes, uint32_t slots, void **server)
{
    return zeknox_server_create_ex(device_id, budget_bytes, slots, 0, server);
}

extern "C" RustError zeknox_server_create_ex(size_t device_id, uint64_t budget_bytes, uint32_t slots, uint32_t flags,
                                             void **server)
{
    return zk::guard([&] {
        if (!server) throw zk::arg_failure("null out pointer");
        if (slots == 0 || slots > 64) throw zk::arg_failure("slots must be 1..64");
        if (budget_bytes < zk::ARENA_ALIGN) throw zk::arg_failure("budget below one allocation unit");
        if (flags & ~(uint32_t)ZK_SERVE_DEVICE_LOOP) throw zk::arg_failure("unknown server flags");
        zk::DeviceCtx &c = zk::device(device_id);
        Server *s = new Server();
        try {
            s->ctx = &c;
            s->budget = budget_bytes / zk::ARENA_ALIGN * zk::ARENA_ALIGN;
            {
                std::lock_guard<std::recursive_mutex> dl(c.mu);
                // the pool's cached temporaries go back to the driver first, so
                // the reservation sees the device's free memory
                cudaMemPool_t pool;
                if (cudaDeviceGetDefaultMemPool(&pool, c.id) == cudaSuccess) (void)cudaMemPoolTrimTo(pool, 0);
                ZK_CUDA(cudaMalloc((void **)&s->arena, s->budget));
            }
            s->ranges.init(s->budget);
            s->slot_stream.assign(slots, nullptr);
            s->slot_ticket.assign(slots, 0);
            for (auto &st : s->slot_stream) ZK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            ZK_CUDA(cudaEventCreateWithFlags(&s->tables_ready, cudaEventDisableTiming));
            if (flags & ZK_SERVE_DEVICE_LOOP) {
                std::lock_guard<std::recursive_mutex> dl(c.mu);
                zk::create_device_loop(s, slots);
            }
        } catch (...) {
            for (auto &st : s->slot_stream)
                if (st) cudaStreamDestroy(st);
            if (s->tables_ready) cudaEventDestroy(s->tables_ready);
            if (s->arena) cudaFree(s->arena);
            zk::free_device_loop(s);
            delete s;
            throw;
        }
        s->worker = std::thread([s] {
            cudaSetDevice(s->ctx->id);
            s->loop();
        });
        *server = s;
    });
}

extern "C" RustError zeknox_server_submit(void *server, const zk_serve_request *req, uint64_t *ticket)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (!req || !ticket) throw zk::arg_failure("null pointer");
        zk_commit_job j{};
        j.lg_n = req->lg_n;
        j.rate_bits = req->rate_bits;
        j.cols = req->cols;
        j.cap_height = req->cap_height;
        j.hash_type = req->hash_type;
        j.input = req->input;
        j.leaves = (uint64_t *)1;  // buffers are the server's: check shape only
        j.digests = (uint64_t *)1;
        j.caps = (uint64_t *)1;
        zk::check_job(j);
        if (s->device_loop && (req->lg_n < 9 || req->lg_n > 22))
            throw zk::arg_failure("the device loop takes inputs of 2^9 .. 2^22 per column");
        // the server's kernels read the input in place
        if (!zk::device_can_read(req->input, s->ctx->id))
            throw zk::arg_failure("input is pageable host memory this GPU cannot read: pass device or pinned host memory");
        const uint64_t bytes = Server::job_bytes(*req);
        std::lock_guard<std::mutex> lk(s->mu);
        if (bytes > s->budget) throw zk::arg_failure("request needs more device memory than the server's budget");
        const uint64_t id = s->next_id++;
        zk::Ticket &t = s->tickets[id];
        t.req = *req;
        t.bytes = bytes;
        t.t_submit = zk::Clock::now();
        s->queue.push_back(id);
        *ticket = id;
        s->cv.notify_all();
    });
}

extern "C" RustError zeknox_server_wait(void *server, uint64_t ticket, double timeout_ms, zk_serve_result *result)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        auto done = [&] { return it->second.status == 2 || it->second.status < 0; };
        if (timeout_ms < 0) s->cv.wait(lk, done);
        else s->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done);
        const zk::Ticket &t = it->second;
        if (result) {
            result->status = t.status;
            result->latency_ms = t.status == 2 ? std::chrono::duration<double, std::milli>(t.t_done - t.t_submit).count() : 0;
            result->queue_ms = t.status >= 1 || t.status < 0
                                   ? std::chrono::duration<double, std::milli>(t.t_admit - t.t_submit).count()
                                   : 0;
            result->leaves = t.status == 2 ? t.leaves : nullptr;
            result->digests = t.status == 2 ? t.digests : nullptr;
            result->caps = t.status == 2 ? t.caps : nullptr;
        }
    });
}

extern "C" RustError zeknox_server_release(void *server, uint64_t ticket)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        zk::Ticket &t = it->second;
        if (t.status == 0 || t.status == 1) throw zk::arg_failure("ticket still queued or running");
        s->unadmit(t);  // its work has finished: the range is free at once
        s->tickets.erase(it);
        s->cv.notify_all();
    });
}

extern "C" RustError zeknox_server_trace(void *server, uint64_t ticket, uint32_t *kinds, uint64_t *ns, uint32_t max,
                                         uint32_t *n)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (!n) throw zk::arg_failure("null count");
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        const zk::Ticket &t = it->second;
        const uint32_t m = (uint32_t)t.trace_ns.size();
        for (uint32_t q = 0; q < m && q < max; q++) {
            if (kinds) kinds[q] = t.trace_kind[q];
            if (ns) ns[q] = t.trace_ns[q];
        }
        *n = m;
    });
}

extern "C" RustError zeknox_server_stats(void *server, uint64_t *in_use_bytes, uint64_t *peak_bytes,
                                         uint64_t *completed)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::lock_guard<std::mutex> lk(s->mu);
        if (in_use_bytes) *in_use_bytes = s->in_use;
        if (peak_bytes) *peak_bytes = s->peak;
        if (completed) *completed = s->completed;
    });
}

extern "C" RustError zeknox_server_prepare(void *server, uint32_t lg_n_min, uint32_t lg_n_max, uint32_t rate_bits,
                                           uint64_t coset_gen)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (lg_n_min == 0 || lg_n_min > lg_n_max || rate_bits == 0 || rate_bits > 32 || lg_n_max > 32 - rate_bits)
            throw zk::arg_failure("need 1 <= lg_n_min <= lg_n_max and lg_n_max + rate_bits <= 32");
        std::lock_guard<std::recursive_mutex> dl(s->ctx->mu);
        ZK_CUDA(cudaSetDevice(s->ctx->id));
        for (uint32_t lg = lg_n_min; lg <= lg_n_max; lg++) {
            zk_commit_job j{};
            j.lg_n = lg;
            j.rate_bits = rate_bits;
            j.coset_gen = coset_gen;
            j.input_is_values = 1;  // the inverse tables too
            zk::prepare_job(*s->ctx, j);
            // the device loop's pass split (row-output radix 2^8)
            if (s->device_loop)
                zk::lde_rows_plan_tables(*s->ctx, lg, rate_bits, (coset_gen ? coset_gen : ZK_GENERATOR) % zk::GL_P);
        }
        s->ctx->sync();
    });
}

extern "C" RustError zeknox_server_cancel(void *server, uint64_t ticket)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        zk::Ticket &t = it->second;
        if (t.status != 0) throw zk::arg_failure("only a queued request can be cancelled");
        for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
            if (*q == ticket) {
                s->queue.erase(q);
                break;
            }
        if (s->blocked_head == ticket) s->blocked_head = 0;
        t.status = ZK_SERVE_CANCELLED;  // never admitted: it holds no range
        t.t_done = t.t_admit = zk::Clock::now();
        s->cv.notify_all();
    });
}

extern "C" RustError zeknox_server_inject_failure(void *server, int stage)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (stage < 0 || stage > ZK_SERVE_FAIL_GATE) throw zk::arg_failure("unknown failure stage");
        if (stage == ZK_SERVE_FAIL_GATE && !s->device_loop) throw zk::arg_failure("the start gate is the device loop's");
        std::lock_guard<std::mutex> lk(s->mu);
        s->inject_next = stage;
    });
}

extern "C" RustError zeknox_server_destroy(void *server)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
            s->cv.notify_all();
        }
        s->worker.join();
        std::lock_guard<std::recursive_mutex> dl(s->ctx->mu);
        ZK_CUDA(cudaSetDevice(s->ctx->id));
        for (auto &st : s->slot_stream) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        cudaEventDestroy(s->tables_ready);
        zk::free_device_loop(s);
        cudaFree(s->arena);
        delete s;
    });
}
