// batch.cu -- commit jobs and graph-captured batches of jobs.
#include <algorithm>
#include <cstring>
#include <list>
#include <mutex>
#include <string>
#include <vector>

#include "batch.cuh"
#include "ntt_api.cuh"
#include "zk_constants.h"

namespace zk {

void check_job(const zk_commit_job &j)
{
    if (j.lg_n == 0 || j.rate_bits == 0 || j.cols == 0) throw arg_failure("lg_n, rate_bits and cols must be >= 1");
    if (j.rate_bits > 32 || j.lg_n > 32 - j.rate_bits) throw arg_failure("extended size above 2^32");
    if (j.cap_height > j.lg_n + j.rate_bits) throw arg_failure("cap_height above log2 of the leaf count");
    if (!j.input || !j.leaves || !j.caps || (!j.digests && j.cap_height < j.lg_n + j.rate_bits))
        throw arg_failure("null buffer");
    if (j.hash_type > 4) throw arg_failure("unsupported hash_type");
}

uint64_t commit_scratch_words(uint32_t lg_n, uint32_t rate_bits, uint32_t cols, bool values, bool host_input)
{
    uint64_t w = lde_rows_scratch_elems(lg_n, rate_bits, cols);
    if (values) w += 2 * ((uint64_t)cols << lg_n);  // coefficients + inverse-transform temporary
    else if (host_input) w += (uint64_t)cols << lg_n;  // device staging of the coefficients
    return w;
}

bool is_host_pointer(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return true;  // not known to CUDA: pageable host memory
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

bool device_can_read(const void *p, int dev)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        a.type = cudaMemoryTypeUnregistered;
    }
    if (a.type != cudaMemoryTypeUnregistered) return true;  // device, managed or pinned (mapped) host memory
    int pageable = 0;
    if (cudaDeviceGetAttribute(&pageable, cudaDevAttrPageableMemoryAccess, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return pageable != 0;
}

static uint64_t gen_of(const zk_commit_job &j) { return j.coset_gen ? j.coset_gen : ZK_GENERATOR; }

void prepare_job(DeviceCtx &c, const zk_commit_job &j)
{
    prepare_tables(c, j.lg_n, j.rate_bits, gen_of(j), j.input_is_values != 0);
}

void commit_enqueue(DeviceCtx &c, const zk_commit_job &j, cudaStream_t s, uint64_t *scratch, bool host_input)
{
    NvtxRange range("zeknox commit");
    const uint64_t n = 1ULL << j.lg_n;
    const uint64_t N = n << j.rate_bits;
    cudaStream_t keep = c.stream;
    c.stream = s;
    try {
        const uint64_t *coeffs = j.input;
        const uint64_t *host_coeffs = nullptr;
        uint64_t *lde_scratch = scratch;
        uint64_t *extra = scratch + lde_rows_scratch_elems(j.lg_n, j.rate_bits, j.cols);
        if (j.input_is_values) {
            // evaluations on H -> coefficients (inverse NTT), then the LDE
            uint64_t *cf = extra;
            ZK_CUDA(cudaMemcpyAsync(cf, j.input, n * j.cols * 8, cudaMemcpyDefault, s));
            ntt_batch_device(c, cf, j.lg_n, j.cols, true, false, cf + n * j.cols);
            coeffs = cf;
        } else if (host_input) {
            host_coeffs = j.input;
            coeffs = extra;  // staging, filled chunk by chunk
        }
        lde_rows_device(c, j.leaves, coeffs, j.lg_n, j.rate_bits, j.cols, gen_of(j), lde_scratch, host_coeffs);
        std::string err;
        const uint64_t n_caps = 1ULL << j.cap_height;
        if (!merkle_device(j.digests, j.caps, j.leaves, 2 * (N - n_caps), n_caps, N, j.cols, j.cap_height,
                           j.hash_type, s, err))
            throw arg_failure(err);
    } catch (...) {
        c.stream = keep;
        throw;
    }
    c.stream = keep;
}

// ------------------------------------------------------------ graph cache

namespace {

struct BatchGraph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t *> scratch;  // per branch
    ~BatchGraph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        for (uint64_t *p : scratch)
            if (p) cudaFree(p);
    }
};

constexpr int BRANCHES = 8;
constexpr size_t CACHE = 4;

struct DevBatchState {
    int dev = -1;
    cudaStream_t branch[BRANCHES] = {};
    cudaEvent_t fork = nullptr, join[BRANCHES] = {};
    std::list<BatchGraph> graphs;  // most recent first
};

std::vector<DevBatchState> g_state;
std::mutex g_state_mu;

DevBatchState &state_for(DeviceCtx &c)
{
    std::lock_guard<std::mutex> lk(g_state_mu);
    for (auto &s : g_state)
        if (s.dev == c.id) return s;
    g_state.emplace_back();
    DevBatchState &s = g_state.back();
    s.dev = c.id;
    for (int b = 0; b < BRANCHES; b++) {
        ZK_CUDA(cudaStreamCreateWithFlags(&s.branch[b], cudaStreamNonBlocking));
        ZK_CUDA(cudaEventCreateWithFlags(&s.join[b], cudaEventDisableTiming));
    }
    ZK_CUDA(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming));
    return s;
}

std::vector<uint64_t> batch_key(const zk_commit_job *jobs, uint32_t njobs)
{
    std::vector<uint64_t> k;
    k.reserve(njobs * 7 + 2);
    k.push_back(0xC0FFULL);  // distinct from Merkle batch keys
    k.push_back(tune_generation());
    for (uint32_t i = 0; i < njobs; i++) {
        const zk_commit_job &j = jobs[i];
        k.push_back(((uint64_t)j.lg_n << 48) | ((uint64_t)j.rate_bits << 40) | ((uint64_t)j.cap_height << 32) | j.cols);
        k.push_back(((uint64_t)j.hash_type << 32) | j.input_is_values);
        k.push_back(j.coset_gen);
        k.push_back((uint64_t)j.input);
        k.push_back((uint64_t)j.leaves);
        k.push_back((uint64_t)j.digests);
        k.push_back((uint64_t)j.caps);
    }
    return k;
}

}  // namespace

// Record njobs jobs into one graph (cached under `key`), jobs spread over
// the branch streams by cost, and launch it on c.stream.
template <class Enqueue>
static void run_graph(DeviceCtx &c, std::vector<uint64_t> key, uint32_t njobs, const std::vector<double> &cost,
                      const std::vector<uint64_t> &scratch_words, Enqueue enqueue)
{
    DevBatchState &st = state_for(c);
    for (auto it = st.graphs.begin(); it != st.graphs.end(); ++it) {
        if (it->key == key) {
            st.graphs.splice(st.graphs.begin(), st.graphs, it);
            ZK_CUDA(cudaGraphLaunch(st.graphs.front().exec, c.stream));
            return;
        }
    }
    std::vector<uint32_t> order(njobs);
    for (uint32_t i = 0; i < njobs; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
    const int nb = (int)std::min<uint32_t>(BRANCHES, njobs);
    std::vector<double> load(nb, 0.0);
    std::vector<std::vector<uint32_t>> lanes(nb);
    std::vector<uint64_t> need(nb, 0);
    for (uint32_t i : order) {
        int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[b] += cost[i];
        lanes[b].push_back(i);
        need[b] = std::max<uint64_t>(need[b], scratch_words[i]);
    }
    st.graphs.emplace_front();
    BatchGraph &g = st.graphs.front();
    g.key = std::move(key);
    g.scratch.assign(nb, nullptr);
    try {
        for (int b = 0; b < nb; b++)
            if (need[b]) ZK_CUDA(cudaMalloc(&g.scratch[b], need[b] * 8));
    } catch (...) {
        st.graphs.pop_front();
        throw;
    }
    cudaGraph_t graph = nullptr;
    ZK_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
        ZK_CUDA(cudaEventRecord(st.fork, c.stream));
        for (int b = 0; b < nb; b++) {
            ZK_CUDA(cudaStreamWaitEvent(st.branch[b], st.fork, 0));
            for (uint32_t i : lanes[b]) enqueue(i, st.branch[b], g.scratch[b]);
            ZK_CUDA(cudaEventRecord(st.join[b], st.branch[b]));
            ZK_CUDA(cudaStreamWaitEvent(c.stream, st.join[b], 0));
        }
    } catch (...) {
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(c.stream, &dead);
        if (dead) cudaGraphDestroy(dead);
        st.graphs.pop_front();
        throw;
    }
    ZK_CUDA(cudaStreamEndCapture(c.stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        st.graphs.pop_front();
        ZK_CUDA(e);
    }
    while (st.graphs.size() > CACHE) st.graphs.pop_back();
    ZK_CUDA(cudaGraphLaunch(g.exec, c.stream));
}

void commit_batch_graph(DeviceCtx &c, const zk_commit_job *jobs, uint32_t njobs)
{
    NvtxRange range("zeknox commit_batch");
    if (njobs == 0) return;
    std::vector<double> cost(njobs);
    std::vector<uint64_t> words(njobs);
    for (uint32_t i = 0; i < njobs; i++) {
        const zk_commit_job &j = jobs[i];
        cost[i] = (double)(1ULL << (j.lg_n + j.rate_bits)) * ((j.cols + 7) / 8 + 1);
        if (is_host_pointer(j.input)) throw arg_failure("batched commits take device inputs");
        words[i] = commit_scratch_words(j.lg_n, j.rate_bits, j.cols, j.input_is_values != 0, false);
        prepare_job(c, j);
    }
    ZK_CUDA(cudaStreamSynchronize(c.stream));
    run_graph(c, batch_key(jobs, njobs), njobs, cost, words,
              [&](uint32_t i, cudaStream_t s, uint64_t *scratch) { commit_enqueue(c, jobs[i], s, scratch); });
}

void merkle_batch_graph(DeviceCtx &c, const zk_merkle_job *jobs, uint32_t njobs)
{
    NvtxRange range("zeknox merkle_batch");
    if (njobs == 0) return;
    std::vector<double> cost(njobs);
    std::vector<uint64_t> words(njobs, 0);
    std::vector<uint64_t> key;
    key.push_back(0xFEEDULL);  // distinct from commit keys
    key.push_back(tune_generation());
    for (uint32_t i = 0; i < njobs; i++) {
        const zk_merkle_job &j = jobs[i];
        std::string err;
        const uint64_t n_caps = 1ULL << j.cap_height;
        if (j.cap_height >= 63 || !merkle_geometry_ok(2 * (j.n_leaves - n_caps), n_caps, j.n_leaves, j.cap_height, err))
            throw arg_failure("tree " + std::to_string(i) + ": " + (err.empty() ? "bad cap_height" : err));
        if (j.hash_type > 4) throw arg_failure("tree " + std::to_string(i) + ": unsupported hash_type");
        if (!j.leaves || !j.caps || (!j.digests && n_caps < j.n_leaves)) throw arg_failure("null buffer");
        cost[i] = (double)j.n_leaves * ((j.leaf_size + 7) / 8 + 1);
        for (uint64_t v : {(uint64_t)j.leaves, (uint64_t)j.digests, (uint64_t)j.caps, j.n_leaves, j.leaf_size,
                           ((uint64_t)j.cap_height << 32) | j.hash_type})
            key.push_back(v);
    }
    run_graph(c, std::move(key), njobs, cost, words, [&](uint32_t i, cudaStream_t s, uint64_t *) {
        const zk_merkle_job &j = jobs[i];
        std::string err;
        const uint64_t n_caps = 1ULL << j.cap_height;
        if (!merkle_device(j.digests, j.caps, j.leaves, 2 * (j.n_leaves - n_caps), n_caps, j.n_leaves, j.leaf_size,
                           j.cap_height, j.hash_type, s, err))
            throw arg_failure(err);
    });
}

}  // namespace zk
