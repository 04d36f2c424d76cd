// runtime.cu -- device registry, tables and temporaries.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <memory>

#include "gl64.cuh"
#include "ntt.cuh"
#include "runtime.cuh"
#include "zk_constants.h"

namespace zk {

static const uint64_t H_OMEGA[33] = {ZK_OMEGA_LIST};
static const uint64_t H_OMEGA_INV[33] = {ZK_OMEGA_INV_LIST};

void cuda_check(cudaError_t e, const char *what, const char *file, int line)
{
    if (e == cudaSuccess) return;
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
    (void)cudaGetLastError();  // clear a non-sticky error so the context stays usable
    throw cuda_failure(-(int)e, buf);
}

uint32_t ilog2_exact(uint64_t x)
{
    if (x == 0 || (x & (x - 1))) return ~0u;
    uint32_t l = 0;
    while ((1ULL << l) < x) l++;
    return l;
}

static std::atomic<uint64_t> g_launches{0};
void note_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

static std::mutex g_tune_mu;
static std::map<std::pair<std::string, uint32_t>, uint64_t> g_tune;
static std::atomic<uint64_t> g_tune_gen{0};

uint64_t tune_generation() { return g_tune_gen.load(std::memory_order_relaxed); }

// A table named by ZEKNOX_TUNE_FILE ("none": no table) is read at the first
// knob lookup, so consumers of the C ABI get tuned knobs without calling
// zeknox_tune_load.
static std::once_flag g_tune_env_once;
static void tune_env_load()
{
    const char *path = getenv("ZEKNOX_TUNE_FILE");
    if (!path || !*path || strcmp(path, "none") == 0) return;
    try {
        tune_load_file(path);
    } catch (const std::exception &e) {
        fprintf(stderr, "zeknox: ZEKNOX_TUNE_FILE ignored: %s\n", e.what());
    }
}

uint64_t tune_get(const std::string &name, uint32_t lg, uint64_t dflt)
{
    std::call_once(g_tune_env_once, tune_env_load);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({name, lg});
    if (it != g_tune.end()) return it->second;
    it = g_tune.find({name, TUNE_ANY});
    return it != g_tune.end() ? it->second : dflt;
}

void tune_set(const std::string &name, uint32_t lg, uint64_t value)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{name, lg}] = value;
    g_tune_gen.fetch_add(1, std::memory_order_relaxed);
}

void tune_clear()
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    g_tune_gen.fetch_add(1, std::memory_order_relaxed);
}

void tune_load_file(const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f) throw arg_failure(std::string("cannot open tuning table ") + path);
    std::vector<std::tuple<std::string, uint32_t, uint64_t>> entries;
    char line[256];
    int ln = 0;
    while (fgets(line, sizeof line, f)) {
        ln++;
        char *hash = strchr(line, '#');
        if (hash) *hash = 0;
        char name[128], lgs[32], extra[8];
        unsigned long long value;
        const int got = sscanf(line, "%127s %31s %llu %7s", name, lgs, &value, extra);
        if (got == EOF || got == 0) continue;  // blank or comment-only line
        char *end = nullptr;
        const unsigned long lg = strtoul(lgs, &end, 10);
        const bool any = strcmp(lgs, "*") == 0;
        if (got != 3 || (!any && (*end || lg > 64))) {
            fclose(f);
            throw arg_failure(std::string(path) + ":" + std::to_string(ln) + ": expected '<name> <lg|*> <value>'");
        }
        entries.emplace_back(name, any ? TUNE_ANY : (uint32_t)lg, (uint64_t)value);
    }
    fclose(f);
    // all or nothing: a malformed table changes no knob
    for (auto &e : entries) tune_set(std::get<0>(e), std::get<1>(e), std::get<2>(e));
}

static std::mutex g_reg_mu;
static std::vector<std::unique_ptr<DeviceCtx>> g_devs;
static int g_ndev = -1;

int device_count()
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    if (g_ndev < 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            (void)cudaGetLastError();
            n = 0;
        }
        g_ndev = n;
        g_devs.resize(n);
    }
    return g_ndev;
}

DeviceCtx &device(size_t id)
{
    int n = device_count();
    if (id >= (size_t)n) throw arg_failure("invalid device id " + std::to_string(id) + " (" + std::to_string(n) + " GPUs)");
    std::lock_guard<std::mutex> lk(g_reg_mu);
    if (!g_devs[id]) {
        auto c = std::make_unique<DeviceCtx>();
        c->id = (int)id;
        ZK_CUDA(cudaSetDevice((int)id));
        // blocking stream: ordered with the legacy default stream like the
        // reference's per-GPU "zero" stream (native/utils/gpu_t.cuh:247)
        ZK_CUDA(cudaStreamCreate(&c->stream));
        ZK_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, (int)id));
        // keep freed temporaries in the stream-ordered pool across calls
        // instead of returning them to the driver at every synchronisation
        cudaMemPool_t pool;
        ZK_CUDA(cudaDeviceGetDefaultMemPool(&pool, (int)id));
        uint64_t keep = UINT64_MAX;
        ZK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        g_devs[id] = std::move(c);
    }
    ZK_CUDA(cudaSetDevice((int)id));
    return *g_devs[id];
}

cudaStream_t DeviceCtx::copy_stream_get()
{
    if (!copy_stream) ZK_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    return copy_stream;
}

cudaEvent_t DeviceCtx::chunk_event(size_t i)
{
    while (chunk_events.size() <= i) {
        cudaEvent_t e;
        ZK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        chunk_events.push_back(e);
    }
    return chunk_events[i];
}

uint64_t *DeviceCtx::alloc(size_t bytes)
{
    void *p = nullptr;
    ZK_CUDA(cudaMallocAsync(&p, bytes, stream));
    return (uint64_t *)p;
}

void DeviceCtx::free(void *p)
{
    if (p) (void)cudaFreeAsync(p, stream);
}

void DeviceCtx::sync()
{
    ZK_CUDA(cudaStreamSynchronize(stream));
    check_waits();
}

unsigned *DeviceCtx::wait_status()
{
    if (!wait_status_dev) {
        void *h = nullptr;
        ZK_CUDA(cudaHostAlloc(&h, sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable));
        *(volatile unsigned *)h = 0;
        void *d = nullptr;
        ZK_CUDA(cudaHostGetDevicePointer(&d, h, 0));
        wait_status_host = (unsigned *)h;
        wait_status_dev = (unsigned *)d;
    }
    return wait_status_dev;
}

void DeviceCtx::check_waits()
{
    if (!wait_status_host) return;
    const unsigned n = *(volatile unsigned *)wait_status_host;
    if (!n) return;
    *(volatile unsigned *)wait_status_host = 0;
    throw cuda_failure(-(int)cudaErrorLaunchTimeout,
                       std::to_string(n) + " CTA(s) stopped: a bulk-copy stage did not complete within its wait limit");
}

static uint64_t *build_powers(DeviceCtx &c, uint64_t w, uint64_t count)
{
    uint64_t *t = nullptr;
    ZK_CUDA(cudaMalloc(&t, count * 8));
    uint64_t blocks = (count + 255) / 256;
    if (blocks > (uint64_t)c.sm_count * 16) blocks = (uint64_t)c.sm_count * 16;
    powers_kernel<<<(unsigned)blocks, 256, 0, c.stream>>>(t, count, w);
    note_launch();
    ZK_CUDA(cudaGetLastError());
    return t;
}

const uint64_t *DeviceCtx::twiddles(uint32_t lg, bool inverse)
{
    if (lg > 32) throw arg_failure("transform size 2^" + std::to_string(lg) + " exceeds the field's 2^32 roots");
    uint64_t *&t = tw[inverse ? 1 : 0][lg];
    if (!t) t = build_powers(*this, inverse ? H_OMEGA_INV[lg] : H_OMEGA[lg], 1ULL << lg);
    return t;
}

void DeviceCtx::set_coset(uint32_t lg, uint64_t gen)
{
    if (coset) {
        ZK_CUDA(cudaStreamSynchronize(stream));
        ZK_CUDA(cudaFree(coset));
        coset = nullptr;
    }
    coset_gen = gen % GL_P;
    coset_set = true;
    coset_lg = lg;
    coset = build_powers(*this, coset_gen, 1ULL << lg);
}

const uint64_t *DeviceCtx::coset_powers(uint32_t lg)
{
    if (!coset_set) coset_gen = 7;  // GROUP_GENERATOR; init_coset() was never called
    if (!coset || coset_lg < lg) {
        uint64_t gen = coset_gen;
        set_coset(lg > coset_lg ? lg : coset_lg, gen);
    }
    return coset;
}

const uint64_t *DeviceCtx::lde_table(uint32_t lg_n, uint32_t rate, uint64_t g)
{
    auto key = std::make_tuple(lg_n, rate, g);
    auto it = lde_tabs.find(key);
    if (it != lde_tabs.end()) return it->second;
    uint64_t n = 1ULL << lg_n;
    uint64_t count = n << rate;
    uint64_t *t = nullptr;
    ZK_CUDA(cudaMalloc(&t, count * 8));
    uint64_t blocks = (count + 255) / 256;
    if (blocks > (uint64_t)sm_count * 16) blocks = (uint64_t)sm_count * 16;
    coset_powers_kernel<<<(unsigned)blocks, 256, 0, stream>>>(t, n, 1u << rate, g, H_OMEGA[lg_n + rate]);
    note_launch();
    ZK_CUDA(cudaGetLastError());
    lde_tabs[key] = t;
    return t;
}

}  // namespace zk
