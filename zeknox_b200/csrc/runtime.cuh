// runtime.cuh -- per-GPU state of the library.
//
// Replaces zeknox's native/utils/gpu_t.cuh + all_gpus.cu device registry and
// the global twiddle/coset arrays of native/ntt/ntt.cu:25-27.  Differences:
//   * tables are built by parallel kernels (the reference runs a serial
//     <<<1,1>>> kernel per table) and lazily on first use, so a missing
//     init_twiddle_factors() is not a null dereference;
//   * every call takes the device's mutex, so concurrent calls from several
//     host threads are serialised instead of racing on shared state;
//   * temporaries come from the stream-ordered allocator on the device's
//     stream and are returned on the same stream.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace zk {

// CUDA failure: code is the negated cudaError_t (native/utils/exception.cuh:21).
struct cuda_failure : std::runtime_error {
    int code;
    cuda_failure(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
// Argument failure: code is +cudaErrorInvalidValue (native/ntt/ntt.cu:256,318,480).
struct arg_failure : std::runtime_error {
    int code;
    explicit arg_failure(const std::string &m) : std::runtime_error(m), code((int)cudaErrorInvalidValue) {}
};

void cuda_check(cudaError_t e, const char *what, const char *file, int line);
#define ZK_CUDA(x) ::zk::cuda_check((x), #x, __FILE__, __LINE__)

struct DeviceCtx {
    int id = 0;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    int sm_count = 0;

    // twiddle tables: tw[inv][lg] = w_{2^lg}^t for t < 2^lg (w = OMEGA or OMEGA_INV)
    uint64_t *tw[2][33] = {};
    // coset powers g^i, i < 2^coset_lg (init_coset)
    uint64_t *coset = nullptr;
    uint32_t coset_lg = 0;
    uint64_t coset_gen = 7;
    bool coset_set = false;
    // LDE coset tables: (lg_n, rate, g) -> (g * w_N^c)^j
    std::map<std::tuple<uint32_t, uint32_t, uint64_t>, uint64_t *> lde_tabs;

    const uint64_t *twiddles(uint32_t lg, bool inverse);
    const uint64_t *coset_powers(uint32_t lg);  // builds g^i up to 2^lg if needed
    const uint64_t *lde_table(uint32_t lg_n, uint32_t rate, uint64_t g);
    void set_coset(uint32_t lg, uint64_t gen);

    // host->device staging of commit inputs: a copy stream and per-chunk events
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> chunk_events;
    cudaStream_t copy_stream_get();
    cudaEvent_t chunk_event(size_t i);

    uint64_t *alloc(size_t bytes);
    void free(void *p);
    // Synchronises the stream, then reports a bounded device wait that ran
    // out since the last check (cuda_failure, -cudaErrorLaunchTimeout).
    void sync();

    // Status word of the bounded device waits (bulk-copy stages): mapped
    // pinned memory, so kernels raise it with a system-scope atomic and sync()
    // reads it without a copy.  Calls queued on a caller's stream are reported
    // by the device's next synchronous call.
    unsigned *wait_status_host = nullptr;
    unsigned *wait_status_dev = nullptr;
    unsigned *wait_status();
    void check_waits();
    // Test hook: the next inject_wait_timeouts bulk transposes declare 16
    // bytes more than they copy, so one stage's wait runs out.
    uint32_t inject_wait_timeouts = 0;
};

int device_count();
DeviceCtx &device(size_t id);  // throws arg_failure for a bad id; makes it current

// RAII temporary on the device stream
struct DevBuf {
    DeviceCtx *ctx = nullptr;
    uint64_t *p = nullptr;
    DevBuf() = default;
    DevBuf(DeviceCtx &c, size_t elems) : ctx(&c), p(elems ? c.alloc(elems * 8) : nullptr) {}
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf()
    {
        if (p) ctx->free(p);
    }
};

uint32_t ilog2_exact(uint64_t x);  // -1u if x is not a power of two

// Tuning table: named knobs, optionally per log2 size, set by the autotuner
// (zeknox_tune_set / zeknox_tune_load); tune_get falls back to the size-free
// entry and then to `dflt`.  Knobs: "leaf_threads.<hash>" (64/128/256),
// "lde_chunk_mib", "lde_host_chunk_mib", "lde_last_logr" (1..8), "wide_level_nodes.<hash>",
// "coop_leaves.<hash>", "transpose_bulk" (0 16-byte form, 1..8 bulk-copy tile
// shape, 9 by column count), "ntt_split_logr" (largest pass of a
// column-output transform, 1..10; 0 the built-in split).
uint64_t tune_get(const std::string &name, uint32_t lg, uint64_t dflt);
void tune_set(const std::string &name, uint32_t lg, uint64_t value);
void tune_clear();
// Reads "<name> <lg|*> <value>" lines ('#' comments); throws arg_failure on a
// malformed line, in which case no knob is changed.
void tune_load_file(const char *path);
// Bumped by every tune_set / tune_clear: cached CUDA graphs record it in their
// key, so a graph captured under other knob values is not replayed.
uint64_t tune_generation();
constexpr uint32_t TUNE_ANY = 0xFFFFFFFFu;

// NVTX range over a host-side stage (queuing an LDE, a forest, a commit, a
// batch): a profiler that records NVTX (nsys, ncu's NVTX filters) shows the
// stages by name; without one attached a range costs a few nanoseconds.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Count of kernels this library has launched (diagnostics: zeknox_launch_count).
void note_launch(uint64_t n = 1);
uint64_t launch_count();

}  // namespace zk
