// noalloc.cu -- zeknox_lde_rows_noalloc: the fused LDE for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need the LDE:
// code recording into a CUDA graph, code running under an allocator that owns
// all device memory (a framework's caching allocator or a fixed arena), or a
// host thread that must never block on the driver's allocator.  The regular
// entry points take their temporaries and tables from the stream-ordered pool
// and build tables on first use, which allocates.  This entry point instead
// keeps everything it needs in file-scope device arrays that exist from the
// moment the library's device code is loaded on a GPU until the process exits:
//   * scratch: NOALLOC_SCRATCH_WORDS words (32 MiB), the inter-pass buffer of
//     one column chunk;
//   * the twiddle tables w_{2^k}^t (k <= 18) and the coset table of the last
//     shape used.
// Limits: lg_n + rate_bits <= NOALLOC_MAX_LG (18).  The scratch is shared by
// every call on a GPU and keeps the last call's contents (it needs no
// clearing: each pass fully writes what the next pass reads); calls whose
// work overlaps on the GPU race on it and on the coset table, so callers
// serialise them (one stream, or their own ordering).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/zeknox_b200.h"
#include "gl64.cuh"
#include "ntt.cuh"
#include "ntt_api.cuh"
#include "runtime.cuh"
#include "zk_constants.h"

namespace {

constexpr uint32_t NOALLOC_MAX_LG = 18;
constexpr uint64_t NOALLOC_SCRATCH_WORDS = 1ULL << 22;  // 32 MiB
constexpr uint64_t NOALLOC_TW_WORDS = 1ULL << (NOALLOC_MAX_LG + 1);  // tables k = 0..18 back to back
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) uint64_t g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];
static __device__ __align__(256) uint64_t g_noalloc_twiddles[NOALLOC_TW_WORDS];
static __device__ __align__(256) uint64_t g_noalloc_coset[1ULL << NOALLOC_MAX_LG];

const uint64_t H_OMEGA[33] = {ZK_OMEGA_LIST};

// Per-device device addresses of the arrays above (host code may not use the
// arrays' names as device pointers) and what the tables currently hold.
struct NoAllocState {
    bool ready = false;
    uint64_t *scratch = nullptr, *twiddles = nullptr, *coset = nullptr;
    uint32_t tw_built = 0;  // bit k set: table of 2^k entries filled
    uint32_t cos_lg = ~0u, cos_rate = ~0u;
    uint64_t cos_gen = 0;
};
NoAllocState g_state[NOALLOC_MAX_DEVICES];
std::mutex g_mu;

__global__ void noalloc_powers(uint64_t *tab, uint64_t count, uint64_t w)
{
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x)
        tab[t] = zk::gl_pow(w, t);
}

__global__ void noalloc_coset_powers(uint64_t *tab, uint64_t n, uint32_t cosets, uint64_t g, uint64_t wN)
{
    uint64_t total = n * cosets;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t c = k / n, j = k % n;
        tab[k] = zk::gl_pow(zk::gl_mul(g, zk::gl_pow(wN, c)), j);
    }
}

uint64_t *tw_table(NoAllocState &st, uint32_t k) { return st.twiddles + ((1ULL << k) - 1); }

void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw zk::cuda_failure(-(int)e, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

}  // namespace

extern "C" RustError zeknox_lde_rows_noalloc(size_t device_id, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n,
                                             uint32_t rate_bits, uint32_t cols, uint64_t coset_gen, void *stream)
{
    RustError r{0, nullptr};
    try {
        if (lg_n == 0 || rate_bits == 0 || cols == 0) throw zk::arg_failure("lg_n, rate_bits and cols must be >= 1");
        if (lg_n + rate_bits > NOALLOC_MAX_LG)
            throw zk::arg_failure("zeknox_lde_rows_noalloc: lg_n + rate_bits = " + std::to_string(lg_n + rate_bits) +
                                  " exceeds the static limit of " + std::to_string(NOALLOC_MAX_LG));
        if (!rows || !coeffs) throw zk::arg_failure("null buffer");
        if (device_id >= (size_t)NOALLOC_MAX_DEVICES) throw zk::arg_failure("device id out of range");
        int ndev = 0;
        check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (device_id >= (size_t)ndev) throw zk::arg_failure("invalid device id");
        check(cudaSetDevice((int)device_id), "cudaSetDevice");
        cudaStream_t s = (cudaStream_t)stream;  // NULL: the legacy default stream
        const uint64_t gen = (coset_gen ? coset_gen : ZK_GENERATOR) % zk::GL_P;

        std::lock_guard<std::mutex> lk(g_mu);
        NoAllocState &st = g_state[device_id];
        if (!st.ready) {
            // one-time set-up on this device (with it current): device
            // addresses of the file-scope arrays
            check(cudaGetSymbolAddress((void **)&st.scratch, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
            check(cudaGetSymbolAddress((void **)&st.twiddles, g_noalloc_twiddles), "cudaGetSymbolAddress(twiddles)");
            check(cudaGetSymbolAddress((void **)&st.coset, g_noalloc_coset), "cudaGetSymbolAddress(coset)");
            st.ready = true;
        }
        // tables: filled by kernels into the static arrays, once per size
        const uint64_t *tw[33] = {};
        auto need = [&](uint32_t k) {
            if (!(st.tw_built >> k & 1)) {
                noalloc_powers<<<(unsigned)(((1ULL << k) + 255) / 256 < 1024 ? ((1ULL << k) + 255) / 256 : 1024), 256, 0,
                                 s>>>(tw_table(st, k), 1ULL << k, H_OMEGA[k]);
                check(cudaGetLastError(), "twiddle table");
                st.tw_built |= 1u << k;
            }
            tw[k] = tw_table(st, k);
        };
        need(12);
        for (auto &p : zk::lde_rows_passes(lg_n))
            if (p.first) need(p.first + p.second);
        if (st.cos_lg != lg_n || st.cos_rate != rate_bits || st.cos_gen != gen) {
            const uint64_t total = 1ULL << (lg_n + rate_bits);
            noalloc_coset_powers<<<(unsigned)((total + 255) / 256 < 1024 ? (total + 255) / 256 : 1024), 256, 0, s>>>(
                st.coset, 1ULL << lg_n, 1u << rate_bits, gen, H_OMEGA[lg_n + rate_bits]);
            check(cudaGetLastError(), "coset table");
            st.cos_lg = lg_n;
            st.cos_rate = rate_bits;
            st.cos_gen = gen;
        }
        // column chunk so that the intermediate fits the static scratch
        const uint64_t N = 1ULL << (lg_n + rate_bits);
        uint64_t chunk = (NOALLOC_SCRATCH_WORDS / N) / 16 * 16;
        if (chunk < 16) throw zk::arg_failure("static scratch too small for this size");
        zk::lde_rows_explicit(s, rows, coeffs, lg_n, rate_bits, cols, st.coset, tw, st.scratch, chunk);
        if (!stream) check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    } catch (const zk::arg_failure &e) {
        r.code = e.code;
        r.message = strdup(e.what());
    } catch (const zk::cuda_failure &e) {
        r.code = e.code;
        r.message = strdup(e.what());
    } catch (const std::exception &e) {
        r.code = -(int)cudaErrorUnknown;
        r.message = strdup(e.what());
    }
    return r;
}
