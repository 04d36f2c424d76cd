// noalloc.cu -- zeknox_lde_rows_noalloc: the fused LDE for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc where they need the LDE: code whose
// device memory is all owned by another allocator (a framework's caching
// allocator or an arena reserved at start-up, where a cudaMalloc fails or
// fragments that arena), or a host thread on a latency-critical path that must
// not enter the driver's allocator (cudaMalloc and cudaFree can synchronise
// the device).  The regular entry points take their temporaries and tables
// from the stream-ordered pool and build tables on first use, which allocates.
// This entry point instead keeps everything it needs in file-scope device
// arrays that exist from the moment the library's device code is loaded on a
// GPU until the process exits:
//   * scratch: NOALLOC_SCRATCH_WORDS words (32 MiB), the inter-pass buffer of
//     one column chunk;
//   * the twiddle tables w_{2^k}^t for every k <= 18, filled once per device
//     by the first call;
//   * the coset table (g * w_N^c)^j, rebuilt by every call for its own shape
//     and generator before its transform, so a call never depends on what an
//     earlier call of another shape left there.
// Limits: lg_n + rate_bits <= NOALLOC_MAX_LG (18).  The scratch and the coset
// table are shared by every call on a GPU and keep the last call's contents
// (the scratch needs no clearing: each pass fully writes what the next pass
// reads); calls whose work overlaps on the GPU race on them, so callers
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
// arrays' names as device pointers); set, with every twiddle table filled, by
// the first call on the device.
struct NoAllocState {
    bool ready = false;
    uint64_t *scratch = nullptr, *twiddles = nullptr, *coset = nullptr;
};
NoAllocState g_state[NOALLOC_MAX_DEVICES];
std::mutex g_mu;

__global__ void noalloc_powers(uint64_t *tab, uint64_t count, uint64_t w)
{
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x)
        tab[t] = zk::gl_pow(w, t);
}

// tab[c * n + j] = (g * wN^c)^j: each thread fills a run of COSET_RUN
// consecutive j with one exponentiation and then one multiply per entry.
constexpr uint32_t COSET_RUN = 16;
__global__ void noalloc_coset_powers(uint64_t *tab, uint64_t n, uint32_t cosets, uint64_t g, uint64_t wN)
{
    const uint64_t runs_per_coset = (n + COSET_RUN - 1) / COSET_RUN;
    const uint64_t runs = runs_per_coset * cosets;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < runs; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = k / runs_per_coset, j0 = (k - c * runs_per_coset) * COSET_RUN;
        const uint64_t base = zk::gl_mul(g, zk::gl_pow(wN, c));
        uint64_t v = zk::gl_pow(base, j0);
        for (uint32_t i = 0; i < COSET_RUN && j0 + i < n; i++) {
            tab[c * n + j0 + i] = v;
            v = zk::gl_mul(v, base);
        }
    }
}

uint64_t *tw_table(NoAllocState &st, uint32_t k) { return st.twiddles + ((1ULL << k) - 1); }

unsigned grid_for(uint64_t items) { return (unsigned)((items + 255) / 256 < 1024 ? (items + 255) / 256 : 1024); }

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
        // each term on its own first, so the sum below cannot wrap
        if (rate_bits > NOALLOC_MAX_LG || lg_n > NOALLOC_MAX_LG - rate_bits)
            throw zk::arg_failure("zeknox_lde_rows_noalloc: lg_n = " + std::to_string(lg_n) + " with rate_bits = " +
                                  std::to_string(rate_bits) + " exceeds the static limit lg_n + rate_bits <= " +
                                  std::to_string(NOALLOC_MAX_LG));
        if (!rows || !coeffs) throw zk::arg_failure("null buffer");
        if (device_id >= (size_t)NOALLOC_MAX_DEVICES) throw zk::arg_failure("device id out of range");
        int ndev = 0;
        check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (device_id >= (size_t)ndev) throw zk::arg_failure("invalid device id");
        check(cudaSetDevice((int)device_id), "cudaSetDevice");
        // an error left by earlier, unrelated work is reported as such (and
        // left pending for its owner) rather than taken for one of ours
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess)
            throw zk::cuda_failure(-(int)pending, std::string("zeknox_lde_rows_noalloc: a CUDA error from earlier work "
                                                              "is pending: ") + cudaGetErrorString(pending));
        cudaStream_t s = (cudaStream_t)stream;  // NULL: the legacy default stream
        const uint64_t gen = (coset_gen ? coset_gen : ZK_GENERATOR) % zk::GL_P;

        std::lock_guard<std::mutex> lk(g_mu);
        NoAllocState &st = g_state[device_id];
        if (!st.ready) {
            // one-time set-up on this device (with it current): device
            // addresses of the file-scope arrays, then every twiddle table the
            // size limit can use, finished before the call goes on
            NoAllocState t;
            check(cudaGetSymbolAddress((void **)&t.scratch, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
            check(cudaGetSymbolAddress((void **)&t.twiddles, g_noalloc_twiddles), "cudaGetSymbolAddress(twiddles)");
            check(cudaGetSymbolAddress((void **)&t.coset, g_noalloc_coset), "cudaGetSymbolAddress(coset)");
            for (uint32_t k = 0; k <= NOALLOC_MAX_LG; k++) {
                noalloc_powers<<<grid_for(1ULL << k), 256, 0, s>>>(tw_table(t, k), 1ULL << k, H_OMEGA[k]);
                check(cudaGetLastError(), "twiddle table");
            }
            check(cudaStreamSynchronize(s), "twiddle tables");
            t.ready = true;
            st = t;
        }
        const uint64_t *tw[33] = {};
        for (uint32_t k = 0; k <= NOALLOC_MAX_LG; k++) tw[k] = tw_table(st, k);
        // this call's coset table, queued ahead of its transform
        const uint64_t n = 1ULL << lg_n;
        noalloc_coset_powers<<<grid_for(((n + COSET_RUN - 1) / COSET_RUN) << rate_bits), 256, 0, s>>>(
            st.coset, n, 1u << rate_bits, gen, H_OMEGA[lg_n + rate_bits]);
        check(cudaGetLastError(), "coset table");
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

namespace zk {
cudaError_t oob_take_noalloc(uint64_t r[4]) { return oob_take_local(r); }
}  // namespace zk
