// bounds.cuh -- compiled-in range checks of the kernels' global-memory
// accesses, for the checked build (`make -C zeknox_b200 checked`, which
// defines ZK_BOUNDS_CHECK and writes libzeknox_checked.so).
//
// In the checked build every instrumented load or store first tests its index
// against the extent of the buffer it addresses.  An index out of range is not
// accessed: the kernel counts it, records the first one (site, index, extent)
// in a device word of its translation unit, and goes on -- no trap, no fault,
// the context stays usable.  zeknox_bounds_report() collects and clears the
// records.  In the normal build ZK_IN_BOUNDS is the constant true and the
// checks compile away.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace zk {

// Access sites named in the records.
enum OobSite : uint32_t {
    OOB_NTT_SRC = 1,        // a pass's source load
    OOB_NTT_TAB = 2,        // a pass's coset / scale table load
    OOB_NTT_DST = 3,        // a pass's column-output store
    OOB_NTT_ROWS = 4,       // a pass's leaf-row store
    OOB_NTT_SCATTER = 5,    // a leaf-row store into one of several destination buffers
    OOB_NTT_TWIDDLE = 6,    // a pass twiddle load
    OOB_REORDER_SRC = 7,
    OOB_REORDER_DST = 8,
    OOB_TRANSPOSE_IN = 9,
    OOB_TRANSPOSE_OUT = 10,
    OOB_MERKLE_LEAF = 11,   // a leaf row read by the sponge (its last word)
    OOB_MERKLE_DIGEST = 12, // a digest store
    OOB_MERKLE_CAP = 13,    // a cap store
    OOB_MERKLE_NODE = 14,   // a stored digest read back by the upper levels
};

#if defined(ZK_BOUNDS_CHECK) && defined(__CUDACC__)
// count of out-of-range accesses, then site, index and extent of the first
static __device__ unsigned long long g_zk_oob[4];

__device__ __forceinline__ bool in_bounds(uint64_t idx, uint64_t extent, uint32_t site)
{
    if (idx < extent) return true;
    if (atomicAdd(&g_zk_oob[0], 1ULL) == 0) {
        g_zk_oob[1] = site;
        g_zk_oob[2] = idx;
        g_zk_oob[3] = extent;
    }
    return false;
}
#define ZK_IN_BOUNDS(idx, extent, site) (::zk::in_bounds((uint64_t)(idx), (uint64_t)(extent), (uint32_t)(site)))

// this translation unit's record, read and cleared on the current device
static inline cudaError_t oob_take_local(uint64_t r[4])
{
    cudaError_t e = cudaMemcpyFromSymbol(r, g_zk_oob, 4 * sizeof(uint64_t));
    if (e != cudaSuccess) return e;
    const uint64_t z[4] = {0, 0, 0, 0};
    return cudaMemcpyToSymbol(g_zk_oob, z, 4 * sizeof(uint64_t));
}
constexpr bool BOUNDS_CHECKED = true;
#else
#define ZK_IN_BOUNDS(idx, extent, site) (true)
static inline cudaError_t oob_take_local(uint64_t r[4])
{
    r[0] = r[1] = r[2] = r[3] = 0;
    return cudaSuccess;
}
constexpr bool BOUNDS_CHECKED = false;
#endif

// the records of the translation units that hold kernels (ntt.cu, merkle.cu,
// noalloc.cu), read and cleared on the current device
cudaError_t oob_take_ntt(uint64_t r[4]);
cudaError_t oob_take_merkle(uint64_t r[4]);
cudaError_t oob_take_noalloc(uint64_t r[4]);

}  // namespace zk
