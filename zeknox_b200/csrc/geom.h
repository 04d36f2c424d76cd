// geom.h -- argument checks shared by the GPU and CPU Merkle builders.
#pragma once
#include <stdint.h>

#include <string>

namespace zk {

inline uint32_t log2_pow2(uint64_t x)
{
    if (x == 0 || (x & (x - 1))) return ~0u;
    uint32_t l = 0;
    while ((1ULL << l) < x) l++;
    return l;
}

// The linear layout needs 2^cap_height subtrees of a power-of-two number of
// leaves each and 2 * (leaves - caps) digest slots
// (native/merkle/merkle.cu:185-191 asserts the same relations).
inline bool merkle_geometry_check(uint64_t n_digests, uint64_t n_caps, uint64_t n_leaves, uint64_t cap_height,
                                  std::string &err)
{
    if (n_leaves == 0) {
        err = "no leaves";
        return false;
    }
    if (cap_height >= 63 || n_caps != (1ULL << cap_height)) {
        err = "cap_buf_size must be 2^cap_height";
        return false;
    }
    if (n_caps > n_leaves || n_leaves % n_caps) {
        err = "leaves_buf_size must be a multiple of cap_buf_size";
        return false;
    }
    if (log2_pow2(n_leaves / n_caps) == ~0u) {
        err = "leaves per subtree must be a power of two";
        return false;
    }
    if (n_digests != 2 * (n_leaves - n_caps)) {
        err = "digests_buf_size must be 2 * (leaves_buf_size - cap_buf_size)";
        return false;
    }
    return true;
}

}  // namespace zk
