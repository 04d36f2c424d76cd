// multi_split.h -- how the in-process multi-GPU entry points divide work.
//
// compute_batched_lde_multi_gpu: columns are independent; GPU g of G takes
// batches / G columns, and the first batches % G GPUs one more, in order
// (native/ntt/ntt.cu:324-337).
// fill_digests_buf_linear_multigpu_with_gpu_ptr: subtrees are independent; the
// largest power of two of GPUs that is at most the GPU count and the cap count
// each build a contiguous run of caps / G whole subtrees (the reference does
// one subtree per GPU, native/merkle/merkle.cu:381-438).
// Host-only (no CUDA types), so a CPU test compiles it on its own.
#pragma once
#include <stdint.h>

#include <vector>

namespace zk {

struct ColumnSplit {
    std::vector<uint64_t> take, first;  // per GPU: column count, first column
};

inline ColumnSplit split_columns(uint64_t batches, uint32_t gpus)
{
    ColumnSplit s;
    uint64_t acc = 0;
    for (uint32_t g = 0; g < gpus; g++) {
        const uint64_t t = batches / gpus + (g < batches % gpus ? 1 : 0);
        s.take.push_back(t);
        s.first.push_back(acc);
        acc += t;
    }
    return s;
}

inline uint64_t merkle_gpu_count(uint64_t gpus, uint64_t n_caps)
{
    uint64_t g = 1;
    while (g * 2 <= gpus && g * 2 <= n_caps) g *= 2;
    return g;
}

}  // namespace zk
