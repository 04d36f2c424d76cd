// batch.cuh -- one commit as a stream of launches, and batches of commits as
// one CUDA graph.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/zeknox_b200.h"
#include "runtime.cuh"

namespace zk {

void check_job(const zk_commit_job &j);

// Words of scratch commit_enqueue needs for a job of this shape.
uint64_t commit_scratch_words(uint32_t lg_n, uint32_t rate_bits, uint32_t cols, bool values, bool host_input = false);

// True when p is host memory (pinned or pageable).
bool is_host_pointer(const void *p);
// False for pageable host memory when device `dev` cannot read pageable memory
// (no HMM / ATS): kernels that read such a pointer directly would fault.
bool device_can_read(const void *p, int dev);

// Queue one commit on `s` using `scratch` (commit_scratch_words words, may be
// null when that is 0).  Allocates nothing and never synchronises, so it can be
// recorded into a CUDA graph once prepare_job() has built the tables it reads.
// host_input: j.input is host memory, staged through the scratch chunk by chunk.
void commit_enqueue(DeviceCtx &c, const zk_commit_job &j, cudaStream_t s, uint64_t *scratch, bool host_input = false);
void prepare_job(DeviceCtx &c, const zk_commit_job &j);

// Run a batch of commits: the launches of every job are recorded once into a
// CUDA graph whose branches run jobs concurrently (jobs assigned to branches by
// size), the graph is cached under the batch's shape and buffer addresses and
// replayed on later calls with the same key.
void commit_batch_graph(DeviceCtx &c, const zk_commit_job *jobs, uint32_t njobs);
void merkle_batch_graph(DeviceCtx &c, const zk_merkle_job *jobs, uint32_t njobs);

}  // namespace zk
