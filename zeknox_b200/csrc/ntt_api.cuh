// ntt_api.cuh -- host-side entry points of the NTT engine (used by abi.cu).
#pragma once
#include <stdint.h>

#include <utility>
#include <vector>

#include "ntt_args.h"
#include "runtime.cuh"

namespace zk {

// compute_batched_ntt on device memory: natural order in and out, in place.
// `scratch` (n * batches words) may be null: then it comes from the stream-ordered pool.
void ntt_batch_device(DeviceCtx &c, uint64_t *inout, uint32_t lg, uint64_t batches, bool inverse, bool with_coset,
                      uint64_t *scratch = nullptr);

// compute_batched_lde on device memory: column-major natural-order evaluations.
void lde_batch_device(DeviceCtx &c, uint64_t *out, const uint64_t *in, uint32_t lg_n, uint32_t rate, uint64_t batches,
                      bool inverse, bool with_coset);

// Fused LDE + bit-reverse + transpose: rows[r * cols + b] = LDE_b[rev_{lg_n+rate}(r)]
// (the leaf-major matrix compute_transpose_rev would produce).  `scratch` may
// be null (allocated on the stream) or hold lde_rows_scratch_elems() words.
// When host_coeffs is non-null the coefficients are read from that host
// memory, staged chunk by chunk into `coeffs` (a device buffer of cols * 2^lg_n
// words) on the context's copy stream, overlapping the transfer with the
// transform of the previous chunk.
// Row output spread over several buffers: row r of the LDE goes to
// dst_tab[r >> log_rows_per_dst] (a device array of base pointers, which may
// be other GPUs' memory mapped for peer access) at row r mod 2^log_rows_per_dst,
// columns [col_offset, col_offset + cols) of rows that are row_stride words long.
struct RowScatter {
    uint64_t *const *dst_tab;
    uint32_t log_rows_per_dst;
    uint64_t col_offset;
    uint64_t row_stride;
};

void lde_rows_device(DeviceCtx &c, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n, uint32_t rate, uint64_t cols,
                     uint64_t coset_gen, uint64_t *scratch, const uint64_t *host_coeffs = nullptr,
                     const RowScatter *scatter = nullptr);
uint64_t lde_rows_scratch_elems(uint32_t lg_n, uint32_t rate, uint64_t cols);
uint32_t lde_rows_chunk_cols(uint32_t lg_n, uint32_t rate, uint64_t cols);

// The fused LDE with caller-provided tables and scratch (no allocation, no
// DeviceCtx): tw[lg] = w_{2^lg}^t tables for lg 12 and every pass's lg M,
// lde_tab = (g * w_N^c)^j, scratch = 2^(lg_n+rate) * chunk_cols words when
// the size needs more than one pass.  Launches on `stream`.
void lde_rows_explicit(cudaStream_t stream, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n, uint32_t rate,
                       uint64_t cols, const uint64_t *lde_tab, const uint64_t *const *tw, uint64_t *scratch,
                       uint64_t chunk_cols);
std::vector<std::pair<uint32_t, uint32_t>> lde_rows_passes(uint32_t lg_n);

// The fused LDE's passes as data (the persistent serving loop runs them):
// every pass of every column chunk with its arguments, tile count and kernel
// shape (radix, load and store modes, direct first sub-step), the row-output
// pass at radix 2^8.  The tables must be resident (lde_rows_plan_tables, on a
// stream no persistent kernel occupies); `scratch` as for lde_rows_device.
struct PlannedPass {
    NttPassArgs a;
    uint64_t grid;
    uint32_t logr;
    int load, store, direct;
    int inv;  // inverse roots
};
// The bit-reversal reorder after a column-output transform, as data.
struct PlannedReorder {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t src_stride, dst_stride;
    uint32_t lg_t, rate;
    uint64_t cols, mul, src_len, dst_len, blocks;
};
bool lde_rows_plan_tables_resident(DeviceCtx &c, uint32_t lg_n, uint32_t rate, uint64_t coset_gen);
void lde_rows_plan_tables(DeviceCtx &c, uint32_t lg_n, uint32_t rate, uint64_t coset_gen);
std::vector<PlannedPass> lde_rows_plan(DeviceCtx &c, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n,
                                       uint32_t rate, uint64_t cols, uint64_t coset_gen, uint64_t *scratch);

// compute_batched_ntt's inverse (no coset) on device memory as data: the
// passes of ntt_batch_device into `scratch` (n * batches words) and the
// reorder back into `inout` with the factor n^-1.  Its tables must be
// resident (ntt_inverse_plan_tables).
bool ntt_inverse_plan_tables_resident(DeviceCtx &c, uint32_t lg);
void ntt_inverse_plan_tables(DeviceCtx &c, uint32_t lg);
std::vector<PlannedPass> ntt_inverse_plan(DeviceCtx &c, uint64_t *inout, uint32_t lg, uint64_t batches,
                                          uint64_t *scratch, PlannedReorder &reorder);

// Build every table a commit of this shape uses (before graph capture).
void prepare_tables(DeviceCtx &c, uint32_t lg_n, uint32_t rate, uint64_t coset_gen, bool values);

void transpose_rev_device(DeviceCtx &c, uint64_t *out, const uint64_t *in, uint32_t lg, uint64_t cols);

void salt_device(DeviceCtx &c, uint64_t *out, uint64_t count);

// Merkle forest on device memory, launched on `stream`; returns false (with a
// message in err) on invalid geometry or an unsupported hash.
bool merkle_device(uint64_t *digests, uint64_t *caps, const uint64_t *leaves, uint64_t n_digests, uint64_t n_caps,
                   uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height, uint64_t hash_type, cudaStream_t stream,
                   std::string &err);

bool merkle_geometry_ok(uint64_t n_digests, uint64_t n_caps, uint64_t n_leaves, uint64_t cap_height, std::string &err);

}  // namespace zk
