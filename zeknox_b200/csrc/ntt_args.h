// ntt_args.h -- the arguments of one NTT pass (shared by the kernels in
// ntt.cuh and the host code that plans passes).
#pragma once
#include <stdint.h>

namespace zk {

enum NttLoad : int {
    LOAD_PLAIN = 0,      // src[v * src_stride + j]
    LOAD_SCALE = 1,      // src[v * src_stride + j] * tab[j]              (coset powers g^j)
    LOAD_COSETS = 2,     // src[(v >> rate) * src_stride + j] * tab[(v & (2^rate-1)) * n + j]
    LOAD_EXTEND = 3,     // j < n_src ? src[v * src_stride + j] : 0        (zero-extended transform)
};

enum NttStore : int {
    STORE_SAME = 0,      // dst[v * dst_stride + position]
    STORE_ROWS = 1,      // leaf-major: dst[(rev_rate(v & mask) * n + position) * cols + (v >> rate)]
};

struct NttPassArgs {
    const uint64_t *src;
    uint64_t *dst;
    const uint64_t *tab;      // LOAD_SCALE / LOAD_COSETS / LOAD_EXTEND_SCALE table
    const uint64_t *tw_pass;  // w_M^t, t < M   (M = R * S); unused when S == 1
    const uint64_t *tw_small; // w_4096^t, t < 4096 (inverse roots for INV)
    uint64_t src_stride;      // elements between consecutive source columns
    uint64_t dst_stride;
    uint64_t n_src;           // LOAD_EXTEND: nonzero prefix length
    uint64_t vcols;           // virtual columns
    uint32_t L;               // log2 transform size
    uint32_t s_lo;            // lowest stage of this pass
    uint32_t rate;            // LOAD_COSETS / STORE_ROWS: log2 cosets per column
    uint32_t cols;            // STORE_ROWS: real columns in this launch
    uint64_t row_stride;      // STORE_ROWS: words per output row (>= cols; dst points at the first column)
    // STORE_ROWS scattered over destination buffers (null: one buffer, dst):
    // row r goes to dst_tab[r >> log_rows_per_dst] at row r & (2^log_rows_per_dst - 1),
    // column col_offset + b -- the buffers may be other GPUs' memory (P2P stores)
    uint64_t *const *dst_tab;
    uint32_t log_rows_per_dst;
    uint64_t col_offset;
    // extents in words of src, dst (each destination buffer for dst_tab) and
    // tab from the pass's first element on: read only by the checked build
    uint64_t src_len, dst_len, tab_len;
};

}  // namespace zk
