// ntt.cu -- host drivers of the batched NTT / LDE / transpose.
//
// Semantics follow zeknox native/ntt/ntt.cu (batch_ntt :253-309, batch_lde
// :477-564, compute_transpose_rev :182-226); the execution plan is this
// project's: a handful of multi-stage DIF passes (ntt.cuh) plus one tiled
// reorder, instead of one HBM pass per radix-2 stage.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "ntt.cuh"
#include "ntt_api.cuh"
#include "runtime.cuh"
#include "zk_constants.h"

namespace zk {

static const uint64_t H_SIZE_INV[33] = {ZK_DOMAIN_SIZE_INV_LIST};
static const uint64_t H_OMEGA_N[33] = {ZK_OMEGA_LIST};

static constexpr int PASS_NT = 256;
static constexpr int PASS_TILE = 4096;  // 32 KiB of shared memory; measured 1.07-1.14x over 512 x 8192
static constexpr uint32_t LOG_PASS_TILE = __builtin_ctz(PASS_TILE);
static constexpr uint32_t MAX_SPLIT_LOGR = LOG_PASS_TILE - 2;  // passes before the last (see plan_passes)
static constexpr uint32_t MAX_ROWS_LOGR = LOG_PASS_TILE - 4;   // row-output passes: 16 columns x 2^LOGR
static constexpr uint32_t COL_SPLIT_LOGR = 9;  // largest pass of a multi-pass column-output transform

// ------------------------------------------------------------- pass dispatch

template <int LOGR, int INV, int LOADM, int STOREM, int DIRECT>
static void launch_one(const NttPassArgs &a, uint64_t grid, uint32_t smem, cudaStream_t s)
{
    auto k = ntt_pass_kernel<LOGR, INV, PASS_NT, PASS_TILE, LOADM, STOREM, DIRECT>;
    // the 64 KiB dynamic shared-memory opt-in is per device
    static std::atomic<uint64_t> attr_set{0};
    int dev = 0;
    ZK_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = 1ULL << (dev & 63);
    if (!(attr_set.load(std::memory_order_relaxed) & bit)) {
        ZK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, PASS_TILE * 8));
        ZK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
        attr_set.fetch_or(bit, std::memory_order_relaxed);
    }
    k<<<(unsigned)grid, PASS_NT, smem, s>>>(a);
    note_launch();
}

// Whether a pass reads its first sub-step (and, for STORE_SAME, writes its
// last) straight between global memory and registers: only where a warp's
// accesses then stay sector-complete -- row tiles of at least 8 consecutive
// positions per task, or STORE_SAME tiles that are runs of >= 4 consecutive
// offsets.
static bool direct_io(uint32_t logr, const NttPassArgs &a, bool rows)
{
    if (rows) return logr >= 7;
    const uint32_t log_tile = std::min<uint32_t>(a.L, __builtin_ctz(PASS_TILE));
    if (log_tile < logr) return false;
    const uint32_t log_g = log_tile - logr;
    return a.s_lo >= log_g && log_g >= 2;
}

template <int INV, int LOADM, int STOREM>
static void launch_pass(uint32_t logr, const NttPassArgs &a, uint64_t grid, uint32_t smem, cudaStream_t s)
{
    const bool direct = direct_io(logr, a, STOREM == STORE_ROWS);
    // row-output passes never exceed MAX_ROWS_LOGR (plan_passes): no kernels above it
#define ZK_R(r) ((STOREM == STORE_ROWS && (r) > (int)MAX_ROWS_LOGR) ? (int)MAX_ROWS_LOGR : (r))
#define ZK_CASE(r)                                                                       \
    case r:                                                                              \
        if (direct) launch_one<ZK_R(r), INV, LOADM, STOREM, 1>(a, grid, smem, s);        \
        else launch_one<ZK_R(r), INV, LOADM, STOREM, 0>(a, grid, smem, s);               \
        break;
    switch (logr) {
        ZK_CASE(1) ZK_CASE(2) ZK_CASE(3) ZK_CASE(4) ZK_CASE(5) ZK_CASE(6)
        ZK_CASE(7) ZK_CASE(8) ZK_CASE(9) ZK_CASE(10) ZK_CASE(11) ZK_CASE(12)
    default: throw arg_failure("bad pass radix");
    }
#undef ZK_CASE
#undef ZK_R
}

struct Pass {
    uint32_t s_lo, logr;
};

// Split L stages into passes.  A pass of 2^LOGR points on a tile of 2^LT
// elements holds 2^(LT - LOGR) groups; passes other than the last are kept to
// LOGR <= LT - 2 so a tile's rows are runs of >= 4 consecutive offsets (whole
// 32-byte sectors); a row-output pass spans at most 2^(LT - 4) positions of 16
// columns.  Single-pass transforms may use the whole tile.

static std::vector<Pass> plan_passes_last(uint32_t L, bool rows, uint32_t last_rows, uint32_t split_logr = 0)
{
    std::vector<uint32_t> sizes;
    last_rows = last_rows < 1 ? 1 : (last_rows > MAX_ROWS_LOGR ? MAX_ROWS_LOGR : last_rows);
    // column output: one pass up to the whole tile, else passes of at most
    // 2^COL_SPLIT_LOGR points -- or, with split_logr set (knob
    // ntt_split_logr), passes of at most 2^split_logr points whatever the
    // size.  Radix-2^10 passes are the slowest per stage: at 2^19 and 2^20
    // points three passes beat two (measured on B200: column LDE 8.90 -> 8.05
    // ms for 64 columns x 2^19 at rate 3, NTT 7.24 -> 7.09 ms for 512 x 2^19).
    const uint32_t split = split_logr ? (split_logr < MAX_SPLIT_LOGR ? split_logr : MAX_SPLIT_LOGR) : COL_SPLIT_LOGR;
    const uint32_t last_max = rows ? last_rows : (split_logr ? split : LOG_PASS_TILE);
    if (L <= last_max) {
        sizes.push_back(L);
    } else if (!rows) {
        uint32_t np = (L + split - 1) / split;
        for (uint32_t i = 0; i < np; i++) sizes.push_back(L / np + (i < L % np ? 1 : 0));
    } else {
        uint32_t rem = L - last_rows;
        uint32_t np = (rem + MAX_SPLIT_LOGR - 1) / MAX_SPLIT_LOGR;
        for (uint32_t i = 0; i < np; i++) sizes.push_back(rem / np + (i < rem % np ? 1 : 0));
        sizes.push_back(last_rows);
    }
    std::vector<Pass> p;
    uint32_t hi = L;
    for (uint32_t k : sizes) {
        hi -= k;
        p.push_back({hi, k});
    }
    return p;
}

// The last pass of a row-output transform has radix 2^lde_last_logr (tuned).
static std::vector<Pass> plan_passes(uint32_t L, bool rows)
{
    return plan_passes_last(L, rows, (uint32_t)tune_get("lde_last_logr", L, MAX_ROWS_LOGR),
                            rows ? 0 : (uint32_t)tune_get("ntt_split_logr", L, 0));
}

// Batched DIF over `vcols` virtual columns of size 2^L; output in bit-reversed
// order, either in vcol-major layout at dst (stride dst_stride) or, for
// rows=true, as leaf rows (see STORE_ROWS).  `scratch` (vcols * 2^L words) is
// needed only when rows=true and there is more than one pass.
struct DifJob {
    const uint64_t *src;
    uint64_t src_stride;
    int load;                 // NttLoad of the first pass
    const uint64_t *tab;
    uint64_t n_src;
    uint64_t *dst;
    uint64_t dst_stride;
    uint64_t vcols;
    uint32_t L;
    uint32_t rate;
    uint32_t cols;
    uint64_t row_stride;
    bool rows;
    bool inverse;
    uint64_t *scratch;
    const RowScatter *scatter;  // row output over several buffers (null: dst)
    uint64_t col0;              // first column of this chunk (scattered row output)
    // extents in words of src, dst (each scatter destination), tab and
    // scratch, read only by the checked build's range checks
    uint64_t src_len, dst_len, tab_len, scratch_len;
};

static void run_dif(DeviceCtx &c, const DifJob &j)
{
    if (j.L == 0) {
        // size-1 transform: copy (with scaling) -- handled by the caller's reorder
        throw arg_failure("zero-size transform");
    }
    auto passes = plan_passes(j.L, j.rows);
    const uint64_t n = 1ULL << j.L;
    const uint64_t *tw_small = c.twiddles(12, j.inverse);
    for (size_t pi = 0; pi < passes.size(); pi++) {
        const Pass &ps = passes[pi];
        const bool first = pi == 0, last = pi + 1 == passes.size();
        NttPassArgs a{};
        a.src = first ? j.src : (j.rows ? j.scratch : j.dst);
        a.src_len = first ? j.src_len : (j.rows ? j.scratch_len : j.dst_len);
        a.tab_len = j.tab_len;
        a.src_stride = first ? j.src_stride : (j.rows ? n : j.dst_stride);
        a.tab = j.tab;
        a.n_src = j.n_src;
        a.tw_small = tw_small;
        a.tw_pass = ps.s_lo ? c.twiddles(ps.s_lo + ps.logr, j.inverse) : nullptr;
        a.vcols = j.vcols;
        a.L = j.L;
        a.s_lo = ps.s_lo;
        a.rate = j.rate;
        a.cols = j.cols;
        a.row_stride = j.row_stride;
        const bool store_rows = j.rows && last;
        if (store_rows) {
            a.dst = j.dst;
            a.dst_stride = 0;
            a.dst_len = j.dst_len;
            if (j.scatter) {
                a.dst_tab = j.scatter->dst_tab;
                a.log_rows_per_dst = j.scatter->log_rows_per_dst;
                a.col_offset = j.scatter->col_offset + j.col0;
            }
        } else {
            a.dst = j.rows ? j.scratch : j.dst;
            a.dst_stride = j.rows ? n : j.dst_stride;
            a.dst_len = j.rows ? j.scratch_len : j.dst_len;
        }
        const int load = first ? j.load : LOAD_PLAIN;
        if (store_rows && ps.logr > MAX_ROWS_LOGR) throw arg_failure("row-output pass radix above the tile");
        uint64_t grid;
        uint32_t tile;
        if (store_rows) {
            uint32_t W = (uint32_t)std::min<uint64_t>(n, PASS_TILE / 16);
            tile = 16 * W;
            uint64_t ncg = (j.cols + 15) / 16;
            grid = (n / W) * ncg * (1ULL << j.rate);
        } else {
            tile = (uint32_t)std::min<uint64_t>(n, PASS_TILE);
            grid = j.vcols * (n / tile);
        }
        if (grid == 0) continue;
        if (grid > 0x7FFFFFFFULL) throw arg_failure("transform batch too large for one launch");
        const uint32_t smem = tile * 8;
        if (!j.inverse) {
            if (store_rows) {
                if (load == LOAD_COSETS) launch_pass<0, LOAD_COSETS, STORE_ROWS>(ps.logr, a, grid, smem, c.stream);
                else launch_pass<0, LOAD_PLAIN, STORE_ROWS>(ps.logr, a, grid, smem, c.stream);
            } else {
                if (load == LOAD_COSETS) launch_pass<0, LOAD_COSETS, STORE_SAME>(ps.logr, a, grid, smem, c.stream);
                else if (load == LOAD_SCALE) launch_pass<0, LOAD_SCALE, STORE_SAME>(ps.logr, a, grid, smem, c.stream);
                else launch_pass<0, LOAD_PLAIN, STORE_SAME>(ps.logr, a, grid, smem, c.stream);
            }
        } else {
            if (store_rows) throw arg_failure("inverse transform with row output is not supported");
            if (load == LOAD_EXTEND) launch_pass<1, LOAD_EXTEND, STORE_SAME>(ps.logr, a, grid, smem, c.stream);
            else launch_pass<1, LOAD_PLAIN, STORE_SAME>(ps.logr, a, grid, smem, c.stream);
        }
        ZK_CUDA(cudaGetLastError());
    }
}

// bit-reversed (per virtual column) -> natural, with factor mul and optional table
static void reorder(DeviceCtx &c, const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                    uint32_t lg_t, uint32_t rate, uint64_t cols, uint64_t mul, const uint64_t *tab, uint64_t src_len,
                    uint64_t dst_len)
{
    const uint32_t a = lg_t >= 10 ? 5 : lg_t / 2;
    const uint64_t blocks = cols * (1ULL << (lg_t - 2 * a)) * (1ULL << rate);
    if (blocks > 0x7FFFFFFFULL) throw arg_failure("reorder too large for one launch");
    bitrev_reorder_kernel<<<(unsigned)blocks, 256, 0, c.stream>>>(src, dst, src_stride, dst_stride, lg_t, rate, cols, mul,
                                                                  tab, src_len, dst_len);
    note_launch();
    ZK_CUDA(cudaGetLastError());
}

// --------------------------------------------------------------- public ops

void ntt_batch_device(DeviceCtx &c, uint64_t *inout, uint32_t lg, uint64_t batches, bool inverse, bool with_coset,
                      uint64_t *scratch)
{
    NvtxRange range("zeknox ntt");
    const uint64_t n = 1ULL << lg;
    if (batches == 0) return;
    DevBuf tmp;
    if (scratch) {
        tmp.p = nullptr;
    } else {
        tmp.ctx = &c;
        tmp.p = c.alloc(n * batches * 8);
    }
    uint64_t *tp = scratch ? scratch : tmp.p;
    if (!inverse) {
        DifJob j{};
        j.src = inout;
        j.src_stride = n;
        j.load = with_coset ? LOAD_SCALE : LOAD_PLAIN;
        j.tab = with_coset ? c.coset_powers(lg) : nullptr;
        j.dst = tp;
        j.dst_stride = n;
        j.vcols = batches;
        j.L = lg;
        j.src_len = j.dst_len = n * batches;
        j.tab_len = n;
        run_dif(c, j);
        reorder(c, tp, n, inout, n, lg, 0, batches, 1, nullptr, n * batches, n * batches);
    } else {
        DifJob j{};
        j.src = inout;
        j.src_stride = n;
        j.load = LOAD_PLAIN;
        j.dst = tp;
        j.dst_stride = n;
        j.vcols = batches;
        j.L = lg;
        j.inverse = true;
        j.src_len = j.dst_len = n * batches;
        run_dif(c, j);
        // reference order: coset multiply (forward powers) then n^-1 (ntt.cu:137-143)
        reorder(c, tp, n, inout, n, lg, 0, batches, H_SIZE_INV[lg], with_coset ? c.coset_powers(lg) : nullptr,
                n * batches, n * batches);
    }
}

void lde_batch_device(DeviceCtx &c, uint64_t *out, const uint64_t *in, uint32_t lg_n, uint32_t rate, uint64_t batches,
                      bool inverse, bool with_coset)
{
    NvtxRange range("zeknox lde");
    const uint64_t n = 1ULL << lg_n;
    const uint32_t lgN = lg_n + rate;
    const uint64_t N = 1ULL << lgN;
    if (batches == 0) return;
    DevBuf tmp(c, N * batches);
    if (!inverse) {
        // coset c of column b is virtual column b*2^rate + c of size n
        const uint64_t g = with_coset ? (c.coset_powers(0), c.coset_gen) : 1;
        DifJob j{};
        j.src = in;
        j.src_stride = n;
        j.load = LOAD_COSETS;
        j.tab = c.lde_table(lg_n, rate, g);
        j.dst = tmp.p;
        j.dst_stride = n;
        j.vcols = batches << rate;
        j.L = lg_n;
        j.rate = rate;
        j.src_len = n * batches;
        j.tab_len = N;
        j.dst_len = N * batches;
        run_dif(c, j);
        reorder(c, tmp.p, n, out, N, lg_n, rate, batches, 1, nullptr, N * batches, N * batches);
    } else {
        // zero-extended inverse transform of size N (ntt.cu:529-535)
        DifJob j{};
        j.src = in;
        j.src_stride = n;
        j.load = LOAD_EXTEND;
        j.n_src = n;
        j.dst = tmp.p;
        j.dst_stride = N;
        j.vcols = batches;
        j.L = lgN;
        j.inverse = true;
        j.src_len = n * batches;
        j.dst_len = N * batches;
        run_dif(c, j);
        reorder(c, tmp.p, N, out, N, lgN, 0, batches, H_SIZE_INV[lgN], with_coset ? c.coset_powers(lgN) : nullptr,
                N * batches, N * batches);
    }
}

// Columns per chunk of the fused LDE: the intermediate of a chunk (2^(lg_n +
// rate) words per column) is kept within lde_chunk_mib MiB, which bounds the
// scratch whatever the job size.  A multiple of the 16-column row tile.
// Larger chunks are faster: the intermediate does not stay in the 126 MB L2
// anyway (the streaming row output shares it), and fewer, larger launches
// lose less to their last partial wave (256 x 2^15 at rate 3: 1.21 ms in one
// chunk against 1.32 ms in 48-column chunks).  Inputs in host memory use
// lde_host_chunk_mib instead: there each chunk's copy overlaps the transform of
// the one before, so a whole-input chunk would expose the whole copy.
static constexpr uint64_t ZK_CHUNK_MIB = 512;       // default; the autotuner may set "lde_chunk_mib"
static constexpr uint64_t ZK_HOST_CHUNK_MIB = 96;   // "lde_host_chunk_mib"

static uint32_t chunk_cols_for(uint64_t mib, uint32_t lg_n, uint32_t rate, uint64_t cols)
{
    const uint64_t per_col = 8ULL << (lg_n + rate);
    uint64_t c = (mib << 20) / per_col;
    c = c < 16 ? 16 : (c / 16) * 16;
    return (uint32_t)(c < cols ? c : ((cols + 15) / 16) * 16);
}

uint32_t lde_rows_chunk_cols(uint32_t lg_n, uint32_t rate, uint64_t cols)
{
    return chunk_cols_for(tune_get("lde_chunk_mib", lg_n + rate, ZK_CHUNK_MIB), lg_n, rate, cols);
}

// ------------------------------------------------- explicit-table variant
//
// The same passes as run_dif / lde_rows_device for the fused LDE, with every
// table and the scratch passed in by the caller and no DeviceCtx involved (no
// lazy table builds, no pool allocations).  tw[lg] must hold w_{2^lg}^t,
// t < 2^lg, for lg = 12 and every pass's lg M.
void lde_rows_explicit(cudaStream_t stream, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n, uint32_t rate,
                       uint64_t cols, const uint64_t *lde_tab, const uint64_t *const *tw, uint64_t *scratch,
                       uint64_t chunk_cols)
{
    const uint64_t n = 1ULL << lg_n;
    const auto passes = plan_passes(lg_n, true);
    for (uint64_t c0 = 0; c0 < cols; c0 += chunk_cols) {
        const uint64_t cc = cols - c0 < chunk_cols ? cols - c0 : chunk_cols;
        for (size_t pi = 0; pi < passes.size(); pi++) {
            const Pass &ps = passes[pi];
            const bool first = pi == 0, last = pi + 1 == passes.size();
            NttPassArgs a{};
            a.src = first ? coeffs + c0 * n : scratch;
            a.src_stride = n;
            a.tab = lde_tab;
            a.tw_small = tw[12];
            a.tw_pass = ps.s_lo ? tw[ps.s_lo + ps.logr] : nullptr;
            a.vcols = cc << rate;
            a.L = lg_n;
            a.s_lo = ps.s_lo;
            a.rate = rate;
            a.cols = (uint32_t)cc;
            a.row_stride = cols;
            a.dst = last ? rows + c0 : scratch;
            a.dst_stride = n;
            a.src_len = first ? (cols - c0) * n : (n << rate) * chunk_cols;
            a.dst_len = last ? (n << rate) * cols - c0 : (n << rate) * chunk_cols;
            a.tab_len = n << rate;
            uint64_t grid;
            uint32_t tile;
            if (last) {
                const uint32_t W = (uint32_t)std::min<uint64_t>(n, PASS_TILE / 16);
                tile = 16 * W;
                grid = (n / W) * ((cc + 15) / 16) * (1ULL << rate);
                if (first) launch_pass<0, LOAD_COSETS, STORE_ROWS>(ps.logr, a, grid, tile * 8, stream);
                else launch_pass<0, LOAD_PLAIN, STORE_ROWS>(ps.logr, a, grid, tile * 8, stream);
            } else {
                tile = (uint32_t)std::min<uint64_t>(n, PASS_TILE);
                grid = a.vcols * (n / tile);
                if (first) launch_pass<0, LOAD_COSETS, STORE_SAME>(ps.logr, a, grid, tile * 8, stream);
                else launch_pass<0, LOAD_PLAIN, STORE_SAME>(ps.logr, a, grid, tile * 8, stream);
            }
            ZK_CUDA(cudaGetLastError());
        }
    }
}

// ------------------------------------------- planned passes (serving loop)
//
// The fused LDE's passes as data instead of launches, for a persistent kernel
// that runs every tile of each pass itself (serve_loop.cu): the same chunks,
// arguments and tables as lde_rows_device, with the row-output pass at radix
// 2^8 whatever the tuning table says (the loop compiles a fixed set of pass
// shapes; every split gives the same rows).
static constexpr uint32_t LOOP_LAST_LOGR = MAX_ROWS_LOGR;

bool lde_rows_plan_tables_resident(DeviceCtx &c, uint32_t lg_n, uint32_t rate, uint64_t coset_gen)
{
    if (!c.lde_tabs.count(std::make_tuple(lg_n, rate, coset_gen % GL_P)) || !c.tw[0][12]) return false;
    for (const Pass &ps : plan_passes_last(lg_n, true, LOOP_LAST_LOGR))
        if (ps.s_lo && !c.tw[0][ps.s_lo + ps.logr]) return false;
    return true;
}

void lde_rows_plan_tables(DeviceCtx &c, uint32_t lg_n, uint32_t rate, uint64_t coset_gen)
{
    c.lde_table(lg_n, rate, coset_gen % GL_P);
    c.twiddles(12, false);
    for (const Pass &ps : plan_passes_last(lg_n, true, LOOP_LAST_LOGR))
        if (ps.s_lo) c.twiddles(ps.s_lo + ps.logr, false);
}

std::vector<PlannedPass> lde_rows_plan(DeviceCtx &c, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n,
                                       uint32_t rate, uint64_t cols, uint64_t coset_gen, uint64_t *scratch)
{
    if (!lde_rows_plan_tables_resident(c, lg_n, rate, coset_gen)) throw arg_failure("tables of this shape not built");
    const uint64_t n = 1ULL << lg_n;
    const auto passes = plan_passes_last(lg_n, true, LOOP_LAST_LOGR);
    const bool multi = passes.size() > 1;
    const uint64_t chunk = multi ? lde_rows_chunk_cols(lg_n, rate, cols) : cols;
    if (multi && !scratch) throw arg_failure("null scratch");
    const uint64_t *tab = c.lde_table(lg_n, rate, coset_gen % GL_P);
    std::vector<PlannedPass> out;
    for (uint64_t c0 = 0; c0 < cols; c0 += chunk) {
        const uint64_t cc = cols - c0 < chunk ? cols - c0 : chunk;
        for (size_t pi = 0; pi < passes.size(); pi++) {
            const Pass &ps = passes[pi];
            const bool first = pi == 0, last = pi + 1 == passes.size();
            PlannedPass pp{};
            NttPassArgs &a = pp.a;
            a.src = first ? coeffs + c0 * n : scratch;
            a.src_stride = n;
            a.tab = tab;
            a.tw_small = c.twiddles(12, false);
            a.tw_pass = ps.s_lo ? c.twiddles(ps.s_lo + ps.logr, false) : nullptr;
            a.vcols = cc << rate;
            a.L = lg_n;
            a.s_lo = ps.s_lo;
            a.rate = rate;
            a.cols = (uint32_t)cc;
            a.row_stride = cols;
            a.dst = last ? rows + c0 : scratch;
            a.dst_stride = n;
            a.src_len = first ? (cols - c0) * n : (n << rate) * chunk;
            a.dst_len = last ? (n << rate) * cols - c0 : (n << rate) * chunk;
            a.tab_len = n << rate;
            if (last) {
                const uint32_t W = (uint32_t)std::min<uint64_t>(n, PASS_TILE / 16);
                pp.grid = (n / W) * ((cc + 15) / 16) * (1ULL << rate);
            } else {
                pp.grid = a.vcols * (n / std::min<uint64_t>(n, PASS_TILE));
            }
            pp.logr = ps.logr;
            pp.load = first ? LOAD_COSETS : LOAD_PLAIN;
            pp.store = last ? STORE_ROWS : STORE_SAME;
            pp.direct = direct_io(ps.logr, a, last) ? 1 : 0;
            out.push_back(pp);
        }
    }
    return out;
}

bool ntt_inverse_plan_tables_resident(DeviceCtx &c, uint32_t lg)
{
    if (!c.tw[1][12]) return false;
    for (const Pass &ps : plan_passes(lg, false))
        if (ps.s_lo && !c.tw[1][ps.s_lo + ps.logr]) return false;
    return true;
}

void ntt_inverse_plan_tables(DeviceCtx &c, uint32_t lg)
{
    c.twiddles(12, true);
    for (const Pass &ps : plan_passes(lg, false))
        if (ps.s_lo) c.twiddles(ps.s_lo + ps.logr, true);
}

std::vector<PlannedPass> ntt_inverse_plan(DeviceCtx &c, uint64_t *inout, uint32_t lg, uint64_t batches,
                                          uint64_t *scratch, PlannedReorder &ro)
{
    if (lg == 0 || batches == 0) throw arg_failure("empty transform");
    if (!ntt_inverse_plan_tables_resident(c, lg)) throw arg_failure("tables of this shape not built");
    const uint64_t n = 1ULL << lg;
    const auto passes = plan_passes(lg, false);
    std::vector<PlannedPass> out;
    for (size_t pi = 0; pi < passes.size(); pi++) {
        const Pass &ps = passes[pi];
        const bool first = pi == 0;
        PlannedPass pp{};
        NttPassArgs &a = pp.a;
        // as run_dif for a column-output inverse DIF: inout -> scratch, then in place
        a.src = first ? inout : scratch;
        a.src_len = n * batches;
        a.src_stride = n;
        a.tw_small = c.twiddles(12, true);
        a.tw_pass = ps.s_lo ? c.twiddles(ps.s_lo + ps.logr, true) : nullptr;
        a.vcols = batches;
        a.L = lg;
        a.s_lo = ps.s_lo;
        a.dst = scratch;
        a.dst_stride = n;
        a.dst_len = n * batches;
        pp.grid = batches * (n / std::min<uint64_t>(n, PASS_TILE));
        pp.logr = ps.logr;
        pp.load = LOAD_PLAIN;
        pp.store = STORE_SAME;
        pp.direct = direct_io(ps.logr, a, false) ? 1 : 0;
        pp.inv = 1;
        out.push_back(pp);
    }
    // bit-reversed -> natural order, times n^-1 (reorder(), no coset table)
    const uint32_t ra = lg >= 10 ? 5 : lg / 2;
    ro = PlannedReorder{scratch, inout, n, n, lg, 0, batches, H_SIZE_INV[lg], n * batches, n * batches,
                        batches * (1ULL << (lg - 2 * ra))};
    return out;
}

// Passes of the fused LDE of 2^lg_n-point columns: (s_lo, log radix) pairs.
std::vector<std::pair<uint32_t, uint32_t>> lde_rows_passes(uint32_t lg_n)
{
    std::vector<std::pair<uint32_t, uint32_t>> v;
    for (const Pass &p : plan_passes(lg_n, true)) v.push_back({p.s_lo, p.logr});
    return v;
}

uint64_t lde_rows_scratch_elems(uint32_t lg_n, uint32_t rate, uint64_t cols)
{
    if (plan_passes(lg_n, true).size() == 1) return 0;
    return (1ULL << (lg_n + rate)) * lde_rows_chunk_cols(lg_n, rate, cols);
}

void lde_rows_device(DeviceCtx &c, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n, uint32_t rate, uint64_t cols,
                     uint64_t coset_gen, uint64_t *scratch, const uint64_t *host_coeffs, const RowScatter *scatter)
{
    NvtxRange range("zeknox lde_rows");
    const uint64_t n = 1ULL << lg_n;
    if (cols == 0) return;
    const bool multi = plan_passes(lg_n, true).size() > 1;
    uint64_t chunk = multi ? lde_rows_chunk_cols(lg_n, rate, cols) : cols;
    if (multi && host_coeffs) {
        // never above the scratch sized by lde_rows_chunk_cols
        const uint64_t h = chunk_cols_for(tune_get("lde_host_chunk_mib", lg_n + rate, ZK_HOST_CHUNK_MIB), lg_n, rate, cols);
        chunk = h < chunk ? h : chunk;
    }
    DevBuf tmp;
    if (multi && !scratch) {
        tmp.ctx = &c;
        tmp.p = c.alloc(lde_rows_scratch_elems(lg_n, rate, cols) * 8);
        scratch = tmp.p;
    }
    const uint64_t *tab = c.lde_table(lg_n, rate, coset_gen % GL_P);
    if (host_coeffs) {
        // coefficients are in host memory: copy chunk by chunk on the copy
        // stream into `coeffs` (device staging) so chunk k+1 crosses PCIe while
        // chunk k is transformed
        cudaStream_t cs = c.copy_stream_get();
        cudaEvent_t ready = c.chunk_event(0);
        ZK_CUDA(cudaEventRecord(ready, c.stream));
        ZK_CUDA(cudaStreamWaitEvent(cs, ready, 0));  // staging is free once earlier work on the stream is done
        size_t k = 1;
        for (uint64_t c0 = 0; c0 < cols; c0 += chunk, k++) {
            const uint64_t cc = cols - c0 < chunk ? cols - c0 : chunk;
            ZK_CUDA(cudaMemcpyAsync((void *)(coeffs + c0 * n), host_coeffs + c0 * n, cc * n * 8, cudaMemcpyHostToDevice, cs));
            ZK_CUDA(cudaEventRecord(c.chunk_event(k), cs));
        }
    }
    size_t k = 1;
    for (uint64_t c0 = 0; c0 < cols; c0 += chunk, k++) {
        const uint64_t cc = cols - c0 < chunk ? cols - c0 : chunk;
        if (host_coeffs) ZK_CUDA(cudaStreamWaitEvent(c.stream, c.chunk_event(k), 0));
        DifJob j{};
        j.src = coeffs + c0 * n;
        j.src_stride = n;
        j.load = LOAD_COSETS;
        j.tab = tab;
        j.dst = scatter ? nullptr : rows + c0;
        j.row_stride = scatter ? scatter->row_stride : cols;
        j.scatter = scatter;
        j.col0 = c0;
        j.vcols = cc << rate;
        j.L = lg_n;
        j.rate = rate;
        j.cols = (uint32_t)cc;
        j.rows = true;
        j.scratch = scratch;
        j.src_len = (cols - c0) * n;
        j.tab_len = n << rate;
        j.dst_len = scatter ? (1ULL << scatter->log_rows_per_dst) * scatter->row_stride : (n << rate) * cols - c0;
        j.scratch_len = multi ? (n << rate) * chunk : 0;
        run_dif(c, j);
    }
}

// Tables a commit of this shape reads, built now (the batched path captures
// its launches in a CUDA graph, where nothing may allocate).
void prepare_tables(DeviceCtx &c, uint32_t lg_n, uint32_t rate, uint64_t coset_gen, bool values)
{
    c.lde_table(lg_n, rate, coset_gen % GL_P);
    c.twiddles(12, false);
    for (const Pass &ps : plan_passes(lg_n, true))
        if (ps.s_lo) c.twiddles(ps.s_lo + ps.logr, false);
    if (values) {
        c.twiddles(12, true);
        for (const Pass &ps : plan_passes(lg_n, false))
            if (ps.s_lo) c.twiddles(ps.s_lo + ps.logr, true);
    }
}

// The bulk-copy transpose: persistent CTAs, as many as fit on the SMs with
// their stage buffers.
template <uint32_t TI, uint32_t TB, uint32_t ST>
static void launch_transpose_bulk(DeviceCtx &c, uint64_t *out, const uint64_t *in, uint32_t lg, uint64_t cols,
                                  uint32_t extra, uint64_t wait_ns)
{
    using G = TrBulk<TI, TB, ST>;
    static int per_sm_of[64] = {};  // per device, set once under its lock
    int &per_sm = per_sm_of[c.id & 63];
    if (!per_sm) {
        ZK_CUDA(cudaFuncSetAttribute(transpose_rev_bulk_kernel<TI, TB, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)G::SMEM_BYTES));
        ZK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, transpose_rev_bulk_kernel<TI, TB, ST>, G::THREADS,
                                                              G::SMEM_BYTES));
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t n = 1ULL << lg;
    const uint64_t tiles_i = n / TI, n_tiles = tiles_i * ((cols + TB - 1) / TB);
    const uint64_t ctas = std::min<uint64_t>(n_tiles, (uint64_t)c.sm_count * per_sm);
    transpose_rev_bulk_kernel<TI, TB, ST><<<(unsigned)ctas, G::THREADS, G::SMEM_BYTES, c.stream>>>(
        in, out, lg, cols, tiles_i, n_tiles, c.wait_status(), extra, wait_ns);
}

void transpose_rev_device(DeviceCtx &c, uint64_t *out, const uint64_t *in, uint32_t lg, uint64_t cols)
{
    NvtxRange range("zeknox transpose_rev");
    const uint64_t n = 1ULL << lg;
    if (cols == 0) return;
    dim3 grid((unsigned)((n + 63) / 64), (unsigned)((cols + 31) / 32));
    if (grid.y > 65535) throw arg_failure("too many columns for transpose");
    const bool vec16 = lg >= 1 && cols % 2 == 0 && ((uintptr_t)in % 16) == 0 && ((uintptr_t)out % 16) == 0;
    // knob transpose_bulk: 0 the 16-byte form, 1..8 a bulk-copy tile shape,
    // 9 (default) by column count: 64 x 64 tiles with 3 stages from 48
    // columns, else 64 x 32 with 4 (measured on B200: 0.198 against 0.213 ms
    // for the 16-byte form at 256 x 2^18, 0.223 against 0.240 ms at 16 x 2^22)
    uint64_t form = vec16 ? tune_get("transpose_bulk", lg, 9) : 0;
    if (form == 9) form = cols >= 48 ? 3 : 1;
    if (form >= 1 && form <= 8 && lg >= (form == 4 || form == 5 ? 7u : 6u)) {
        uint32_t extra = 0;
        uint64_t wait_ns = 1000000000ULL;  // 1 s: a stage of tens of KiB lands in microseconds
        if (c.inject_wait_timeouts) {
            c.inject_wait_timeouts--;
            extra = 16;
            wait_ns = 20000000ULL;
        }
        switch (form) {
        case 1: launch_transpose_bulk<64, 32, 4>(c, out, in, lg, cols, extra, wait_ns); break;
        case 2: launch_transpose_bulk<64, 32, 2>(c, out, in, lg, cols, extra, wait_ns); break;
        case 3: launch_transpose_bulk<64, 64, 3>(c, out, in, lg, cols, extra, wait_ns); break;
        case 4: launch_transpose_bulk<128, 32, 3>(c, out, in, lg, cols, extra, wait_ns); break;
        case 5: launch_transpose_bulk<128, 32, 2>(c, out, in, lg, cols, extra, wait_ns); break;
        case 6: launch_transpose_bulk<64, 32, 8>(c, out, in, lg, cols, extra, wait_ns); break;
        case 7: launch_transpose_bulk<64, 64, 2>(c, out, in, lg, cols, extra, wait_ns); break;
        default: launch_transpose_bulk<32, 64, 4>(c, out, in, lg, cols, extra, wait_ns); break;
        }
    } else if (vec16) {
        transpose_rev_v2_kernel<<<grid, 256, 0, c.stream>>>(in, out, lg, cols);
    } else {
        transpose_rev_kernel<<<grid, 256, 0, c.stream>>>(in, out, lg, cols);
    }
    note_launch();
    ZK_CUDA(cudaGetLastError());
}

// salt columns: seeded counter-based values in [0, p) (the reference draws
// curand numbers seeded with time(NULL), native/ntt/ntt.cu:541-546)
__global__ void salt_kernel(uint64_t *out, uint64_t count, uint64_t seed)
{
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (k + 1) * 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        out[k] = z >= GL_P ? z - GL_P : z;
    }
}

void salt_device(DeviceCtx &c, uint64_t *out, uint64_t count)
{
    uint64_t seed;
    const char *env = getenv("ZEKNOX_SALT_SEED");
    if (env) seed = strtoull(env, nullptr, 0);
    else seed = (uint64_t)std::chrono::steady_clock::now().time_since_epoch().count();
    uint64_t blocks = std::min<uint64_t>((count + 255) / 256, (uint64_t)c.sm_count * 8);
    if (blocks == 0) return;
    salt_kernel<<<(unsigned)blocks, 256, 0, c.stream>>>(out, count, seed);
    note_launch();
    ZK_CUDA(cudaGetLastError());
}

cudaError_t oob_take_ntt(uint64_t r[4]) { return oob_take_local(r); }

}  // namespace zk
