// ntt.cuh -- batched Goldilocks NTT passes (device side).
//
// Replaces the radix-2 stage kernels of zeknox native/ntt/kernels.cu:160-392
// (one global pass per stage) with a multi-pass decimation-in-frequency
// engine: each pass applies k = LOGR consecutive DIF stages to every group of
// R = 2^k elements spaced S = 2^s_lo apart, through shared memory, so a 2^L
// transform costs ceil(L / k) passes over HBM instead of L.
//
// Math.  For a block of M = R*S elements viewed as x[m*S + o] (m < R, o < S),
// the first k DIF stages leave, at position m'*S + o,
//     w_M^(o * f) * sum_m x[m*S + o] * w_R^(m * f),     f = rev_k(m'),
// after which every run of S contiguous positions is an independent DIF of
// size S.  The R-point transform inside a pass is itself split the same way
// into register-resident E-point DIFs (E <= 16) whose twiddles are powers of
// w_E, i.e. powers of 2 (w_64 = 2^39 for zeknox's roots), so they cost a shift
// and a reduction instead of a multiplication.  After the last pass position
// j of each transform holds X[rev_L(j)] (bit-reversed order).
//
// A "virtual column" is one independent transform.  For a low-degree
// extension of rate 2^rate, coset c of input column b is its own virtual
// column: coefficient j is scaled by (g * w_N^c)^j and transformed at size n,
// and its bit-reversed output is exactly rows [rev_rate(c)*n, (rev_rate(c)+1)*n)
// of the bit-reversed size-N evaluation -- zero-extension never touches memory.
#pragma once
#include <stdint.h>

#include "bounds.cuh"
#include "bulk.cuh"
#include "gl64.cuh"
#include "ntt_args.h"

namespace zk {

// w_{2^h} = 2^EXP for the reference's roots (h = 1..6), forward and inverse.
__host__ __device__ constexpr unsigned root_exp(int h, int inv)
{
    return inv ? (h == 1 ? 96 : h == 2 ? 144 : h == 3 ? 72 : h == 4 ? 36 : h == 5 ? 114 : 153)
               : (h == 1 ? 96 : h == 2 ? 48 : h == 3 ? 120 : h == 4 ? 156 : h == 5 ? 78 : 39);
}

// The butterfly sum with its carry chains as multiply-adds x * 1 + y: the NTT
// passes are bound by the integer ALU and leave the multiply pipe mostly idle
// (measured 1.01-1.02x on the fused LDE; moving the twiddle products'
// reduction and the difference's correction there as well measured 0.96x).
// The 1 and 0 come from the constant bank, so the compiler cannot fold the
// products back into additions.
static __constant__ uint32_t d_ntt_one = 1, d_ntt_zero = 0;
__device__ __forceinline__ uint64_t ntt_add(uint64_t a, uint64_t b)
{
    uint32_t r0, r1, t0, t1, c;
    asm("{\n\t"
        "mad.lo.cc.u32   %0, %5, %9, %7;\n\t"    // r = a + b
        "madc.lo.cc.u32  %1, %6, %9, %8;\n\t"
        "madc.lo.u32     %4, %10, %10, %10;\n\t"  // c = carry
        "mad.lo.cc.u32   %2, %9, 0xffffffff, %0;\n\t"  // t = r + EPS
        "madc.lo.cc.u32  %3, %10, %10, %1;\n\t"
        "madc.lo.u32     %4, %10, %10, %4;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(t0), "=&r"(t1), "=&r"(c)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)), "r"(d_ntt_one),
          "r"(d_ntt_zero));
    return c ? (((uint64_t)t1 << 32) | t0) : (((uint64_t)r1 << 32) | r0);  // gl_add's selection
}

// ---- lazily reduced butterfly arithmetic.  Inside a pass the values are any
// 64-bit representatives ("nc"), as in the hash permutations: sums and
// differences fold their carry or borrow back in (2^64 = EPS mod p) with no
// comparison and no canonicalisation, twiddle products stay unreduced, and a
// value is canonicalised once, when the pass stores it to global memory.

// a + b for any 64-bit a, b: lo + 2^64 c = lo + c * EPS, which can carry once
// more (only when both operands are >= p).  A plain carry chain: on B200 it
// measured about 12 instructions against about 16 for the same sum with its
// carries taken through multiply-adds, and the passes are issue-bound.
__device__ __forceinline__ uint64_t ntt_add_nc(uint64_t a, uint64_t b)
{
    uint32_t r0, r1, c;
    asm("{\n\t"
        "add.cc.u32      %0, %3, %5;\n\t"
        "addc.cc.u32     %1, %4, %6;\n\t"
        "addc.u32        %2, 0, 0;\n\t"
        "neg.s32         %2, %2;\n\t"       // carry ? EPS : 0
        "add.cc.u32      %0, %0, %2;\n\t"
        "addc.cc.u32     %1, %1, 0;\n\t"
        "addc.u32        %2, 0, 0;\n\t"
        "neg.s32         %2, %2;\n\t"
        "add.cc.u32      %0, %0, %2;\n\t"   // second carry: r + EPS < 2 EPS
        "addc.u32        %1, %1, 0;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(c)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// a - b for any 64-bit a, b: the wrapped difference d stands for d - 2^64 =
// d - EPS on a borrow, which can borrow once more (d < EPS).
__device__ __forceinline__ uint64_t ntt_sub_nc(uint64_t a, uint64_t b)
{
    uint32_t r0, r1, m;
    asm("{\n\t"
        "sub.cc.u32      %0, %3, %5;\n\t"
        "subc.cc.u32     %1, %4, %6;\n\t"
        "subc.u32        %2, 0, 0;\n\t"       // m = borrow ? EPS : 0
        "sub.cc.u32      %0, %0, %2;\n\t"
        "subc.cc.u32     %1, %1, 0;\n\t"
        "subc.u32        %2, 0, 0;\n\t"
        "sub.cc.u32      %0, %0, %2;\n\t"
        "subc.u32        %1, %1, 0;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(m)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// a * 2^E for 0 < E < 96 and any 64-bit a, unreduced.  With t = E mod 32 and
// a * 2^t = q0 + 2^32 q1 + 2^64 q2 (two wide multiplies of a's halves):
//   E <  32:  q0 + 2^32 q1 + EPS q2
//   E <  64:  2^32 q0 + EPS q1 - q2          (2^96 = -1)
//   E <  96:  EPS q0 - q1 - 2^32 q2          (2^128 = -2^32)
// each folded to 64 bits with at most two carry / borrow corrections.
template <unsigned E>
__device__ __forceinline__ uint64_t ntt_mul_pow2_nc(uint64_t a)
{
    static_assert(E > 0 && E < 96, "exponent");
    const uint32_t m = 1u << (E & 31);
    uint32_t q0, q1, q2;
    asm("{\n\t"
        ".reg .u64 p0, p1;\n\t"
        ".reg .u32 h0, l1, h1;\n\t"
        "mul.wide.u32    p0, %3, %5;\n\t"
        "mul.wide.u32    p1, %4, %5;\n\t"
        "mov.b64         {%0, h0}, p0;\n\t"
        "mov.b64         {l1, h1}, p1;\n\t"
        "add.cc.u32      %1, h0, l1;\n\t"
        "addc.u32        %2, h1, 0;\n\t"
        "}"
        : "=r"(q0), "=r"(q1), "=r"(q2)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"(m));
    uint32_t t0, t1;
    if constexpr (E < 32) {
        // (q1:q0) + q2 * EPS < 2^65 - 2^33: one correction
        uint64_t e;
        asm("mul.wide.u32 %0, %1, 0xffffffff;" : "=l"(e) : "r"(q2));
        asm("{\n\t"
            ".reg .u32 c;\n\t"
            "add.cc.u32      %0, %2, %4;\n\t"
            "addc.cc.u32     %1, %3, %5;\n\t"
            "addc.u32        c, 0, 0;\n\t"
            "mad.lo.cc.u32   %0, c, 0xffffffff, %0;\n\t"
            "addc.u32        %1, %1, 0;\n\t"
            "}"
            : "=&r"(t0), "=&r"(t1)
            : "r"(q0), "r"(q1), "r"((uint32_t)e), "r"((uint32_t)(e >> 32)));
    } else if constexpr (E < 64) {
        // 2^32 q0 + q1 * EPS - q2 with a signed top limb in {-1, 0, 1}
        uint64_t e;
        asm("mul.wide.u32 %0, %1, 0xffffffff;" : "=l"(e) : "r"(q1));
        asm("{\n\t"
            ".reg .u32 top, cl, ch;\n\t"
            "add.cc.u32      %1, %2, %4;\n\t"
            "addc.u32        top, 0, 0;\n\t"
            "sub.cc.u32      %0, %3, %5;\n\t"
            "subc.cc.u32     %1, %1, 0;\n\t"
            "subc.u32        top, top, 0;\n\t"
            "neg.s32         cl, top;\n\t"
            "shr.s32         ch, top, 31;\n\t"
            "add.cc.u32      %0, %0, cl;\n\t"
            "addc.u32        %1, %1, ch;\n\t"
            "}"
            : "=&r"(t0), "=&r"(t1)
            : "r"(q0), "r"((uint32_t)e), "r"((uint32_t)(e >> 32)), "r"(q2));
    } else {
        // (q0 - q2) * 2^32 - q0 - q1, in (-2^64, 2^64): a borrow stands for
        // -2^64 = -EPS, which can borrow once more
        asm("{\n\t"
            ".reg .u32 b;\n\t"
            "sub.cc.u32      %0, 0, %2;\n\t"
            "subc.cc.u32     %1, %2, %4;\n\t"
            "subc.u32        b, 0, 0;\n\t"
            "sub.cc.u32      %0, %0, %3;\n\t"
            "subc.cc.u32     %1, %1, 0;\n\t"
            "subc.u32        b, b, 0;\n\t"       // 0 or -1 (the value is above -2^64)
            "sub.cc.u32      %0, %0, b;\n\t"     // b = -1 = EPS as a u32: subtract EPS
            "subc.cc.u32     %1, %1, 0;\n\t"
            "subc.u32        b, 0, 0;\n\t"
            "sub.cc.u32      %0, %0, b;\n\t"
            "subc.u32        %1, %1, 0;\n\t"
            "}"
            : "=&r"(t0), "=&r"(t1)
            : "r"(q0), "r"(q1), "r"(q2));
    }
    return ((uint64_t)t1 << 32) | t0;
}

// In-register DIF on E = 2^LOGE values: natural input, bit-reversed output,
// values lazily reduced.  Stages and butterflies are expanded at compile time
// so every index and every shift amount is a constant (the values stay in
// registers).  A twiddle w_{2^H}^I = 2^k with 96 <= k is -2^(k-96): the
// difference is taken the other way round instead of negated.
template <int INV, int H, int SPAN, int BLK, int I>
__device__ __forceinline__ void dif_bfly(uint64_t *x)
{
    constexpr unsigned K = (root_exp(H, INV) * (unsigned)I) % 192u;
    constexpr bool NEG = K >= 96;
    constexpr unsigned E = NEG ? K - 96 : K;
    const uint64_t u = x[BLK + I], v = x[BLK + I + SPAN];
    x[BLK + I] = ntt_add_nc(u, v);
    const uint64_t d = NEG ? ntt_sub_nc(v, u) : ntt_sub_nc(u, v);
    if constexpr (E == 0) x[BLK + I + SPAN] = d;
    else x[BLK + I + SPAN] = ntt_mul_pow2_nc<E>(d);
    if constexpr (I + 1 < SPAN) dif_bfly<INV, H, SPAN, BLK, I + 1>(x);
}

template <int INV, int E, int H, int BLK>
__device__ __forceinline__ void dif_stage(uint64_t *x)
{
    constexpr int SPAN = 1 << (H - 1);
    dif_bfly<INV, H, SPAN, BLK, 0>(x);
    if constexpr (BLK + 2 * SPAN < E) dif_stage<INV, E, H, BLK + 2 * SPAN>(x);
}

template <int INV, int E, int H>
__device__ __forceinline__ void dif_stages(uint64_t *x)
{
    dif_stage<INV, E, H, 0>(x);
    if constexpr (H > 1) dif_stages<INV, E, H - 1>(x);
}

template <int LOGE, int INV>
__device__ __forceinline__ void dif_regs(uint64_t *x)
{
    dif_stages<INV, 1 << LOGE, LOGE>(x);
}

// XOR-fold swizzle of a shared-memory word index (8-byte words): every
// power-of-two access stride used below hits 16 distinct 8-byte banks.
__device__ __forceinline__ uint32_t swz(uint32_t w) { return w ^ (((w >> 4) ^ (w >> 8) ^ (w >> 12)) & 15u); }

// Sub-step of the in-CTA R-point DIF: every task owns E elements spaced Q apart
// inside a block of size R_cur = E * Q.  The task base (block * R_cur + m_lo,
// m_lo < Q) and the element offsets e * Q occupy disjoint bits, and swz() is
// linear over XOR, so swz(base + e * Q) = swz(base) ^ swz(e * Q) with the
// second term a compile-time constant.
__host__ __device__ constexpr uint32_t swz_c(uint32_t w) { return w ^ (((w >> 4) ^ (w >> 8) ^ (w >> 12)) & 15u); }

// bits-bit reversal of a compile-time value
__host__ __device__ constexpr uint32_t bitrev_c(uint32_t x, int bits)
{
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

template <int LOGE, int INV, int NT, int LOG_RCUR>
__device__ __forceinline__ void dif_substep(uint64_t *sm, uint32_t tile_elems, const uint64_t *__restrict__ tw_small)
{
    constexpr int E = 1 << LOGE;
    constexpr uint32_t Q = 1u << (LOG_RCUR - LOGE);
    const uint32_t tasks = tile_elems >> LOGE;
    for (uint32_t t = threadIdx.x; t < tasks; t += NT) {
        const uint32_t m_lo = t & (Q - 1);
        const uint32_t blk = t >> (LOG_RCUR - LOGE);  // block of R_cur (across groups)
        const uint32_t sb = swz((blk << LOG_RCUR) + m_lo);
        uint64_t x[E];
#pragma unroll
        for (int e = 0; e < E; e++) x[e] = sm[sb ^ swz_c(e * Q)];
        dif_regs<LOGE, INV>(x);
        if (Q > 1) {
            // position p gets w_{R_cur}^(m_lo * rev_e(p)); w_{R_cur} = w_4096^(4096 / R_cur)
            const uint32_t step = m_lo << (12 - LOG_RCUR);
#pragma unroll
            for (int p = 1; p < E; p++) {
                const uint32_t f = bitrev32((uint32_t)p, LOGE);
                x[p] = gl_mul_nc(x[p], __ldg(tw_small + ((step * f) & 4095u)));
            }
        }
#pragma unroll
        for (int e = 0; e < E; e++) sm[sb ^ swz_c(e * Q)] = x[e];
    }
}

// All sub-steps of an R = 2^LOGR point DIF: 16-point steps, then the remainder.
template <int LOGR, int INV, int NT, int LOG_RCUR>
__device__ __forceinline__ void dif_substeps(uint64_t *sm, uint32_t tile, const uint64_t *__restrict__ tw_small)
{
    if constexpr (LOG_RCUR >= 4) dif_substep<4, INV, NT, LOG_RCUR>(sm, tile, tw_small);
    else dif_substep<LOG_RCUR, INV, NT, LOG_RCUR>(sm, tile, tw_small);
    __syncthreads();
    if constexpr (LOG_RCUR > 4) dif_substeps<LOGR, INV, NT, LOG_RCUR - 4>(sm, tile, tw_small);
}

// log2 of the block size of the last sub-step of an R = 2^LOGR point DIF
// (16-point sub-steps first): LOGR - 4 * floor((LOGR - 1) / 4).
__host__ __device__ constexpr int last_substep_log(int logr) { return logr - 4 * ((logr - 1) / 4); }

// The sub-steps strictly between the first (LOG_RCUR = LOGR) and the last
// (LOG_RCUR = last_substep_log(LOGR)), smem to smem.
template <int INV, int NT, int LOG_RCUR, int LAST>
__device__ __forceinline__ void dif_middle_substeps(uint64_t *sm, uint32_t tile, const uint64_t *__restrict__ tw_small)
{
    if constexpr (LOG_RCUR > LAST) {
        dif_substep<4, INV, NT, LOG_RCUR>(sm, tile, tw_small);
        __syncthreads();
        dif_middle_substeps<INV, NT, LOG_RCUR - 4, LAST>(sm, tile, tw_small);
    }
}

// The inner twiddles after the first sub-step's E-point DIFs: position p of
// task m_lo gets w_R^(m_lo * rev_e(p)), w_R = w_4096^(4096 / R).
template <int LOGE, int LOGR>
__device__ __forceinline__ void first_substep_twiddles(uint64_t *x, uint32_t m_lo, const uint64_t *__restrict__ tw_small)
{
    constexpr int E = 1 << LOGE;
    if constexpr (LOGR > LOGE) {
        const uint32_t step = m_lo << (12 - LOGR);
#pragma unroll
        for (int p = 1; p < E; p++) {
            const uint32_t f = bitrev32((uint32_t)p, LOGE);
            x[p] = gl_mul_nc(x[p], __ldg(tw_small + ((step * f) & 4095u)));
        }
    }
}

// One pass: LOGR stages on groups of R = 2^LOGR elements; at most TILE
// elements per CTA (dynamic shared memory of TILE words).
//   STORE_SAME tiles: min(TILE, n) positions of one virtual column; when the
//     group spacing S is at least the number of groups per tile the rows of a
//     tile are runs of consecutive offsets, otherwise the tile is one
//     contiguous span of whole blocks.
//   STORE_ROWS tiles (last pass, S == 1): 16 virtual columns of one coset and
//     consecutive source columns x W positions, so every output leaf row gets
//     16 consecutive 8-byte words.
// DIRECT (chosen by the host when a warp's accesses stay sector-complete:
// STORE_ROWS, or STORE_SAME with row-run tiles of >= 4 groups): the first
// sub-step loads its elements straight from global memory into registers and,
// for STORE_SAME, the last sub-step stores straight from registers, instead of
// separate load / store loops through shared memory.
// Threads per SM the register budget aims at: 1280 (five 256-thread CTAs, 48
// registers) for the LDE's coset-expanding column pass of up to 2^9 points,
// whose first sub-step waits on its global loads; 1024 (64 registers)
// otherwise.  Measured on B200: fused LDE 1.065 against 1.101 ms at 256 x
// 2^15, rate 3; five CTAs for every pass (the row pass then spills): 1.068 ms,
// and for every column pass the plain NTT's passes measured 1-4% slower; six
// (40 registers, spilling): 1.091 ms; 8-point register sub-steps at 40 or 64
// registers: 1.18-1.23 ms.  Radices of 2^10 and above spill at 48 registers.
template <int LOGR, int LOADM, int STOREM>
__host__ __device__ constexpr int pass_threads_per_sm()
{
    return (LOADM == LOAD_COSETS && STOREM == STORE_SAME && LOGR < 10) ? 1280 : 1024;
}

// One CTA's work of a pass: tile ZK_PASS_BLK of the launch described by `a`,
// with TILE words of shared memory at sm.  ntt_pass_kernel runs it for its own
// block index; ntt_pass_body for any tile (the persistent serving loop runs
// every tile of a pass through it).
template <int LOGR, int INV, int NT, int TILE, int LOADM, int STOREM, int DIRECT>
__global__ void __launch_bounds__(NT, pass_threads_per_sm<LOGR, LOADM, STOREM>() / NT) ntt_pass_kernel(NttPassArgs a)
{
    extern __shared__ uint64_t sm[];
#define ZK_PASS_BLK blockIdx.x
#include "ntt_pass_body.inc"
#undef ZK_PASS_BLK
}

template <int LOGR, int INV, int NT, int TILE, int LOADM, int STOREM, int DIRECT>
__device__ __forceinline__ void ntt_pass_body(const NttPassArgs &a, uint32_t blk, uint64_t *sm)
{
#define ZK_PASS_BLK blk
#include "ntt_pass_body.inc"
#undef ZK_PASS_BLK
}

// ------------------------------------------------------------------ reorders

// Bit-reversed -> natural order with optional per-element factor:
//   dst[v * dst_stride + i] = src[v * src_stride + rev_L(i)] * scale(i)
// where scale(i) = mul (a constant, e.g. n^-1), times tab[i] when tab != null.
// For the LDE interleave (rate > 0): natural index i = c + 2^rate * t takes
// virtual column v * 2^rate + c at bit-reversed position t.
// Tiles of 32 x 32 through shared memory so both sides are coalesced.
static __global__ void __launch_bounds__(256) bitrev_reorder_kernel(const uint64_t *__restrict__ src, uint64_t *__restrict__ dst,
                                                             uint64_t src_stride, uint64_t dst_stride, uint32_t lg_t,
                                                             uint32_t rate, uint64_t cols, uint64_t mul,
                                                             const uint64_t *__restrict__ tab, uint64_t src_len,
                                                             uint64_t dst_len)
{
    __shared__ uint64_t tile[32][33];
#define ZK_REORDER_BLK blockIdx.x
#include "ntt_reorder_body.inc"
#undef ZK_REORDER_BLK
}

// One tile of the reorder: tile `blk` of the launch described by the
// arguments, with `tile` (32 x 33 words) in shared memory.
__device__ __forceinline__ void bitrev_reorder_body(const uint64_t *src, uint64_t *dst, uint64_t src_stride,
                                                    uint64_t dst_stride, uint32_t lg_t, uint32_t rate, uint64_t cols,
                                                    uint64_t mul, const uint64_t *tab, uint64_t src_len,
                                                    uint64_t dst_len, uint64_t blk_index, uint64_t (*tile)[33])
{
#define ZK_REORDER_BLK blk_index
#include "ntt_reorder_body.inc"
#undef ZK_REORDER_BLK
}

// out[rev_lg(i) * cols + b] = in[b * n + i]: tiles of 64 positions x 32
// columns through shared memory, so reads are 512-byte runs of a column and
// writes 256-byte runs of a leaf row.  The general form: any column count and
// any 8-byte alignment.
static __global__ void __launch_bounds__(256) transpose_rev_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                                                            uint32_t lg, uint64_t cols)
{
    constexpr uint32_t TI = 64, TB = 32;
    __shared__ uint64_t tile[TB][TI + 1];
    const uint64_t n = 1ULL << lg;
    const uint64_t i0 = (uint64_t)blockIdx.x * TI;
    const uint64_t b0 = (uint64_t)blockIdx.y * TB;
    for (uint32_t e = threadIdx.x; e < TI * TB; e += 256) {
        const uint32_t r = e / TI, c = e % TI;
        const uint64_t b = b0 + r, i = i0 + c;
        if (b < cols && i < n && ZK_IN_BOUNDS(b * n + i, n * cols, OOB_TRANSPOSE_IN)) tile[r][c] = in[b * n + i];
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < TI * TB; e += 256) {
        const uint32_t r = e / TB, c = e % TB;
        const uint64_t i = i0 + r, b = b0 + c;
        const uint64_t oi = bitrev64(i, lg) * cols + b;
        if (b < cols && i < n && ZK_IN_BOUNDS(oi, n * cols, OOB_TRANSPOSE_OUT)) out[oi] = tile[c][r];
    }
}

// The same transpose with 16-byte global accesses: a thread reads two
// consecutive positions of a column and writes two consecutive columns of a
// leaf row.  For an even column count, n >= 2 and 16-byte aligned buffers
// (transpose_rev_device checks).  Measured on B200, 256 x 2^18: 0.196 against
// 0.227 ms for the 8-byte form (5.47 against 4.72 TB/s); a 128-position tile
// measured 0.207 ms, and putting the column blocks first in the grid changed
// nothing.
static __global__ void __launch_bounds__(256) transpose_rev_v2_kernel(const uint64_t *__restrict__ in,
                                                               uint64_t *__restrict__ out, uint32_t lg, uint64_t cols)
{
    constexpr uint32_t TI = 64, TB = 32;
    __shared__ uint64_t tile[TB][TI + 2];
    const uint64_t n = 1ULL << lg;
    const uint64_t i0 = (uint64_t)blockIdx.x * TI;
    const uint64_t b0 = (uint64_t)blockIdx.y * TB;
    for (uint32_t e = threadIdx.x; e < TI * TB / 2; e += 256) {
        const uint32_t r = e / (TI / 2), c = 2 * (e % (TI / 2));
        const uint64_t b = b0 + r, i = i0 + c;
        if (b < cols && i < n && ZK_IN_BOUNDS(b * n + i + 1, n * cols, OOB_TRANSPOSE_IN)) {
            // i even and n even: i + 1 < n too
            const ulonglong2 v = *(const ulonglong2 *)(in + b * n + i);
            tile[r][c] = v.x;
            tile[r][c + 1] = v.y;
        }
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < TI * TB / 2; e += 256) {
        const uint32_t r = e / (TB / 2), c = 2 * (e % (TB / 2));
        const uint64_t i = i0 + r, b = b0 + c;
        const uint64_t oi = bitrev64(i, lg) * cols + b;
        if (b < cols && i < n && ZK_IN_BOUNDS(oi + 1, n * cols, OOB_TRANSPOSE_OUT)) {
            // b even and cols even: b + 1 < cols too
            ulonglong2 v;
            v.x = tile[c][r];
            v.y = tile[c + 1][r];
            *(ulonglong2 *)(out + oi) = v;
        }
    }
}

// The same transpose with the column tiles staged by bulk-async copies:
// persistent CTAs walk the tiles (tile t: positions (t mod tiles_i) * TI,
// columns (t / tiles_i) * TB); warp 0 keeps STAGES tiles in flight, one
// TI * 8-byte cp.async.bulk per column of the tile into a padded row of the
// stage (row pitch TI + 2 words, 16-byte aligned), completed on the stage's
// mbarrier.  The threads then write the tile as bit-reversed leaf rows: a warp
// writes 4 rows x 8 column pairs, 128 contiguous bytes per row, and reads the
// stage without bank conflicts (words 8m + 2r mod 32 over pairs m < 4, rows
// r < 4).  Needs n >= TI, an even column count and 16-byte aligned buffers.  A
// stage that is not complete after wait_ns sets *status and the CTA stops
// (after waiting, bounded again, for the copies it has in flight); extra_tx > 0
// declares that many bytes more than CTA 0's first tile delivers (a test of
// that path).
template <uint32_t TI, uint32_t TB, uint32_t STAGES>
struct TrBulk {
    static constexpr uint32_t THREADS = 256, PITCH = TI + 2, STAGE_WORDS = TB * PITCH;
    static constexpr uint32_t SMEM_BYTES = STAGES * STAGE_WORDS * 8;
    static_assert((PITCH * 8) % 16 == 0 && (STAGE_WORDS * 8) % 16 == 0, "bulk copy destinations must be 16-byte aligned");
    static_assert(TB % 16 == 0 && TI % 4 == 0 && (TI * TB / 2) % THREADS == 0, "tile shape");
};

template <uint32_t TI, uint32_t TB, uint32_t STAGES>
static __global__ void __launch_bounds__(256)
    transpose_rev_bulk_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out, uint32_t lg, uint64_t cols,
                              uint64_t tiles_i, uint64_t n_tiles, unsigned *status, uint32_t extra_tx, uint64_t wait_ns)
{
    using G = TrBulk<TI, TB, STAGES>;
    constexpr uint32_t THREADS = G::THREADS, PITCH = G::PITCH, STAGE_WORDS = G::STAGE_WORDS;
    extern __shared__ __align__(128) uint64_t stage_buf[];
    __shared__ __align__(8) uint64_t full[STAGES];
    const uint64_t n = 1ULL << lg;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
#pragma unroll
        for (uint32_t s = 0; s < STAGES; s++) mbar_init(smem_u32(&full[s]), 1);
        mbar_init_fence();
    }
    __syncthreads();
    // warp 0: local tile k into stage k % STAGES
    auto issue = [&](uint64_t k) {
        const uint64_t t = blockIdx.x + k * gridDim.x;
        if (t >= n_tiles) return;
        const uint32_t s = (uint32_t)(k % STAGES);
        const uint64_t i0 = (t % tiles_i) * TI, b0 = (t / tiles_i) * TB;
        const uint32_t nb = (uint32_t)(cols - b0 < TB ? cols - b0 : TB);
        const uint32_t bar = smem_u32(&full[s]);
        if (lane == 0) mbar_arrive_expect_tx(bar, nb * TI * 8 + (k == 0 && blockIdx.x == 0 ? extra_tx : 0));
        __syncwarp();
        for (uint32_t j = lane; j < nb; j += 32)
            if (ZK_IN_BOUNDS((b0 + j) * n + i0 + TI - 1, n * cols, OOB_TRANSPOSE_IN))
                bulk_load(smem_u32(stage_buf + s * STAGE_WORDS + j * PITCH), in + (b0 + j) * n + i0, TI * 8, bar);
    };
    if (warp == 0) {
#pragma unroll 1
        for (uint32_t k = 0; k < STAGES; k++) issue(k);
    }
    uint64_t k = 0;
    bool failed = false;
#pragma unroll 1
    for (;; k++) {
        const uint64_t t = blockIdx.x + k * gridDim.x;
        if (t >= n_tiles) break;
        const uint32_t s = (uint32_t)(k % STAGES);
        const bool ok = mbar_wait_bounded(smem_u32(&full[s]), (uint32_t)(k / STAGES) & 1, wait_ns);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        const uint64_t i0 = (t % tiles_i) * TI, b0 = (t / tiles_i) * TB;
        const uint64_t *tile = stage_buf + s * STAGE_WORDS;
#pragma unroll
        for (uint32_t q = 0; q < TI * TB / 2 / THREADS; q++) {
            const uint32_t u = tid + q * THREADS, w = u >> 5, l = u & 31;
            const uint32_t r = 4 * (w / (TB / 16)) + (l >> 3), c = 2 * (8 * (w % (TB / 16)) + (l & 7));
            const uint64_t b = b0 + c;
            const uint64_t oi = bitrev64(i0 + r, lg) * cols + b;
            // b even and cols even: b + 1 < cols too
            if (b < cols && ZK_IN_BOUNDS(oi + 1, n * cols, OOB_TRANSPOSE_OUT)) {
                ulonglong2 v;
                v.x = tile[c * PITCH + r];
                v.y = tile[(c + 1) * PITCH + r];
                *(ulonglong2 *)(out + oi) = v;
            }
        }
        __syncthreads();
        if (warp == 0) {
            fence_proxy_async_smem();
            issue(k + STAGES);
        }
    }
    if (failed && tid == 0) {
        atomicAdd_system(status, 1u);
        // the copies still in flight target this CTA's shared memory: wait
        // for them (bounded) before the CTA ends
        for (uint64_t j = k; j < k + STAGES; j++) {
            if (blockIdx.x + j * gridDim.x >= n_tiles) break;
            (void)mbar_wait_bounded(smem_u32(&full[j % STAGES]), (uint32_t)(j / STAGES) & 1, wait_ns / 8);
        }
    }
}

// Multiply every element of a batch of columns by mul (e.g. n^-1) and, when
// tab != null, by tab[i] (i = index within the column).  Used for transforms
// too small for the tiled reorder.
static __global__ void scale_kernel(uint64_t *x, uint64_t n, uint64_t cols, uint64_t mul, const uint64_t *__restrict__ tab)
{
    uint64_t total = n * cols;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = k % n;
        uint64_t v = x[k];
        if (mul != 1) v = gl_mul(v, mul);
        if (tab) v = gl_mul(v, __ldg(tab + i));
        x[k] = v;
    }
}

// tab[t] = w^t for t < count (one square-and-multiply per entry).
static __global__ void powers_kernel(uint64_t *tab, uint64_t count, uint64_t w)
{
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x)
        tab[t] = gl_pow(w, t);
}

// LDE coset table: tab[c * n + j] = (g * w_N^c)^j for c < 2^rate, j < n.
static __global__ void coset_powers_kernel(uint64_t *tab, uint64_t n, uint32_t cosets, uint64_t g, uint64_t wN)
{
    uint64_t total = n * cosets;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t c = k / n, j = k % n;
        uint64_t base = gl_mul(g, gl_pow(wN, c));
        tab[k] = gl_pow(base, j);
    }
}

}  // namespace zk
