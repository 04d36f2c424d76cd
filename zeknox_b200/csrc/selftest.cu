// selftest.cu -- the device field arithmetic and permutations on caller data.
//
// The hashes and the NTT keep lanes lazily reduced (any 64-bit representative)
// and run their reductions as carry chains whose rare branches -- a wrap, a
// borrow, a second correction -- are taken only near the field's edges: 0,
// p - 1, 2^32 neighbours, 2^64 - 2^32 and the non-canonical range [p, 2^64).
// Seeded uniform data reaches those with probability ~2^-32 per operation, so
// these entry points let a test drive every primitive with chosen operands and
// compare with exact arithmetic, and run whole permutations on chosen states.
// No reference counterpart (the reference's tests call its primitives from a
// test binary, native/tests/tests.cu).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "../../include/zeknox_b200.h"
#include "coop.cuh"
#include "gl64.cuh"
#include "hash.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

namespace {

using namespace zk;

// Output op-major: out[op * n + i] for operands a[i], b[i], c[i].  Operations
// that need canonical operands get gl_canon of them; the others take the raw
// 64-bit words.  Every result is canonicalised.
__global__ void field_selftest_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b,
                                      const uint64_t *__restrict__ c, uint64_t n, uint64_t *__restrict__ out)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t x = a[i], y = b[i], z = c[i];
        const uint64_t xc = gl_canon(x), yc = gl_canon(y);
        uint64_t r[ZK_SELFTEST_OPS];
        r[0] = gl_add(xc, yc);
        r[1] = gl_sub(xc, yc);
        r[2] = ntt_add(xc, yc);
        r[3] = gl_mul(x, y);
        r[4] = gl_canon(gl_mul_nc<true>(x, y));
        r[5] = gl_canon(gl_mul_nc<false>(x, y));
        r[6] = gl_canon(gl_sqr_nc<true>(x));
        r[7] = gl_canon(gl_sqr_nc<false>(x));
        r[8] = gl_canon(gl_mul_add_nc<true>(x, y, z));
        r[9] = gl_canon(gl_mul_add_nc<false>(x, y, z));
        r[10] = gl_canon(gl_sbox7_nc<true, false>(x));
        r[11] = gl_canon(gl_sbox7_nc<true, true>(x));
        r[12] = gl_mul_pow2(x, (unsigned)(z % 192));
        r[13] = gl_canon(gl_add_nc(x, yc));
        {
            // 12 full products: the accumulator's 2^128 overflow counter moves
            WideAcc w;
            w.zero();
#pragma unroll
            for (int k = 0; k < 4; k++) {
                w.mac(x, y);
                w.mac(y, z);
                w.mac(z, x);
            }
            r[14] = gl_canon(w.reduce<true>());
            r[15] = gl_canon(w.reduce<false>());
        }
        {
            Sum64 s;
            s.set(x);
#pragma unroll
            for (int k = 0; k < 5; k++) s.add(y);
#pragma unroll
            for (int k = 0; k < 6; k++) s.add(z);
            r[16] = gl_canon(s.reduce());
        }
        {
            // the largest small-constant dot product the MDS layers form
            Acc96 m;
            m.zero();
#pragma unroll
            for (int k = 0; k < 4; k++) {
                m.mac(x, 41);
                m.mac(y, 39);
                m.mac(z, 34);
            }
            m.add(yc);
            r[17] = gl_canon(m.reduce());
        }
        r[18] = gl_canon(
            p2_combine_pieces((uint32_t)(x & 0xFFFFFFF), (uint32_t)(y & 0xFFFFFFF), (uint32_t)(z & 0xFFFFFFF)));
        r[19] = gl_reduce128(x, y);
        r[20] = gl_reduce96(x, y & 0xFFFFFFFFULL);
        r[21] = gl_mul_pow2_lt64(x, (unsigned)(y % 64));
        // the NTT passes' lazily reduced butterfly arithmetic
        r[22] = gl_canon(ntt_add_nc(x, y));
        r[23] = gl_canon(ntt_sub_nc(x, y));
        r[24] = gl_canon(ntt_mul_pow2_nc<1>(x));
        r[25] = gl_canon(ntt_mul_pow2_nc<24>(x));
        r[26] = gl_canon(ntt_mul_pow2_nc<31>(x));
        r[27] = gl_canon(ntt_mul_pow2_nc<32>(x));
        r[28] = gl_canon(ntt_mul_pow2_nc<60>(x));
        r[29] = gl_canon(ntt_mul_pow2_nc<63>(x));
        r[30] = gl_canon(ntt_mul_pow2_nc<64>(x));
        r[31] = gl_canon(ntt_mul_pow2_nc<72>(x));
        r[32] = gl_canon(ntt_mul_pow2_nc<84>(x));
        r[33] = gl_canon(ntt_mul_pow2_nc<95>(x));
#pragma unroll
        for (int k = 0; k < ZK_SELFTEST_OPS; k++) out[k * n + i] = r[k];
    }
}

// One permutation per thread on 12-word states (Poseidon, Poseidon-BN128,
// Poseidon2, Monolith) or 25-word states (Keccak-f), lanes canonicalised.
template <int H>
__global__ void permute_kernel(uint64_t *states, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if constexpr (H == HASH_KECCAK) {
        uint64_t s[25];
#pragma unroll
        for (int k = 0; k < 25; k++) s[k] = states[i * 25 + k];
        keccak_f(s);
#pragma unroll
        for (int k = 0; k < 25; k++) states[i * 25 + k] = s[k];
    } else {
        uint64_t s[12];
#pragma unroll
        for (int k = 0; k < 12; k++) s[k] = states[i * 12 + k];
        permute<H>(s);
#pragma unroll
        for (int k = 0; k < 12; k++) states[i * 12 + k] = gl_canon(s[k]);
    }
}

// The cooperative form of coop.cuh: a group of four threads per state.  Every
// thread of every warp takes part (full-warp shuffles); groups past n work on
// a zero state and store nothing.
template <int H>
__global__ void permute_coop_kernel(uint64_t *states, uint64_t n)
{
    CoopGroup g;
    g.init();
    const uint64_t st = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 2;
    const bool live = st < n;
    uint64_t s[4];
#pragma unroll
    for (int k = 0; k < 4; k++) s[k] = (live && g.q < 3) ? states[st * 12 + 4 * g.q + k] : 0;
    if (g.q == 3) {
#pragma unroll
        for (int k = 0; k < 4; k++) s[k] = live ? states[st * 12 + k] : 0;  // thread 3 mirrors thread 0
    }
    permute_coop<H>(s, g);
    if (live && g.q < 3) {
#pragma unroll
        for (int k = 0; k < 4; k++) states[st * 12 + 4 * g.q + k] = gl_canon(s[k]);
    }
}

void check_launch(const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw cuda_failure(-(int)e, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" RustError zeknox_field_selftest(size_t device_id, const uint64_t *a, const uint64_t *b, const uint64_t *c,
                                           uint64_t n, uint64_t *out, void *stream)
{
    RustError r{0, nullptr};
    try {
        if (n && (!a || !b || !c || !out)) throw arg_failure("null buffer");
        DeviceCtx &ctx = device(device_id);
        std::lock_guard<std::recursive_mutex> lk(ctx.mu);
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        if (n) {
            const uint64_t blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
            field_selftest_kernel<<<(unsigned)blocks, 256, 0, s>>>(a, b, c, n, out);
            check_launch("field_selftest_kernel");
            note_launch();
        }
        if (!stream) ctx.sync();
    } catch (const std::exception &e) {
        const arg_failure *af = dynamic_cast<const arg_failure *>(&e);
        const cuda_failure *cf = dynamic_cast<const cuda_failure *>(&e);
        r.code = af ? af->code : cf ? cf->code : -(int)cudaErrorUnknown;
        r.message = strdup(e.what());
    }
    return r;
}

extern "C" RustError zeknox_permute(size_t device_id, uint64_t *states, uint64_t n, uint32_t hash_type,
                                    uint32_t cooperative, void *stream)
{
    RustError r{0, nullptr};
    try {
        if (n && !states) throw arg_failure("null buffer");
        if (hash_type > 4) throw arg_failure("unsupported hash_type");
        if (cooperative && hash_type != HASH_POSEIDON && hash_type != HASH_POSEIDON2)
            throw arg_failure("the cooperative form exists for Poseidon (0) and Poseidon2 (3) only");
        DeviceCtx &ctx = device(device_id);
        std::lock_guard<std::recursive_mutex> lk(ctx.mu);
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx.stream;
        if (n) {
            const uint64_t threads = cooperative ? 4 * n : n;
            const unsigned blocks = (unsigned)((threads + 127) / 128);
            if (cooperative) {
                if (hash_type == HASH_POSEIDON) permute_coop_kernel<HASH_POSEIDON><<<blocks, 128, 0, s>>>(states, n);
                else permute_coop_kernel<HASH_POSEIDON2><<<blocks, 128, 0, s>>>(states, n);
            } else {
                switch (hash_type) {
                case HASH_POSEIDON: permute_kernel<HASH_POSEIDON><<<blocks, 128, 0, s>>>(states, n); break;
                case HASH_KECCAK: permute_kernel<HASH_KECCAK><<<blocks, 128, 0, s>>>(states, n); break;
                case HASH_POSEIDON_BN128: permute_kernel<HASH_POSEIDON_BN128><<<blocks, 128, 0, s>>>(states, n); break;
                case HASH_POSEIDON2: permute_kernel<HASH_POSEIDON2><<<blocks, 128, 0, s>>>(states, n); break;
                default: permute_kernel<HASH_MONOLITH><<<blocks, 128, 0, s>>>(states, n); break;
                }
            }
            check_launch("permute_kernel");
            note_launch();
        }
        if (!stream) ctx.sync();
    } catch (const std::exception &e) {
        const arg_failure *af = dynamic_cast<const arg_failure *>(&e);
        const cuda_failure *cf = dynamic_cast<const cuda_failure *>(&e);
        r.code = af ? af->code : cf ? cf->code : -(int)cudaErrorUnknown;
        r.message = strdup(e.what());
    }
    return r;
}
