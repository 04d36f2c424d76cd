// bn254.cuh -- arithmetic in F_r, r the BN254 scalar field order, and the
// Poseidon-BN128 permutation of the Goldilocks sponge built on it.
//
// Replaces zeknox's native/poseidon/element_bn128.cu (4 x 64-bit limb
// Montgomery field, gnark-style) and poseidon_bn128.cu (iden3's optimised
// t = 5 Poseidon with sparse partial rounds) for hash type 2.  Elements here
// are 8 little-endian 32-bit limbs in Montgomery form (x R mod r, R = 2^256),
// always fully reduced (< r), so every representation of a value is the same
// bit pattern as the reference's after conversion.  Multiplication is CIOS
// Montgomery (Koc, Acar, Kaliski 1996) on 32-bit limbs: 32 x 32 -> 64-bit
// multiply-adds, which the device executes as wide integer multiply-adds.
// The same code runs on the host (CPU Merkle builder) and the device.
#pragma once
#include <stdint.h>

#include "gl64.cuh"
#include "zk_constants.h"

namespace zk {

#ifdef __CUDACC__
// the multiply is large (~130 multiply-adds): one out-of-line copy keeps the
// permutation's code within the instruction cache
#define ZK_FR_NOINLINE static __host__ __device__ __noinline__
#define ZK_FR_HD __host__ __device__ __forceinline__
#else
#define ZK_FR_NOINLINE static
#define ZK_FR_HD static inline
#endif

struct Fr {
    uint32_t w[8];
};

#ifdef __CUDACC__
#define ZK_FR_CX __host__ __device__ constexpr
#else
#define ZK_FR_CX constexpr
#endif
ZK_FR_CX uint32_t bn_r_limb(int i)
{
    constexpr uint32_t r[8] = {ZK_BN254_R_LIST};
    return r[i];
}
ZK_FR_CX uint32_t bn_r2_limb(int i)
{
    constexpr uint32_t r2[8] = {ZK_BN254_R2_LIST};
    return r2[i];
}

ZK_FR_HD Fr fr_zero()
{
    Fr z;
#pragma unroll
    for (int i = 0; i < 8; i++) z.w[i] = 0;
    return z;
}

// x - r when x >= r, else x (x < 2r)
ZK_FR_HD Fr fr_reduce_once(const Fr &x)
{
    Fr t;
    uint32_t borrow = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint64_t d = (uint64_t)x.w[i] - bn_r_limb(i) - borrow;
        t.w[i] = (uint32_t)d;
        borrow = (uint32_t)(d >> 63);
    }
    const uint32_t keep = 0u - borrow;  // all ones: x < r, keep x
    Fr z;
#pragma unroll
    for (int i = 0; i < 8; i++) z.w[i] = (x.w[i] & keep) | (t.w[i] & ~keep);
    return z;
}

// a + b, inputs < r (the sum stays below 2r < 2^255)
ZK_FR_HD Fr fr_add(const Fr &a, const Fr &b)
{
    Fr s;
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint64_t t = (uint64_t)a.w[i] + b.w[i] + c;
        s.w[i] = (uint32_t)t;
        c = (uint32_t)(t >> 32);
    }
    return fr_reduce_once(s);
}

// a * b * R^-1 mod r (CIOS); inputs < r, output < r
ZK_FR_NOINLINE Fr fr_mul(const Fr a, const Fr b)
{
    uint32_t t[10];
#pragma unroll
    for (int j = 0; j < 10; j++) t[j] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint64_t p = (uint64_t)a.w[i] * b.w[j] + t[j] + c;
            t[j] = (uint32_t)p;
            c = p >> 32;
        }
        uint64_t s = (uint64_t)t[8] + c;
        t[8] = (uint32_t)s;
        t[9] = (uint32_t)(s >> 32);
        const uint32_t m = t[0] * ZK_BN254_NP;
        uint64_t p = (uint64_t)m * bn_r_limb(0) + t[0];
        c = p >> 32;
#pragma unroll
        for (int j = 1; j < 8; j++) {
            p = (uint64_t)m * bn_r_limb(j) + t[j] + c;
            t[j - 1] = (uint32_t)p;
            c = p >> 32;
        }
        s = (uint64_t)t[8] + c;
        t[7] = (uint32_t)s;
        t[8] = t[9] + (uint32_t)(s >> 32);
    }
    // t < 2r < 2^255: t[8] is zero
    Fr z;
#pragma unroll
    for (int i = 0; i < 8; i++) z.w[i] = t[i];
    return fr_reduce_once(z);
}

ZK_FR_HD Fr fr_exp5(const Fr &x)
{
    const Fr x2 = fr_mul(x, x);
    const Fr x4 = fr_mul(x2, x2);
    return fr_mul(x4, x);
}

// Sums of products reduced once (the matrix layers' dot products): a 512-bit
// accumulator of products of elements < r, then one Montgomery reduction.
// For at most five products the sum is below 5 r^2 < 2^510 and the reduced
// value (sum + m r) / 2^256 below (5r / 2^256 + 1) r < 2r, so one conditional
// subtraction makes it canonical: the same value as five fr_mul and four
// fr_add, for one reduction instead of five.
struct FrWide {
    uint32_t w[16];
};

ZK_FR_HD void fr_wide_zero(FrWide &t)
{
#pragma unroll
    for (int i = 0; i < 16; i++) t.w[i] = 0;
}

// t += a * b  (t stays below 2^512 for the sums above)
ZK_FR_HD void fr_mac_wide(FrWide &t, const Fr &a, const Fr &b)
{
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint64_t p = (uint64_t)a.w[i] * b.w[j] + t.w[i + j] + c;
            t.w[i + j] = (uint32_t)p;
            c = p >> 32;
        }
#pragma unroll
        for (int k = i + 8; k < 16; k++) {
            const uint64_t s = (uint64_t)t.w[k] + c;
            t.w[k] = (uint32_t)s;
            c = s >> 32;
        }
    }
}

// t * R^-1 mod r for t < 5 r^2, canonical
ZK_FR_HD Fr fr_reduce_wide(FrWide t)
{
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t m = t.w[i] * ZK_BN254_NP;
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint64_t p = (uint64_t)m * bn_r_limb(j) + t.w[i + j] + c;
            t.w[i + j] = (uint32_t)p;
            c = p >> 32;
        }
#pragma unroll
        for (int k = i + 8; k < 16; k++) {
            const uint64_t s = (uint64_t)t.w[k] + c;
            t.w[k] = (uint32_t)s;
            c = s >> 32;
        }
    }
    Fr z;
#pragma unroll
    for (int i = 0; i < 8; i++) z.w[i] = t.w[8 + i];
    return fr_reduce_once(z);
}

// Out-of-line copies of the two steps: a permutation that takes many dot
// products then holds one copy of their code (the instruction cache).
ZK_FR_NOINLINE FrWide fr_mac_wide_ol(FrWide t, const Fr a, const Fr b)
{
    fr_mac_wide(t, a, b);
    return t;
}

ZK_FR_NOINLINE Fr fr_reduce_wide_ol(const FrWide t) { return fr_reduce_wide(t); }

// Montgomery form of a value < r given as plain limbs, and back
ZK_FR_HD Fr fr_to_mont(const Fr &x)
{
    Fr r2;
#pragma unroll
    for (int i = 0; i < 8; i++) r2.w[i] = bn_r2_limb(i);
    return fr_mul(x, r2);
}

ZK_FR_HD Fr fr_from_mont(const Fr &x)
{
    Fr one = fr_zero();
    one.w[0] = 1;
    return fr_mul(x, one);
}

}  // namespace zk
