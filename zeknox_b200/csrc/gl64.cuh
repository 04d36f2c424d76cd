// gl64.cuh -- Goldilocks field arithmetic, p = 2^64 - 2^32 + 1.
//
// Replaces native/ff/gl64_t.cuh (device) and native/ff/goldilocks.hpp (host)
// of zeknox.  Written from the field's structure:
//     2^64 = 2^32 - 1 =: EPS (mod p)        2^96 = -1 (mod p)
// so a 128-bit value  lo + 2^64 (h0 + 2^32 h1)  reduces to  lo + EPS*h0 - h1.
// 2 has multiplicative order 192, so multiplying by 2^s is a shift followed by
// that reduction; every 64th root of unity is a power of 2.
//
// All functions take and return canonical values (< p) unless their name says
// otherwise.  They compile for host and device; the device path uses the
// 64x64->128 multiply-high intrinsic, the host path unsigned __int128.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define ZK_HD __host__ __device__ __forceinline__
#else
#define ZK_HD inline
#endif

namespace zk {

static constexpr uint64_t GL_P = 0xFFFFFFFF00000001ULL;
static constexpr uint64_t GL_EPS = 0xFFFFFFFFULL;  // 2^64 mod p

ZK_HD uint64_t mulhi64(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// a + b for canonical a, b.  If the 64-bit sum wraps, the true sum minus p is
// sum + EPS (no second wrap); otherwise subtract p when sum >= p, which is
// exactly when sum + EPS wraps.
ZK_HD uint64_t gl_add(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    uint32_t r0, r1, t0, t1, c;
    asm("{\n\t"
        "add.cc.u32   %0, %5, %7;\n\t"
        "addc.cc.u32  %1, %6, %8;\n\t"
        "addc.u32     %4, 0, 0;\n\t"
        "add.cc.u32   %2, %0, 0xffffffff;\n\t"
        "addc.cc.u32  %3, %1, 0;\n\t"
        "addc.u32     %4, %4, 0;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(t0), "=&r"(t1), "=&r"(c)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return c ? (((uint64_t)t1 << 32) | t0) : (((uint64_t)r1 << 32) | r0);
#else
    uint64_t s = a + b;
    uint64_t t = s + GL_EPS;
    bool c1 = s < a;
    bool c2 = t < s;
    return (c1 | c2) ? t : s;
#endif
}

// a - b for canonical a, b: a borrow means a - b + 2^64, fix by adding p.
ZK_HD uint64_t gl_sub(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    uint32_t r0, r1, m, m1;
    asm("{\n\t"
        "sub.cc.u32   %0, %4, %6;\n\t"
        "subc.cc.u32  %1, %5, %7;\n\t"
        "subc.u32     %2, 0, 0;\n\t"
        "and.b32      %3, %2, 1;\n\t"
        "add.cc.u32   %0, %0, %3;\n\t"
        "addc.u32     %1, %1, %2;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(m), "=&r"(m1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
#else
    uint64_t d = a - b;
    return (a < b) ? d - GL_EPS : d;
#endif
}

ZK_HD uint64_t gl_neg(uint64_t a) { return a ? GL_P - a : 0; }

ZK_HD uint64_t gl_canon(uint64_t a) { return a >= GL_P ? a - GL_P : a; }

// Reduce lo + 2^64*hi (any 128-bit value) to a canonical element.
ZK_HD uint64_t gl_reduce128(uint64_t lo, uint64_t hi)
{
    uint64_t h1 = hi >> 32;
    uint64_t h0 = hi & GL_EPS;
    uint64_t t0 = lo - h1;
    if (lo < h1) t0 -= GL_EPS;                  // lo - h1 + p, already < p
    uint64_t t1 = (h0 << 32) - h0;              // h0 * EPS < p
    uint64_t t2 = t0 + t1;
    if (t2 < t1) t2 += GL_EPS;                  // wrapped: t0 + t1 - p < 2^64
    return gl_canon(t2);
}

// Reduce lo + 2^64*hi with hi < 2^32 (a "u96" value) to a 64-bit
// representative (_nc) or the canonical value.
ZK_HD uint64_t gl_reduce96_nc(uint64_t lo, uint64_t hi)
{
    uint64_t t1 = (hi << 32) - hi;              // hi * EPS < p
    uint64_t t2 = lo + t1;
    if (t2 < t1) t2 += GL_EPS;                  // wrapped: lo + t1 - p < 2^64
    return t2;
}
ZK_HD uint64_t gl_reduce96(uint64_t lo, uint64_t hi) { return gl_canon(gl_reduce96_nc(lo, hi)); }

// ------------------------------------------------------------------------
// Lazily reduced arithmetic ("nc" = any 64-bit representative, not
// necessarily < p).  On the device these are 32-bit PTX carry chains: the
// 64x64 product is 8 multiply-adds, the reduction of lo + 2^64*(h0 + 2^32*h1)
// to lo - h1 + EPS*h0 is one wide multiply and 10 integer ops (or 13 integer
// ops in the all-ALU form) with no compares or selects.

#ifdef __CUDACC__
__device__ __forceinline__ void mul_wide(uint64_t a, uint64_t b, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    asm("{\n\t"
        "mul.lo.u32      %0, %4, %6;\n\t"
        "mul.hi.u32      %1, %4, %6;\n\t"
        "mad.lo.cc.u32   %1, %5, %6, %1;\n\t"
        "madc.hi.u32     %2, %5, %6, 0;\n\t"
        "mad.lo.cc.u32   %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32  %2, %4, %7, %2;\n\t"
        "addc.u32        %3, 0, 0;\n\t"
        "mad.lo.cc.u32   %2, %5, %7, %2;\n\t"
        "madc.hi.u32     %3, %5, %7, %3;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void sqr_wide(uint64_t a, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    // a^2 = a0^2 + 2^33 a0 a1 + 2^64 a1^2
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    uint32_t m0, m1;
    asm("{\n\t"
        "mul.lo.u32      %4, %6, %7;\n\t"
        "mul.hi.u32      %5, %6, %7;\n\t"
        "mul.lo.u32      %0, %6, %6;\n\t"
        "mul.hi.u32      %1, %6, %6;\n\t"
        "mul.lo.u32      %2, %7, %7;\n\t"
        "mul.hi.u32      %3, %7, %7;\n\t"
        "add.cc.u32      %1, %1, %4;\n\t"
        "addc.cc.u32     %2, %2, %5;\n\t"
        "addc.u32        %3, %3, 0;\n\t"
        "add.cc.u32      %1, %1, %4;\n\t"
        "addc.cc.u32     %2, %2, %5;\n\t"
        "addc.u32        %3, %3, 0;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3), "=&r"(m0), "=&r"(m1)
        : "r"(a0), "r"(a1));
}

// r1:r0 + 2^64 (r2 + 2^32 r3)  ->  64-bit representative, all on the integer
// ALU: lo - r3 + r2 * EPS with the borrow / carry folded in.
__device__ __forceinline__ uint64_t reduce_nc_alu(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3)
{
    uint32_t t0, t1, b, e0, e1, c;
    asm("{\n\t"
        "sub.cc.u32      %0, %6, %9;\n\t"   // t = lo - h1
        "subc.cc.u32     %1, %7, 0;\n\t"
        "subc.u32        %2, 0, 0;\n\t"     // b = borrow ? 0xffffffff : 0
        "sub.cc.u32      %0, %0, %2;\n\t"   // borrow: t -= EPS (t + 1 - 2^32)
        "subc.u32        %1, %1, 0;\n\t"
        "sub.cc.u32      %3, 0, %8;\n\t"    // e = h0 * EPS = 2^32 h0 - h0
        "subc.u32        %4, %8, 0;\n\t"
        "add.cc.u32      %0, %0, %3;\n\t"   // t += e
        "addc.cc.u32     %1, %1, %4;\n\t"
        "addc.u32        %5, 0, 0;\n\t"     // c = carry
        "neg.s32         %5, %5;\n\t"       // carry: t += EPS
        "add.cc.u32      %0, %0, %5;\n\t"
        "addc.u32        %1, %1, 0;\n\t"
        "}"
        : "=&r"(t0), "=&r"(t1), "=&r"(b), "=&r"(e0), "=&r"(e1), "=&r"(c)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return ((uint64_t)t1 << 32) | t0;
}

// The same reduction with r2 * EPS taken by one wide multiply (the multiply
// pipe) and three fewer ALU instructions: (top:t) = (r1:r0) + r2 * EPS - r3
// with a signed top limb in {-1, 0, 1}, then one correction t + top * EPS
// (2^64 = EPS mod p; +EPS cannot wrap again because t <= 2^64 - 2^33 when
// top = 1, and t >= 2^64 - 2^32 when top = -1).  The default of the lazy
// products below: measured 1.03-1.05x on the Poseidon, Poseidon2 and Monolith
// forests and 1.02-1.03x on the NTT passes on B200, whose integer ALU is the
// busier pipe in all of them (the all-ALU form stays for comparison and the
// multiply-rate probe).
__device__ __forceinline__ uint64_t reduce_nc_imad(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3)
{
    uint64_t e;
    asm("mul.wide.u32 %0, %1, 0xffffffff;" : "=l"(e) : "r"(r2));
    uint32_t t0, t1, top, cl, ch;
    asm("{\n\t"
        "add.cc.u32      %0, %5, %7;\n\t"   // t = lo + r2 * EPS
        "addc.cc.u32     %1, %6, %8;\n\t"
        "addc.u32        %2, 0, 0;\n\t"
        "sub.cc.u32      %0, %0, %9;\n\t"   // - r3
        "subc.cc.u32     %1, %1, 0;\n\t"
        "subc.u32        %2, %2, 0;\n\t"    // top in {-1, 0, 1}
        "neg.s32         %3, %2;\n\t"       // top * EPS mod 2^64 = (-top) + 2^32 * (top >> 31)
        "shr.s32         %4, %2, 31;\n\t"
        "add.cc.u32      %0, %0, %3;\n\t"
        "addc.u32        %1, %1, %4;\n\t"
        "}"
        : "=&r"(t0), "=&r"(t1), "=&r"(top), "=&r"(cl), "=&r"(ch)
        : "r"(r0), "r"(r1), "r"((uint32_t)e), "r"((uint32_t)(e >> 32)), "r"(r3));
    return ((uint64_t)t1 << 32) | t0;
}

template <bool IMAD = true>
__device__ __forceinline__ uint64_t reduce_nc(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3)
{
    return IMAD ? reduce_nc_imad(r0, r1, r2, r3) : reduce_nc_alu(r0, r1, r2, r3);
}
#endif

// a * b for any 64-bit representatives; result any 64-bit representative.
template <bool IMAD = true>
ZK_HD uint64_t gl_mul_nc(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    uint32_t r0, r1, r2, r3;
    mul_wide(a, b, r0, r1, r2, r3);
    return reduce_nc<IMAD>(r0, r1, r2, r3);
#else
    unsigned __int128 x = (unsigned __int128)a * b;
    return gl_reduce128((uint64_t)x, (uint64_t)(x >> 64));
#endif
}

template <bool IMAD = true>
ZK_HD uint64_t gl_sqr_nc(uint64_t a)
{
#ifdef __CUDA_ARCH__
    uint32_t r0, r1, r2, r3;
    sqr_wide(a, r0, r1, r2, r3);
    return reduce_nc<IMAD>(r0, r1, r2, r3);
#else
    return gl_mul_nc(a, a);
#endif
}

// a * b + c (c any 64-bit value) reduced once.
template <bool IMAD = true>
ZK_HD uint64_t gl_mul_add_nc(uint64_t a, uint64_t b, uint64_t c)
{
#ifdef __CUDA_ARCH__
    // c enters the first partial product's chain (a*b + c < 2^128)
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t r0, r1, r2, r3;
    asm("{\n\t"
        "mad.lo.cc.u32   %0, %4, %6, %8;\n\t"
        "madc.hi.cc.u32  %1, %4, %6, %9;\n\t"
        "addc.u32        %2, 0, 0;\n\t"
        "mad.lo.cc.u32   %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32  %2, %5, %6, %2;\n\t"
        "addc.u32        %3, 0, 0;\n\t"
        "mad.lo.cc.u32   %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32  %2, %4, %7, %2;\n\t"
        "addc.u32        %3, %3, 0;\n\t"
        "mad.lo.cc.u32   %2, %5, %7, %2;\n\t"
        "madc.hi.u32     %3, %5, %7, %3;\n\t"
        "}"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1), "r"((uint32_t)c), "r"((uint32_t)(c >> 32)));
    return reduce_nc<IMAD>(r0, r1, r2, r3);
#else
    unsigned __int128 x = (unsigned __int128)a * b + c;
    return gl_reduce128((uint64_t)x, (uint64_t)(x >> 64));
#endif
}

// Sum of fewer than 2^32 - 1 full 128-bit products, reduced once: value =
// limbs + 2^128 * top, and 2^128 = 2^96 * 2^32 = -2^32 (mod p).
struct WideAcc {
#ifdef __CUDA_ARCH__
    uint32_t r0, r1, r2, r3, top;
#else
    uint64_t lo, hi;
    uint32_t top;
#endif
    ZK_HD void zero()
    {
#ifdef __CUDA_ARCH__
        r0 = r1 = r2 = r3 = top = 0;
#else
        lo = hi = 0;
        top = 0;
#endif
    }
    // += a * b (any 64-bit representatives)
    ZK_HD void mac(uint64_t a, uint64_t b)
    {
#ifdef __CUDA_ARCH__
        uint32_t p0, p1, p2, p3;
        mul_wide(a, b, p0, p1, p2, p3);
        asm("{\n\t"
            "add.cc.u32   %0, %0, %5;\n\t"
            "addc.cc.u32  %1, %1, %6;\n\t"
            "addc.cc.u32  %2, %2, %7;\n\t"
            "addc.cc.u32  %3, %3, %8;\n\t"
            "addc.u32     %4, %4, 0;\n\t"
            "}"
            : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(top)
            : "r"(p0), "r"(p1), "r"(p2), "r"(p3));
#else
        const unsigned __int128 x = (unsigned __int128)a * b;
        const unsigned __int128 s = (((unsigned __int128)hi << 64) | lo) + x;
        top += s < x;
        lo = (uint64_t)s;
        hi = (uint64_t)(s >> 64);
#endif
    }
    // any 64-bit representative of the sum
    template <bool IMAD = true>
    ZK_HD uint64_t reduce() const
    {
#ifdef __CUDA_ARCH__
        const uint64_t t = reduce_nc<IMAD>(r0, r1, r2, r3);
#else
        const uint64_t t = gl_reduce128(lo, hi);
#endif
        // t - top * 2^32; when it borrows, t - x + p is in [0, 2^64) because
        // x = top * 2^32 <= p
        const uint64_t x = (uint64_t)top << 32;
        const uint64_t d = t - x;
        return t < x ? d - GL_EPS : d;
    }
};

// a + b where at least one operand is < p: one wrap correction suffices
// (a + b - 2^64 + EPS = a + b - p < 2^64).
ZK_HD uint64_t gl_add_nc(uint64_t a, uint64_t b)
{
    uint64_t s = a + b;
    return s + (s < a ? GL_EPS : 0);
}

ZK_HD uint64_t gl_mul(uint64_t a, uint64_t b) { return gl_canon(gl_mul_nc(a, b)); }

ZK_HD uint64_t gl_sqr(uint64_t a) { return gl_canon(gl_sqr_nc(a)); }

// a * 2^s for 0 <= s < 64: the 128-bit shift then the special reduction.  On
// the device the shift is two wide multiplies of a's 32-bit halves by
// 2^(s mod 32) -- the multiply pipe, which the NTT passes leave mostly idle,
// instead of 64-bit shifts on the integer ALU they are bound by -- and the
// reduction knows which limbs are zero: for s < 32 the value is below 2^96
// (lo + EPS * r2), for s >= 32 its low word is 0.  a may be any 64-bit word
// (like gl_mul); the result is canonical.
ZK_HD uint64_t gl_mul_pow2_lt64(uint64_t a, unsigned s)
{
    if (s == 0) return gl_canon(a);
#ifdef __CUDA_ARCH__
    const uint32_t m = 1u << (s & 31);
    uint32_t q0, q1, q2;  // a * m = q0 + 2^32 q1 + 2^64 q2
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
    if (s < 32) {
        // q0 + 2^32 q1 + EPS q2, one correction (no second wrap: the sum is < 2^65 - 2^33)
        uint64_t e;
        asm("mul.wide.u32 %0, %1, 0xffffffff;" : "=l"(e) : "r"(q2));
        asm("{\n\t"
            ".reg .u32 top;\n\t"
            "add.cc.u32      %0, %2, %4;\n\t"
            "addc.cc.u32     %1, %3, %5;\n\t"
            "addc.u32        top, 0, 0;\n\t"
            "neg.s32         top, top;\n\t"
            "add.cc.u32      %0, %0, top;\n\t"
            "addc.u32        %1, %1, 0;\n\t"
            "}"
            : "=&r"(t0), "=&r"(t1)
            : "r"(q0), "r"(q1), "r"((uint32_t)e), "r"((uint32_t)(e >> 32)));
    } else {
        // 2^32 q0 + EPS q1 - q2 with a signed top limb, as reduce_nc_imad
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
    }
    return gl_canon(((uint64_t)t1 << 32) | t0);
#else
    return gl_reduce128(a << s, a >> (64 - s));
#endif
}

// a * 2^s for any s (taken mod 192, the order of 2) and any 64-bit word a;
// canonical result.  2^96 = -1 turns
// s >= 96 into a negation; for 64 <= s < 96, 2^s = 2^(s-32) - 2^(s-64)
// because 2^64 = 2^32 - 1.
ZK_HD uint64_t gl_mul_pow2(uint64_t a, unsigned s)
{
    s %= 192;
    bool neg = s >= 96;
    if (neg) s -= 96;
    // 64 <= s < 96: one multiply by the constant 2^s mod p (2^s = 2^(s-32) - 2^(s-64))
    uint64_t r = s < 64 ? gl_mul_pow2_lt64(a, s)
                        : gl_mul(a, ((1ULL << (s - 32)) - (1ULL << (s - 64))));
    return neg ? gl_neg(r) : r;
}



ZK_HD uint64_t gl_pow(uint64_t a, uint64_t e)
{
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = gl_mul(r, a);
        a = gl_mul(a, a);
        e >>= 1;
    }
    return r;
}

ZK_HD uint64_t gl_inv(uint64_t a) { return gl_pow(a, GL_P - 2); }

// x^7, the Poseidon/Poseidon2 S-box: x^2, x^4, x^3 = x^2 * x, x^7 = x^3 * x^4.
ZK_HD uint64_t gl_sbox7(uint64_t x)
{
    uint64_t x2 = gl_sqr(x);
    uint64_t x4 = gl_sqr(x2);
    uint64_t x3 = gl_mul(x2, x);
    return gl_mul(x3, x4);
}

// Same S-box on lazily reduced values.  SQR selects the dedicated squaring
// product (6 multiplies + 6 adds, fewer on the multiply pipe) for x^2 and x^4
// over the general one (8 multiply-adds): measured 1.005x on Poseidon2 forests,
// whose leaf kernel is bound by the multiply pipe, and 0.98x on Poseidon's.
template <bool IMAD = true, bool SQR = false>
ZK_HD uint64_t gl_sbox7_nc(uint64_t x)
{
    uint64_t x2 = SQR ? gl_sqr_nc<IMAD>(x) : gl_mul_nc<IMAD>(x, x);
    uint64_t x4 = SQR ? gl_sqr_nc<IMAD>(x2) : gl_mul_nc<IMAD>(x2, x2);
    uint64_t x3 = gl_mul_nc<IMAD>(x2, x);
    return gl_mul_nc<IMAD>(x3, x4);
}

ZK_HD uint32_t bitrev32(uint32_t x, unsigned bits)
{
#ifdef __CUDA_ARCH__
    return bits ? __brev(x) >> (32 - bits) : 0;
#else
    uint32_t r = 0;
    for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
#endif
}

ZK_HD uint64_t bitrev64(uint64_t x, unsigned bits)
{
#ifdef __CUDA_ARCH__
    return bits ? __brevll(x) >> (64 - bits) : 0;
#else
    uint64_t r = 0;
    for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1ULL) << (bits - 1 - i);
    return r;
#endif
}

}  // namespace zk
