// Goldilocks field arithmetic, p = 2^64 - 2^32 + 1, for sm_100a.
//
// Every value handed between functions is canonical (in [0, p)), so results
// are bit-identical to zeknox's gl64_t (native/ff/gl64_t.cuh:93-369) and
// cpp_gl64_t (native/ff/goldilocks.hpp:139-177), whose outputs are canonical
// for canonical inputs.  The 64x64 -> 128-bit product is formed from 32-bit
// IMAD chains; the reduction uses 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
#pragma once
#include <stdint.h>

#define ZK_P 0xffffffff00000001ull
#define ZK_EPS 0x00000000ffffffffull  // 2^64 mod p

namespace zk {

// a + b mod p for a, b < p.  With s = a + b (mod 2^64) the result is s + EPS
// (mod 2^64) exactly when the sum carried out or s >= p (i.e. s + EPS carries).
__device__ __forceinline__ uint64_t gl_add(uint64_t a, uint64_t b) {
    uint64_t s, t;
    uint32_t c;
    asm("{\n\t"
        ".reg .u32 c0;\n\t"
        "add.cc.u64 %0, %3, %4;\n\t"
        "addc.u32 c0, 0, 0;\n\t"
        "add.cc.u64 %1, %0, %5;\n\t"
        "addc.u32 %2, c0, 0;\n\t"
        "}"
        : "=l"(s), "=l"(t), "=r"(c)
        : "l"(a), "l"(b), "l"(ZK_EPS));
    return c ? t : s;
}

// a - b mod p for a, b < p: on borrow add p, i.e. subtract EPS.
__device__ __forceinline__ uint64_t gl_sub(uint64_t a, uint64_t b) {
    uint64_t d;
    uint32_t bw;
    asm("{\n\t"
        "sub.cc.u64 %0, %2, %3;\n\t"
        "subc.u32 %1, 0, 0;\n\t"
        "}"
        : "=l"(d), "=r"(bw)
        : "l"(a), "l"(b));
    return bw ? d - ZK_EPS : d;
}

// Reduce the 128-bit value (hi, lo) to canonical form.
// x = lo + 2^64 (hl + 2^32 hh) = lo - hh + hl (2^32 - 1)  (mod p).
__device__ __forceinline__ uint64_t gl_reduce128(uint64_t lo, uint64_t hi) {
    uint32_t hl = (uint32_t)hi, hh = (uint32_t)(hi >> 32);
    uint64_t t0;
    uint32_t bw;
    asm("{\n\t"
        "sub.cc.u64 %0, %2, %3;\n\t"
        "subc.u32 %1, 0, 0;\n\t"
        "}"
        : "=l"(t0), "=r"(bw)
        : "l"(lo), "l"((uint64_t)hh));
    if (bw) t0 -= ZK_EPS;                      // t0 in [p - 2^32 + 1, p) after a borrow
    uint64_t t1 = ((uint64_t)hl << 32) - hl;   // hl * EPS <= p - 2^32
    uint64_t r;
    uint32_t c;
    asm("{\n\t"
        "add.cc.u64 %0, %2, %3;\n\t"
        "addc.u32 %1, 0, 0;\n\t"
        "}"
        : "=l"(r), "=r"(c)
        : "l"(t0), "l"(t1));
    if (c) r += ZK_EPS;                        // cannot carry again: r < p - 2^32 here
    return r >= ZK_P ? r - ZK_P : r;
}

// Full 64 x 64 -> 128-bit product from 32-bit limbs.
__device__ __forceinline__ void mul_wide(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
    uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t r0, r1, r2, r3;
    asm("{\n\t"
        "mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mul.lo.u32 %2, %5, %7;\n\t"
        "mul.hi.u32 %3, %5, %7;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %4, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    lo = ((uint64_t)r1 << 32) | r0;
    hi = ((uint64_t)r3 << 32) | r2;
}

__device__ __forceinline__ uint64_t gl_mul(uint64_t a, uint64_t b) {
    uint64_t lo, hi;
    mul_wide(a, b, lo, hi);
    return gl_reduce128(lo, hi);
}

__device__ __forceinline__ uint64_t gl_sqr(uint64_t a) { return gl_mul(a, a); }

// Reduce a value below 2^96 held as (lo, hi32): lo + hi32 * EPS (mod p).
__device__ __forceinline__ uint64_t gl_reduce96(uint64_t lo, uint32_t hi32) {
    uint64_t t1 = ((uint64_t)hi32 << 32) - hi32;  // hi32 * EPS
    uint64_t r;
    uint32_t c;
    asm("{\n\t"
        "add.cc.u64 %0, %2, %3;\n\t"
        "addc.u32 %1, 0, 0;\n\t"
        "}"
        : "=l"(r), "=r"(c)
        : "l"(lo), "l"(t1));
    if (c) r += ZK_EPS;  // lo + t1 - 2^64 < 2^64 - 2^32, so this cannot carry
    return r >= ZK_P ? r - ZK_P : r;
}

// x^7, the S-box of both Poseidon variants.
__device__ __forceinline__ uint64_t gl_pow7(uint64_t x) {
    uint64_t x2 = gl_sqr(x);
    uint64_t x3 = gl_mul(x, x2);
    uint64_t x4 = gl_sqr(x2);
    return gl_mul(x3, x4);
}

// Canonical representative of an arbitrary u64.
__device__ __forceinline__ uint64_t gl_canon(uint64_t x) { return x >= ZK_P ? x - ZK_P : x; }

}  // namespace zk
