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

__device__ __forceinline__ uint64_t gl_canon_fwd(uint64_t x) { return x >= ZK_P ? x - ZK_P : x; }

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

__device__ __forceinline__ uint64_t pr_mul(uint64_t a, uint64_t b);

// Canonical product: the partially reduced product (below) then one
// conditional subtraction.
__device__ __forceinline__ uint64_t gl_mul(uint64_t a, uint64_t b) { return gl_canon_fwd(pr_mul(a, b)); }

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

// ---------------------------------------------------------------------------
// Partially reduced arithmetic for the hash permutations: a value is any u64
// congruent to the field element (so in [0, 2^64), not necessarily < p).
// Results are exact modulo p; callers canonicalise (gl_canon) before storing.
// ---------------------------------------------------------------------------
namespace zk {

// (h1, h0, l1, l0) 128-bit -> u64 congruent mod p:
//   x = (l1:l0) - h1 + h0 * (2^32 - 1).
__device__ __forceinline__ uint64_t pr_reduce128(uint32_t l0, uint32_t l1, uint32_t h0, uint32_t h1) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 b, k;\n\t"
        "sub.cc.u32  %0, %2, %5;\n\t"   // r = (l1:l0) - h1
        "subc.cc.u32 %1, %3, 0;\n\t"
        "subc.u32    b, 0, 0;\n\t"      // b = all-ones on borrow
        "sub.cc.u32  %0, %0, b;\n\t"    // on borrow: r -= EPS (r + p mod 2^64)
        "subc.u32    %1, %1, 0;\n\t"
        "add.cc.u32  %1, %1, %4;\n\t"   // r += h0 * 2^32
        "addc.u32    k, 0, 0;\n\t"
        "sub.cc.u32  %0, %0, %4;\n\t"   // r -= h0
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32    k, k, 0;\n\t"      // k = 1 iff r + h0*EPS overflowed 2^64
        "neg.s32     k, k;\n\t"
        "add.cc.u32  %0, %0, k;\n\t"    // then add 2^64 mod p = EPS
        "addc.u32    %1, %1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(l0), "r"(l1), "r"(h0), "r"(h1));
    return ((uint64_t)r1 << 32) | r0;
}

// a * b for any u64 a, b; result partially reduced.  The 128-bit product
// comes from the 32-bit multiply-add chain of mul_wide (cheaper here than
// 64-bit-accumulating wide multiplies).
__device__ __forceinline__ uint64_t pr_mul(uint64_t a, uint64_t b) {
    uint64_t lo, hi;
    mul_wide(a, b, lo, hi);
    return pr_reduce128((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}

// a * b + c (a, b any u64; c < 2^68 given as (c_lo, c_hi)); partially reduced.
// (a b + c <= (2^64-1)^2 + 2^68 < 2^128, so the sum does not wrap.)
__device__ __forceinline__ uint64_t pr_mul_add(uint64_t a, uint64_t b, uint64_t c_lo, uint32_t c_hi) {
    uint64_t lo, hi;
    mul_wide(a, b, lo, hi);
    uint32_t r0, r1, r2, r3;
    asm("{\n\t"
        "add.cc.u32  %0, %4, %8;\n\t"
        "addc.cc.u32 %1, %5, %9;\n\t"
        "addc.cc.u32 %2, %6, %10;\n\t"
        "addc.u32    %3, %7, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"((uint32_t)lo), "r"((uint32_t)(lo >> 32)), "r"((uint32_t)hi), "r"((uint32_t)(hi >> 32)),
          "r"((uint32_t)c_lo), "r"((uint32_t)(c_lo >> 32)), "r"(c_hi));
    return pr_reduce128(r0, r1, r2, r3);
}

// a + c for any u64 a and c < p: one wrap at most, fixed by adding EPS.
__device__ __forceinline__ uint64_t pr_add_c(uint64_t a, uint64_t c) {
    const uint64_t s = a + c;
    return s < a ? s + ZK_EPS : s;
}

// a^2 as 128 bits from three 32 x 32 products: a0^2, a1^2 and the cross term
// a0 a1, doubled by a funnel shift and added once.  Against mul_wide(a, a)
// it trades two multiplies (the IMAD pipe, the busiest one in the hash
// kernels) for shifts on the ALU pipe, at the same instruction count
// (Poseidon 2^18 x 135 tree 4.342 -> 4.308 ms, Poseidon2 4.398 -> 4.309 ms).
__device__ __forceinline__ void sqr_wide(uint64_t a, uint64_t &lo, uint64_t &hi) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    uint32_t r0, r1, r2, r3;
    asm("{\n\t"
        ".reg .u32 c0, c1, c2;\n\t"
        "mul.lo.u32 %0, %4, %4;\n\t"
        "mul.hi.u32 %1, %4, %4;\n\t"
        "mul.lo.u32 %2, %5, %5;\n\t"
        "mul.hi.u32 %3, %5, %5;\n\t"
        "mul.lo.u32 c0, %4, %5;\n\t"
        "mul.hi.u32 c1, %4, %5;\n\t"
        "shr.u32 c2, c1, 31;\n\t"              // bit 64 of 2 a0 a1
        "shf.l.wrap.b32 c1, c0, c1, 1;\n\t"
        "shl.b32 c0, c0, 1;\n\t"
        "add.cc.u32 %1, %1, c0;\n\t"
        "addc.cc.u32 %2, %2, c1;\n\t"
        "addc.u32 %3, %3, c2;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1));
    lo = ((uint64_t)r1 << 32) | r0;
    hi = ((uint64_t)r3 << 32) | r2;
}
__device__ __forceinline__ uint64_t pr_sqr(uint64_t a) {
    uint64_t lo, hi;
    sqr_wide(a, lo, hi);
    return pr_reduce128((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}

// x^7 with partial reduction (2 squarings, 2 products).
__device__ __forceinline__ uint64_t pr_pow7(uint64_t x) {
    const uint64_t x2 = pr_sqr(x);
    const uint64_t x3 = pr_mul(x, x2);
    const uint64_t x4 = pr_sqr(x2);
    return pr_mul(x3, x4);
}

// al + ah * 2^32 + c for any al, c < 2^64 and ah < 2^64 - 2^33; partially
// reduced.
__device__ __forceinline__ uint64_t pr_reduce_split(uint64_t al, uint64_t ah, uint64_t c) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 k, j;\n\t"
        "add.cc.u32  %0, %2, %6;\n\t"   // r = al + c
        "addc.cc.u32 %1, %3, %7;\n\t"
        "addc.u32    k, 0, 0;\n\t"
        "add.cc.u32  %1, %1, %4;\n\t"   // r += lo32(ah) * 2^32
        "addc.u32    k, k, %5;\n\t"     // k = 2^64 carries + hi32(ah)
        "add.cc.u32  %1, %1, k;\n\t"    // r += k * EPS = k * 2^32 - k
        "addc.u32    j, 0, 0;\n\t"
        "sub.cc.u32  %0, %0, k;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32    j, j, 0;\n\t"      // j = 1 iff that overflowed 2^64
        "neg.s32     j, j;\n\t"
        "add.cc.u32  %0, %0, j;\n\t"
        "addc.u32    %1, %1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"((uint32_t)al), "r"((uint32_t)(al >> 32)), "r"((uint32_t)ah), "r"((uint32_t)(ah >> 32)),
          "r"((uint32_t)c), "r"((uint32_t)(c >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// al + ah * 2^32 for al < 2^64 and ah < 2^64 - 2^33; partially reduced.
__device__ __forceinline__ uint64_t pr_reduce_split_nc(uint64_t al, uint64_t ah) {
    uint32_t r0 = (uint32_t)al, r1;
    asm("{\n\t"
        ".reg .u32 k, j;\n\t"
        "add.cc.u32  %1, %3, %4;\n\t"   // r = al + lo32(ah) * 2^32
        "addc.u32    k, %5, 0;\n\t"     // k = 2^64 carry + hi32(ah)
        "add.cc.u32  %1, %1, k;\n\t"    // r += k * EPS = k * 2^32 - k
        "addc.u32    j, 0, 0;\n\t"
        "sub.cc.u32  %0, %0, k;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32    j, j, 0;\n\t"      // j = 1 iff that overflowed 2^64
        "neg.s32     j, j;\n\t"
        "add.cc.u32  %0, %0, j;\n\t"
        "addc.u32    %1, %1, 0;\n\t"
        "}"
        : "+r"(r0), "=r"(r1)
        : "r"((uint32_t)al), "r"((uint32_t)(al >> 32)), "r"((uint32_t)ah), "r"((uint32_t)(ah >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

}  // namespace zk
