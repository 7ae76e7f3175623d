// Field operations of the NTT passes (ntt.cu) and the 8-point DFT built on
// them, in their own header so that other kernels can use them.  All take
// canonical operands (in [0, p)) and return canonical results, equal to
// gl_add, gl_sub and gl_mul of gl64.cuh.
#pragma once
#include <stdint.h>

#include "gl64.cuh"

namespace zk {
namespace ntf {

// Field operations of the transform passes.  The passes are bound by the ALU
// pipe (64-bit adds, subtracts, selects and reduction carries on 32-bit
// halves), while the FMA pipe, which runs the multiply-adds, has room.  So
// these forms take no select and move the folds by 2^64 = 2^32 - 1 (mod p)
// onto multiply-adds: x + k (2^32 - 1) for k in {0, 1} is one mad.wide.u32,
// and r + h (2^32 - 1) with its carry-out is a mad.lo.cc / madc.hi.cc pair.
// Results equal gl_add, gl_sub and gl_mul (canonical in, canonical out).
constexpr uint32_t kLo32 = 0xffffffffu;  // 2^32 - 1 = 2^64 mod p

__device__ __forceinline__ uint64_t fold_k(uint32_t k, uint64_t x) {  // x + k (2^32 - 1) mod 2^64
    uint64_t r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(k), "r"(kLo32), "l"(x));
    return r;
}

// Canonical form of any u64: x >= p exactly when x + (2^32 - 1) carries, and
// then x - p = x + (2^32 - 1) mod 2^64.
__device__ __forceinline__ uint64_t nt_canon(uint64_t x) {
    uint32_t k;
    asm("{\n\t"
        ".reg .u32 t;\n\t"
        "add.cc.u32 t, %1, %3;\n\t"
        "addc.cc.u32 t, %2, 0;\n\t"
        "addc.u32 %0, 0, 0;\n\t"
        "}"
        : "=r"(k)
        : "r"((uint32_t)x), "r"((uint32_t)(x >> 32)), "r"(kLo32));
    return fold_k(k, x);
}

// a - b mod p for canonical a, b.  On a borrow, d + p = d - (2^32 - 1) mod
// 2^64: the low word minus 0xffffffff (that is, plus one), and a borrow from
// the high word exactly when that does not wrap.
__device__ __forceinline__ uint64_t nt_sub(uint64_t a, uint64_t b) {
    uint32_t lo, hi;
    asm("{\n\t"
        ".reg .u32 bw;\n\t"
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.cc.u32 %1, %3, %5;\n\t"
        "subc.u32 bw, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, bw;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(lo), "=r"(hi)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)hi << 32) | lo;
}

// a + b mod p for canonical a, b, as a - (p - b): p - b is in (0, p], and
// nt_sub is exact for a subtrahend of p too (a - p borrows, and the
// correction adds p back), so the sum costs a 64-bit negation and the
// three-instruction subtraction instead of two carry chains and a fold
// (measured per application: 5 instructions, all on the ALU pipe, against 8;
// the 8-point DFT 225 against 258, and the 135 x 2^15 LDE -> leaves 0.613
// against 0.628 ms).
__device__ __forceinline__ uint64_t nt_add(uint64_t a, uint64_t b) { return nt_sub(a, ZK_P - b); }

// (h1, h0, l1, l0) 128-bit -> u64 congruent mod p (not canonical):
// l - h1 (minus 2^32 - 1 on a borrow, as in nt_sub), then + h0 (2^32 - 1)
// with its carry folded once more (it cannot carry again).
__device__ __forceinline__ uint64_t nt_reduce128(uint32_t l0, uint32_t l1, uint32_t h0, uint32_t h1) {
    uint32_t r0, r1, k;
    asm("{\n\t"
        ".reg .u32 b;\n\t"
        "sub.cc.u32 %0, %3, %6;\n\t"
        "subc.cc.u32 %1, %4, 0;\n\t"
        "subc.u32 b, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, b;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "mad.lo.cc.u32 %0, %5, %7, %0;\n\t"
        "madc.hi.cc.u32 %1, %5, %7, %1;\n\t"
        "addc.u32 %2, 0, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(k)
        : "r"(l0), "r"(l1), "r"(h0), "r"(h1), "r"(kLo32));
    return fold_k(k, ((uint64_t)r1 << 32) | r0);
}

__device__ __forceinline__ uint64_t nt_mul(uint64_t a, uint64_t b) {
    uint64_t lo, hi;
    mul_wide(a, b, lo, hi);
    return nt_canon(nt_reduce128((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32)));
}

// Multiplication by the 8th roots of unity.  In this field 2^96 = -1, so 2 has
// order 192 and the 8th roots are powers of 2: for omega_8 = 7^((p-1)/8)
// (the root every table here is built from), omega_8 = 2^120 = -2^24,
// omega_8^2 = omega_4 = 2^48, omega_8^3 = -2^72, and the inverses are 2^72,
// -2^48, 2^24.  None of the three is a 64 x 64 product: x * 2^24 and x * 2^48
// are a shift and one reduction, x * 2^72 is two shifts and a subtraction.
__device__ __forceinline__ uint64_t gl_mul2_24(uint64_t x) {
    // x 2^24 = lo + h 2^64 with h < 2^24: lo + h (2^32 - 1), its carry folded.
    uint32_t r0 = (uint32_t)(x << 24), r1 = (uint32_t)(x >> 8), k;
    asm("{\n\t"
        "mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, 0, 0;\n\t"
        "}"
        : "+r"(r0), "+r"(r1), "=r"(k)
        : "r"((uint32_t)(x >> 40)), "r"(kLo32));
    return nt_canon(fold_k(k, ((uint64_t)r1 << 32) | r0));
}
__device__ __forceinline__ uint64_t gl_mul2_48(uint64_t x) {
    const uint64_t lo = x << 48, hi = x >> 16;
    return nt_canon(nt_reduce128((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32)));
}
// x * 2^72 for canonical x: with x = xh 2^24 + xl (xl < 2^24), 2^96 = -1 gives
// x 2^72 = xl 2^72 - xh = xl (2^40 - 2^8) - xh (mod p), where both
// xl (2^40 - 2^8) and xh are below p.
__device__ __forceinline__ uint64_t gl_mul2_72(uint64_t x) {
    const uint64_t xl = x & 0xffffffull, xh = x >> 24;
    return nt_sub((xl << 40) - (xl << 8), xh);
}

// DIF butterfly with w = 1: (u, v) -> (u + v, u - v).
__device__ __forceinline__ void bfly1(uint64_t &u, uint64_t &v) {
    const uint64_t d = nt_sub(u, v);
    u = nt_add(u, v);
    v = d;
}

// 8-point DFT in place (DIF radix-2 inside, natural order in, bit-reversed
// out), with the direction's 8th roots.  Negated roots swap the operands of
// the subtraction instead of negating.
__device__ __forceinline__ void dft8(uint64_t x[8], bool inv) {
    uint64_t d[4];
    d[0] = nt_sub(x[0], x[4]);
    if (!inv) {
        d[1] = gl_mul2_24(nt_sub(x[5], x[1]));      // (x1 - x5) * (-2^24)
        d[2] = gl_mul2_48(nt_sub(x[2], x[6]));      // (x2 - x6) * 2^48
        d[3] = gl_mul2_72(nt_sub(x[7], x[3]));      // (x3 - x7) * (-2^72)
    } else {
        d[1] = gl_mul2_72(nt_sub(x[1], x[5]));      // * 2^72
        d[2] = gl_mul2_48(nt_sub(x[6], x[2]));      // * (-2^48)
        d[3] = gl_mul2_24(nt_sub(x[3], x[7]));      // * 2^24
    }
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = nt_add(x[k], x[k + 4]);
#pragma unroll
    for (int k = 0; k < 4; k++) x[k + 4] = d[k];
    // span 2: (0,2), (1,3)*omega_4, (4,6), (5,7)*omega_4
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
        const uint64_t a0 = nt_add(x[h], x[h + 2]), a2 = nt_sub(x[h], x[h + 2]);
        const uint64_t a1 = nt_add(x[h + 1], x[h + 3]);
        const uint64_t a3 = inv ? gl_mul2_48(nt_sub(x[h + 3], x[h + 1])) : gl_mul2_48(nt_sub(x[h + 1], x[h + 3]));
        // span 1
        x[h] = nt_add(a0, a1);
        x[h + 1] = nt_sub(a0, a1);
        x[h + 2] = nt_add(a2, a3);
        x[h + 3] = nt_sub(a2, a3);
    }
}

}  // namespace ntf
}  // namespace zk
