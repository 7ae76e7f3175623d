// Device hashers of the Merkle path: Poseidon, Poseidon2 (Goldilocks, width
// 12) and Keccak-256 over Goldilocks words, each one thread per hash with the
// whole state in registers.
//
// Semantics follow zeknox:
//   Poseidon   native/poseidon/poseidon.cu:602-791 (4 full, 22 partial,
//              4 full rounds; x^7; MDS circulant + diag(8,0..0))
//   Poseidon2  native/poseidon2/poseidon2.cu:61-209
//   Keccak     native/keccak/keccak.cu:42-135 (rate 136 B, 0x01 .. 0x80 pad,
//              digest word 3 masked to its low byte)
//   sponge     native/poseidon/poseidon_permutation.cuh:226-276 (rate 8,
//              overwrite mode, n <= 4 copies and zero-pads)
#pragma once
#include <stdint.h>

#include "gl64.cuh"
#include "zk_constants.h"

namespace zk {

__constant__ uint64_t c_poseidon_rc[360] = {ZK_POSEIDON_RC_LIST};
__constant__ uint64_t c_poseidon2_rc[360] = {ZK_POSEIDON2_RC_LIST};
__constant__ uint64_t c_poseidon2_diag[12] = {ZK_POSEIDON2_DIAG_LIST};
__constant__ uint64_t c_keccak_rc[24] = {ZK_KECCAK_RC_LIST};

// out = M * x (+ c) for a 12x12 matrix of small non-negative integer
// coefficients (row sums < 2^9).  The 32-bit halves of x are converted to
// doubles and each row is accumulated with FP64 multiply-adds: every product
// and partial sum is an integer below 276 * 2^32 < 2^41 < 2^53, so the FP64
// arithmetic is exact.  This moves the 288 multiply-adds of a layer onto the
// FP64 pipe (full rate on sm_100), next to the integer pipes that carry the
// S-box products.  Each row is then reduced once, adding c[r] (the next
// round's constants; c == nullptr adds nothing).  Inputs and outputs are
// partially reduced.  coef(r, c) must be a constant expression after unrolling.
template <class Coef>
__device__ __forceinline__ void small_matvec12(uint64_t s[12], Coef coef, const uint64_t *c) {
    double lo[12], hi[12];
#pragma unroll
    for (int i = 0; i < 12; i++) {
        lo[i] = __uint2double_rn((uint32_t)s[i]);
        hi[i] = __uint2double_rn((uint32_t)(s[i] >> 32));
    }
#pragma unroll
    for (int r = 0; r < 12; r++) {
        double al = 0.0, ah = 0.0;
#pragma unroll
        for (int k = 0; k < 12; k++) {
            const uint32_t m = coef(r, k);
            if (m) {
                al = fma((double)m, lo[k], al);
                ah = fma((double)m, hi[k], ah);
            }
        }
        s[r] = pr_reduce_split(__double2ull_rz(al), __double2ull_rz(ah), c ? c[r] : 0ull);
    }
}

// ------------------------------------------------------------ Poseidon
struct PoseidonMds {
    __device__ __forceinline__ uint32_t operator()(int r, int c) const {
        constexpr uint32_t circ[12] = {ZK_POSEIDON_MDS_CIRC_LIST};
        constexpr uint32_t diag[12] = {ZK_POSEIDON_MDS_DIAG_LIST};
        return circ[(c - r + 12) % 12] + (r == c ? diag[r] : 0u);
    }
};

// x^7 on all 12 lanes, as three passes over 4 lanes with a rotation between
// them (keeps the loop body, and so the instruction footprint, small).
__device__ __forceinline__ void pow7_all(uint64_t s[12]) {
#pragma unroll 1
    for (int q = 0; q < 3; q++) {
#pragma unroll
        for (int i = 0; i < 4; i++) s[i] = pr_pow7(s[i]);
        const uint64_t t0 = s[0], t1 = s[1], t2 = s[2], t3 = s[3];
#pragma unroll
        for (int i = 0; i < 8; i++) s[i] = s[i + 4];
        s[8] = t0;
        s[9] = t1;
        s[10] = t2;
        s[11] = t3;
    }
}

// The permutation on a partially reduced state (outputs partially reduced).
// Round r adds its 12 constants, applies x^7 (all lanes in rounds 0-3 and
// 26-29, lane 0 otherwise) and the MDS layer; each round's constants are
// added inside the previous round's MDS reduction.
__device__ __forceinline__ void poseidon_permute(uint64_t s[12]) {
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = pr_add_c(s[i], c_poseidon_rc[i]);
#pragma unroll 1
    for (int rnd = 0; rnd < 30; rnd++) {
        if (rnd < 4 || rnd >= 26) pow7_all(s);
        else s[0] = pr_pow7(s[0]);
        small_matvec12(s, PoseidonMds(), rnd < 29 ? &c_poseidon_rc[12 * (rnd + 1)] : nullptr);
    }
}

// ----------------------------------------------------------- Poseidon2
// External layer = (I + [1 1 1] (x) I_4) * blockdiag(M4, M4, M4) with
// M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] (poseidon2.cu:64-110).
struct Poseidon2External {
    __device__ __forceinline__ uint32_t operator()(int r, int c) const {
        constexpr uint32_t m4[16] = {5, 7, 1, 3, 4, 6, 1, 1, 1, 3, 5, 7, 1, 1, 4, 6};
        return m4[(r & 3) * 4 + (c & 3)] * ((r >> 2) == (c >> 2) ? 2u : 1u);
    }
};

// x_i <- x_i * D_i + sum_j x_j (+ next round's constants): poseidon2.cu:131-146.
__device__ __forceinline__ void poseidon2_internal(uint64_t s[12], const uint64_t *c) {
    uint64_t sl = s[0];
    uint32_t sh = 0;
#pragma unroll
    for (int i = 1; i < 12; i++) {
        const uint64_t t = sl + s[i];
        sh += t < sl ? 1u : 0u;
        sl = t;
    }
#pragma unroll
    for (int i = 0; i < 12; i++) {
        const uint64_t cl = sl + c[i];
        const uint32_t ch = sh + (cl < sl ? 1u : 0u);
        s[i] = pr_mul_add(s[i], c_poseidon2_diag[i], cl, ch);
    }
}

__device__ __forceinline__ void poseidon2_permute(uint64_t s[12]) {
    small_matvec12(s, Poseidon2External(), &c_poseidon2_rc[0]);
#pragma unroll 1
    for (int rnd = 0; rnd < 4; rnd++) {
        pow7_all(s);
        small_matvec12(s, Poseidon2External(), &c_poseidon2_rc[12 * (rnd + 1)]);
    }
    // internal rounds: only lane 0 of their constants is non-zero
#pragma unroll 1
    for (int rnd = 4; rnd < 26; rnd++) {
        s[0] = pr_pow7(s[0]);
        poseidon2_internal(s, &c_poseidon2_rc[12 * (rnd + 1)]);
    }
#pragma unroll 1
    for (int rnd = 26; rnd < 30; rnd++) {
        pow7_all(s);
        small_matvec12(s, Poseidon2External(), rnd < 29 ? &c_poseidon2_rc[12 * (rnd + 1)] : nullptr);
    }
}

// --------------------------------------------------------------- Keccak
__device__ __forceinline__ uint64_t rotl64(uint64_t x, int s) {
    return s == 0 ? x : ((x << s) | (x >> (64 - s)));
}

__device__ __forceinline__ void keccak_f1600(uint64_t a[25]) {
    constexpr int rho[25] = {ZK_KECCAK_RHO_LIST};
#pragma unroll 1
    for (int rnd = 0; rnd < 24; rnd++) {
        uint64_t c[5], b[25];
#pragma unroll
        for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) {
            const uint64_t d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
#pragma unroll
            for (int y = 0; y < 25; y += 5) a[x + y] ^= d;
        }
        // rho + pi: B[y, 2x + 3y] = rot(A[x, y], rho[x, y])
#pragma unroll
        for (int x = 0; x < 5; x++)
#pragma unroll
            for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], rho[x + 5 * y]);
        // chi
#pragma unroll
        for (int y = 0; y < 25; y += 5)
#pragma unroll
            for (int x = 0; x < 5; x++) a[x + y] = b[x + y] ^ (~b[(x + 1) % 5 + y] & b[(x + 2) % 5 + y]);
        a[0] ^= c_keccak_rc[rnd];
    }
}

// ------------------------------------------------------------ hashers
enum : int { kPoseidon = 0, kKeccak = 1, kPoseidon2 = 3 };

// Leaf elements are reduced mod p when read (a no-op for canonical inputs).
template <int H>
__device__ __forceinline__ void hash_one(const uint64_t *__restrict__ in, uint32_t n, uint64_t *__restrict__ out) {
    if constexpr (H == kKeccak) {
        if (n < 4) {  // copy n words, leave the rest of the digest as it was
#pragma unroll
            for (uint32_t i = 0; i < 4; i++)
                if (i < n) out[i] = in[i];
            return;
        }
        uint64_t a[25];
#pragma unroll
        for (int i = 0; i < 25; i++) a[i] = 0;
        uint32_t idx = 0;
        for (; idx + 17 <= n; idx += 17) {
#pragma unroll
            for (int i = 0; i < 17; i++) a[i] ^= in[idx + i];
            keccak_f1600(a);
        }
        const uint32_t rem = n - idx;  // 0..16 whole words, then the pad
#pragma unroll
        for (int i = 0; i < 17; i++) {
            uint64_t w = (uint32_t)i < rem ? in[idx + i] : 0ull;
            if ((uint32_t)i == rem) w ^= 0x01ull;
            if (i == 16) w ^= 0x80ull << 56;
            a[i] ^= w;
        }
        keccak_f1600(a);
        out[0] = a[0];
        out[1] = a[1];
        out[2] = a[2];
        out[3] = a[3] & 0xffull;
    } else {
        if (n <= 4) {
#pragma unroll
            for (uint32_t i = 0; i < 4; i++) out[i] = i < n ? in[i] : 0ull;
            return;
        }
        uint64_t s[12];
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = 0;
        for (uint32_t idx = 0; idx < n; idx += 8) {
            const uint32_t len = n - idx < 8 ? n - idx : 8;
            if (len == 8) {
#pragma unroll
                for (int j = 0; j < 8; j++) s[j] = gl_canon(in[idx + j]);
            } else {
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if ((uint32_t)j < len) s[j] = gl_canon(in[idx + j]);
            }
            if constexpr (H == kPoseidon) poseidon_permute(s);
            else poseidon2_permute(s);
        }
        out[0] = gl_canon(s[0]);
        out[1] = gl_canon(s[1]);
        out[2] = gl_canon(s[2]);
        out[3] = gl_canon(s[3]);
    }
}

template <int H>
__device__ __forceinline__ void hash_two(const uint64_t *l, const uint64_t *r, uint64_t *out) {
    if constexpr (H == kKeccak) {
        // keccak256(left[0..25) || right[0..25)): 50 bytes in one block
        uint64_t a[25];
#pragma unroll
        for (int i = 0; i < 25; i++) a[i] = 0;
        const uint64_t r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
        a[0] = l[0];
        a[1] = l[1];
        a[2] = l[2];
        a[3] = (l[3] & 0xffull) | (r0 << 8);
        a[4] = (r0 >> 56) | (r1 << 8);
        a[5] = (r1 >> 56) | (r2 << 8);
        a[6] = (r2 >> 56) | ((r3 & 0xffull) << 8) | (0x01ull << 16);
        a[16] = 0x80ull << 56;
        keccak_f1600(a);
        out[0] = a[0];
        out[1] = a[1];
        out[2] = a[2];
        out[3] = a[3] & 0xffull;
    } else {
        uint64_t s[12];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            s[i] = gl_canon(l[i]);
            s[4 + i] = gl_canon(r[i]);
            s[8 + i] = 0;
        }
        if constexpr (H == kPoseidon) poseidon_permute(s);
        else poseidon2_permute(s);
        out[0] = gl_canon(s[0]);
        out[1] = gl_canon(s[1]);
        out[2] = gl_canon(s[2]);
        out[3] = gl_canon(s[3]);
    }
}

}  // namespace zk
