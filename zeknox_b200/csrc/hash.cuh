// Device hashers of the Merkle path: Poseidon, Poseidon2, Monolith
// (Goldilocks, width 12), Poseidon-BN128 and Keccak-256 over Goldilocks words,
// each one thread per hash with the whole state in registers; Poseidon also
// on six and on two threads per hash, Poseidon2 also on six (end of file), for
// latency-bound work.
//
// Semantics follow zeknox:
//   Poseidon   native/poseidon/poseidon.cu:602-791 (4 full, 22 partial,
//              4 full rounds; x^7; MDS circulant + diag(8,0..0))
//   Poseidon2  native/poseidon2/poseidon2.cu:61-209
//   Keccak     native/keccak/keccak.cu:42-135 (rate 136 B, 0x01 .. 0x80 pad,
//              digest word 3 masked to its low byte)
//   Monolith   native/monolith/monolith.cu:117-233
//   Poseidon-BN128  native/poseidon/poseidon_bn128.cu:111-193
//   sponge     native/poseidon/poseidon_permutation.cuh:226-276 (rate 8,
//              overwrite mode, n <= 4 copies and zero-pads)
#pragma once
#include <stdint.h>

#include <type_traits>

#include "gl64.cuh"
#include "zk_constants.h"

namespace zk {

// ---------------------------------------------------- exact FP64 layers
// The linear layers of both Poseidon variants have small non-negative integer
// coefficients.  They run on the FP64 pipe (full rate on sm_100), next to the
// integer pipes that carry the S-box products: each lane is split into its two
// 32-bit halves, each half-vector goes through the layer in doubles, and every
// product and partial sum is an integer (or half-integer) far below 2^53, so
// the FP64 arithmetic is exact.
//
// No int<->double conversion instruction is used.  A 32-bit x enters as the
// double whose bit pattern is 0x43300000:x, which is 2^52 + x; a result v
// (0 <= v < 2^41) leaves as the double 2^52 + v, whose bit pattern is
// kMagicBits + v.  Those two offsets are cancelled by subtracting
// kMagicAdj = kMagicBits * (1 + 2^32) mod p from the constant that is added
// in the same reduction (the next round's constants), so the constant tables
// used there are stored pre-adjusted.
constexpr double kMagic = 4503599627370496.0;  // 2^52
constexpr uint64_t kMagicBits = 0x4330000000000000ull;
__host__ __device__ constexpr uint64_t cx_canon(uint64_t a) { return a >= ZK_P ? a - ZK_P : a; }
constexpr uint64_t cx_add_mod(uint64_t a, uint64_t b) {  // a, b < p
    return a >= ZK_P - b ? a - (ZK_P - b) : a + b;
}
constexpr uint64_t cx_sub_mod(uint64_t a, uint64_t b) { return a >= b ? a - b : a + (ZK_P - b); }
// kMagicBits * 2^32 = hi32 * 2^64 = hi32 * (2^32 - 1) (mod p) because its low word is zero.
constexpr uint64_t kMagicAdj = cx_add_mod(kMagicBits, (kMagicBits >> 32 << 32) - (kMagicBits >> 32));
static_assert((kMagicBits & 0xffffffffull) == 0 && kMagicAdj == 0x865fffffbcd00000ull, "magic constants");
constexpr uint64_t kMagicNeg = cx_sub_mod(0, kMagicAdj);  // added where no constant follows

struct RcTable {
    uint64_t v[360];
};
constexpr RcTable magic_adjusted(RcTable t) {
    for (int i = 0; i < 360; i++) t.v[i] = cx_sub_mod(cx_canon(t.v[i]), kMagicAdj);
    return t;
}

// Poseidon: the next round's constant c goes into the FP64 accumulators
// instead of the integer reduction.  With m = (c - kMagicAdj) mod p, the low
// and high half-vector outputs of round rnd start from 2^52 + (m mod 2^32) and
// 2^52 + floor(m / 2^32) (exact: both below 2^53), so that
// bits(lo) + bits(hi) * 2^32 = MDS x + c (mod p).  Round 29 has no constant.
struct MdsK {
    double v[30][2][12];
};
constexpr MdsK make_mds_k(RcTable rc) {
    MdsK t{};
    for (int rnd = 0; rnd < 30; rnd++)
        for (int r = 0; r < 12; r++) {
            const uint64_t m = cx_sub_mod(rnd < 29 ? cx_canon(rc.v[12 * (rnd + 1) + r]) : 0, kMagicAdj);
            t.v[rnd][0][r] = kMagic + (double)(m & 0xffffffffull);
            t.v[rnd][1][r] = kMagic + (double)(m >> 32);
        }
    return t;
}

// The round tables of one hasher.  Permutations read them from the
// __constant__ bank (kernels with many resident warps keep it hot) or from a
// block's shared-memory copy of the __device__ twin (latency-bound kernels
// with a few warps, which would otherwise wait on a constant-cache miss in
// every round).
struct PoseidonTab {
    MdsK mdsk;         // next-round constants inside the MDS accumulators
    uint64_t rc0[12];  // round 0, added before the first S-box
};
struct Poseidon2Tab {
    RcTable rcm;        // external rounds: adjusted for the magic offsets
    RcTable rc;         // internal rounds (lane 0) and the first external round after them
    uint64_t diag[12];  // internal-layer diagonal
};
struct KeccakTab {};
constexpr PoseidonTab make_poseidon_tab(RcTable rc) {
    PoseidonTab t{};
    t.mdsk = make_mds_k(rc);
    for (int i = 0; i < 12; i++) t.rc0[i] = cx_canon(rc.v[i]);
    return t;
}
constexpr Poseidon2Tab make_poseidon2_tab(RcTable rc) {
    Poseidon2Tab t{};
    t.rcm = magic_adjusted(rc);
    t.rc = rc;
    constexpr uint64_t d[12] = {ZK_POSEIDON2_DIAG_LIST};
    for (int i = 0; i < 12; i++) t.diag[i] = d[i];
    return t;
}
__constant__ PoseidonTab c_poseidon = make_poseidon_tab(RcTable{{ZK_POSEIDON_RC_LIST}});
__constant__ Poseidon2Tab c_poseidon2 = make_poseidon2_tab(RcTable{{ZK_POSEIDON2_RC_LIST}});
__device__ PoseidonTab g_poseidon = make_poseidon_tab(RcTable{{ZK_POSEIDON_RC_LIST}});
__device__ Poseidon2Tab g_poseidon2 = make_poseidon2_tab(RcTable{{ZK_POSEIDON2_RC_LIST}});
__constant__ uint64_t c_keccak_rc[24] = {ZK_KECCAK_RC_LIST};
__constant__ KeccakTab c_keccak_tab;

__device__ __forceinline__ double magic_in(uint32_t x) { return __hiloint2double(0x43300000, (int)x); }
__device__ __forceinline__ uint64_t magic_out(double v) { return (uint64_t)__double_as_longlong(v); }

// s[r] <- (lo[r] + hi[r] * 2^32 + c[r]) mod p (partially reduced), where lo, hi
// are the magic-offset outputs of a layer and cm the adjusted constants
// (nullptr: no constant).
__device__ __forceinline__ void magic_combine(uint64_t s[12], const double lo[12], const double hi[12],
                                              const uint64_t *cm) {
#pragma unroll
    for (int r = 0; r < 12; r++) s[r] = pr_reduce_split(magic_out(lo[r]), magic_out(hi[r]), cm ? cm[r] : kMagicNeg);
}

// ------------------------------------------------------------ Poseidon
// MDS = C + diag(8, 0, ..., 0), C circulant with C[r][k] = circ[(k - r) mod 12].
// In 6x6 blocks C = [[A, B], [B, A]], so with u = x_lo + x_hi, w = x_lo - x_hi
// (x_lo = lanes 0-5, x_hi = lanes 6-11):
//   2 (C x)_lo = (A + B) u + (A - B) w,   2 (C x)_hi = (A + B) u - (A - B) w,
// which takes 72 multiply-adds per half-vector instead of 144.
#define ZK_MDS_TABLES                                                  \
    constexpr uint32_t circ[12] = {ZK_POSEIDON_MDS_CIRC_LIST};         \
    constexpr uint32_t diag[12] = {ZK_POSEIDON_MDS_DIAG_LIST};
constexpr bool diag_only_lane0() {
    ZK_MDS_TABLES
    for (int i = 1; i < 12; i++)
        if (diag[i]) return false;
    return circ[0] > 0;
}
static_assert(diag_only_lane0(), "the MDS layer below assumes diag(d, 0, ..., 0)");
__host__ __device__ constexpr int mds_diag0() {
    ZK_MDS_TABLES
    return (int)diag[0] + 0 * (int)circ[0];
}
__host__ __device__ constexpr int mds_p2(int r, int k) {  // A + B, plus d on (0, 0)
    ZK_MDS_TABLES
    return (int)(circ[(k - r + 12) % 12] + circ[(k + 6 - r + 12) % 12]) + (r == 0 && k == 0 ? (int)diag[0] : 0);
}
__host__ __device__ constexpr int mds_q2(int r, int k) {  // A - B, plus d on (0, 0)
    ZK_MDS_TABLES
    return (int)circ[(k - r + 12) % 12] - (int)circ[(k + 6 - r + 12) % 12] + (r == 0 && k == 0 ? (int)diag[0] : 0);
}
#undef ZK_MDS_TABLES

// Coefficients of the circulant split for one hasher's MDS.
struct PoseidonCirc {
    __host__ __device__ static constexpr int p2(int r, int k) { return mds_p2(r, k); }
    __host__ __device__ static constexpr int q2(int r, int k) { return mds_q2(r, k); }
    __host__ __device__ static constexpr int d0() { return mds_diag0(); }
};

// One half-vector: a[i] = 2^52 + x[i] in, o[r] = k[r] + (M x)[r] out, M the
// circulant (plus diag(d0, 0, ...)) of C.
template <class C>
__device__ __forceinline__ void circ12_half(const double a[12], double o[12], const double *k) {
    double u[6], w[6], x6 = 0.0;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const double t = a[i + 6] - kMagic;  // x_hi[i]
        if (i == 0) x6 = t;
        w[i] = a[i] - a[i + 6];              // exact: both in [2^52, 2^53)
        u[i] = fma(2.0, t, w[i]);
    }
#pragma unroll
    for (int r = 0; r < 6; r++) {
        // Lanes 0 and 6 (u[0], w[0]) last: in a partial round only lane 0 has
        // just left the S-box, so the other terms need not wait for it.
        double pa = (double)C::p2(r, 1) * u[1], qa = (double)C::q2(r, 1) * w[1];
#pragma unroll
        for (int c = 2; c < 6; c++) {
            pa = fma((double)C::p2(r, c), u[c], pa);
            qa = fma((double)C::q2(r, c), w[c], qa);
        }
        pa = fma((double)C::p2(r, 0), u[0], pa);
        qa = fma((double)C::q2(r, 0), w[0], qa);
        // The (0, 0) terms carry d (u + w) = 2 d x_lo[0] into lane 0; lane 6
        // must not get d (u - w) = 2 d x_hi[0], so it is taken out again.
        double d = pa - qa;
        if constexpr (C::d0() != 0) {
            if (r == 0) d = fma(-2.0 * (double)C::d0(), x6, d);
        }
        o[r] = fma(0.5, pa + qa, k[r]);
        o[r + 6] = fma(0.5, d, k[r + 6]);
    }
}
__device__ __forceinline__ void poseidon_mds_half(const double a[12], double o[12], const double *k) {
    circ12_half<PoseidonCirc>(a, o, k);
}

// s <- MDS s + c, c being round rnd + 1's constants (none after round 29).
__device__ __forceinline__ void poseidon_mds(uint64_t s[12], int rnd, const PoseidonTab &tab) {
    double a[12], lo[12], hi[12];
#pragma unroll
    for (int i = 0; i < 12; i++) a[i] = magic_in((uint32_t)s[i]);
    poseidon_mds_half(a, lo, tab.mdsk.v[rnd][0]);
#pragma unroll
    for (int i = 0; i < 12; i++) a[i] = magic_in((uint32_t)(s[i] >> 32));
    poseidon_mds_half(a, hi, tab.mdsk.v[rnd][1]);
#pragma unroll
    for (int r = 0; r < 12; r++) s[r] = pr_reduce_split_nc(magic_out(lo[r]), magic_out(hi[r]));
}

// x^7 on all 12 lanes.  W = 4: three passes over 4 lanes with a rotation
// between them (a small loop body, and so a small instruction footprint, for
// kernels with many resident warps).  W = 12: all lanes at once (more
// independent work in flight, for kernels whose few warps wait on latency).
template <int W = 4>
__device__ __forceinline__ void pow7_all(uint64_t s[12]) {
    if constexpr (W == 12) {
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = pr_pow7(s[i]);
    } else {
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
}

// The permutation on a partially reduced state (outputs partially reduced).
// Round r adds its 12 constants, applies x^7 (all lanes in rounds 0-3 and
// 26-29, lane 0 otherwise) and the MDS layer; each round's constants are
// added inside the previous round's MDS reduction.
template <int W = 4>
__device__ __forceinline__ void poseidon_permute(uint64_t s[12], const PoseidonTab &tab = c_poseidon) {
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = pr_add_c(s[i], tab.rc0[i]);
#pragma unroll 1
    for (int rnd = 0; rnd < 30; rnd++) {
        if (rnd < 4 || rnd >= 26) pow7_all<W>(s);
        else s[0] = pr_pow7(s[0]);
        poseidon_mds(s, rnd, tab);
    }
}

// ----------------------------------------------------------- Poseidon2
// External layer = (I + [1 1 1] (x) I_4) * blockdiag(M4, M4, M4) with
// M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] (poseidon2.cu:64-110):
// y_b = M4 x_b per 4-lane block, then out_b = y_b + (y_0 + y_1 + y_2).
// M4 x is the 8-addition network of the Poseidon2 paper (Grassi, Khovratovich,
// Schofnegger 2023, section 5.1): t0 = x0 + x1, t1 = x2 + x3, t2 = 2 x1 + t1,
// t3 = 2 x3 + t0, t4 = 4 t1 + t3, t5 = 4 t0 + t2, M4 x = (t3 + t5, t5, t2 + t4, t4).
__device__ __forceinline__ void poseidon2_external_half(const double a[12], double o[12]) {
    double y[12];
#pragma unroll
    for (int b = 0; b < 3; b++) {
        const double x0 = a[4 * b] - kMagic, x1 = a[4 * b + 1] - kMagic;
        const double x2 = a[4 * b + 2] - kMagic, x3 = a[4 * b + 3] - kMagic;
        const double t0 = x0 + x1, t1 = x2 + x3;
        const double t2 = fma(2.0, x1, t1), t3 = fma(2.0, x3, t0);
        const double t4 = fma(4.0, t1, t3), t5 = fma(4.0, t0, t2);
        y[4 * b] = t3 + t5;
        y[4 * b + 1] = t5;
        y[4 * b + 2] = t2 + t4;
        y[4 * b + 3] = t4;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const double sm = (y[j] + y[4 + j]) + (y[8 + j] + kMagic);
#pragma unroll
        for (int b = 0; b < 3; b++) o[4 * b + j] = y[4 * b + j] + sm;
    }
}

__device__ __forceinline__ void poseidon2_external(uint64_t s[12], const uint64_t *cm) {
    double a[12], lo[12], hi[12];
#pragma unroll
    for (int i = 0; i < 12; i++) a[i] = magic_in((uint32_t)s[i]);
    poseidon2_external_half(a, lo);
#pragma unroll
    for (int i = 0; i < 12; i++) a[i] = magic_in((uint32_t)(s[i] >> 32));
    poseidon2_external_half(a, hi);
    magic_combine(s, lo, hi, cm);
}

// x_i <- x_i * D_i + sum_j x_j (+ next round's constants): poseidon2.cu:131-146.
// The sum of the 12 lanes is kept exact in 96 bits (carry chain).
__device__ __forceinline__ void poseidon2_internal(uint64_t s[12], const uint64_t *c, const uint64_t *diag) {
    uint32_t s0 = (uint32_t)s[0], s1 = (uint32_t)(s[0] >> 32), s2 = 0;
#pragma unroll
    for (int i = 1; i < 12; i++) {
        asm("add.cc.u32 %0, %0, %3;\n\t"
            "addc.cc.u32 %1, %1, %4;\n\t"
            "addc.u32 %2, %2, 0;"
            : "+r"(s0), "+r"(s1), "+r"(s2)
            : "r"((uint32_t)s[i]), "r"((uint32_t)(s[i] >> 32)));
    }
#pragma unroll
    for (int i = 0; i < 12; i++) {
        uint32_t c0, c1, c2;
        asm("add.cc.u32 %0, %3, %6;\n\t"
            "addc.cc.u32 %1, %4, %7;\n\t"
            "addc.u32 %2, %5, 0;"
            : "=r"(c0), "=r"(c1), "=r"(c2)
            : "r"(s0), "r"(s1), "r"(s2), "r"((uint32_t)c[i]), "r"((uint32_t)(c[i] >> 32)));
        s[i] = pr_mul_add(s[i], diag[i], ((uint64_t)c1 << 32) | c0, c2);
    }
}

template <int W = 4>
__device__ __forceinline__ void poseidon2_permute(uint64_t s[12], const Poseidon2Tab &tab = c_poseidon2) {
    poseidon2_external(s, &tab.rcm.v[0]);
#pragma unroll 1
    for (int rnd = 0; rnd < 4; rnd++) {
        pow7_all<W>(s);
        poseidon2_external(s, &tab.rcm.v[12 * (rnd + 1)]);
    }
    // internal rounds: only lane 0 of their constants is non-zero
#pragma unroll 1
    for (int rnd = 4; rnd < 26; rnd++) {
        s[0] = pr_pow7(s[0]);
        poseidon2_internal(s, &tab.rc.v[12 * (rnd + 1)], tab.diag);
    }
#pragma unroll 1
    for (int rnd = 26; rnd < 30; rnd++) {
        pow7_all<W>(s);
        poseidon2_external(s, rnd < 29 ? &tab.rcm.v[12 * (rnd + 1)] : nullptr);
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

// --------------------------------------------------------------- Monolith
// Monolith-64, width 12, 6 rounds (native/monolith/monolith.cu:117-233):
// concrete(rc_0), then per round r = 1..6: bars, bricks, concrete(rc_r).
//  * concrete: the circulant matrix (row r column c = ROW[(c - r) mod 12], row
//    sum 160) plus the round constant, mod p.  The same exact FP64 split as
//    the Poseidon MDS, no diagonal.  Lanes 0-3 are canonicalised afterwards:
//    the Bar S-box acts on the bits of the canonical value.
//  * bars: Bar on every byte of lanes 0-3,
//    y = rotl1(x ^ (rotl1(~x) & rotl2(x) & rotl3(x))) (rotations within the byte).
//  * bricks (Feistel type 3): lane i, from 11 down to 1, += (lane i-1)^2 mod p,
//    the square of lane i-1 before the layer.  zeknox keeps that sum as a
//    65-bit value for the next concrete layer; here it is taken mod p
//    (pr_add_c), which is the same field element.
#define ZK_MONO_ROW constexpr uint32_t row[12] = {ZK_MONOLITH_MDS_ROW_LIST};
struct MonolithCirc {
    __host__ __device__ static constexpr int p2(int r, int k) {
        ZK_MONO_ROW
        return (int)(row[(k - r + 12) % 12] + row[(k + 6 - r + 12) % 12]);
    }
    __host__ __device__ static constexpr int q2(int r, int k) {
        ZK_MONO_ROW
        return (int)row[(k - r + 12) % 12] - (int)row[(k + 6 - r + 12) % 12];
    }
    __host__ __device__ static constexpr int d0() { return 0; }
};
#undef ZK_MONO_ROW

// Accumulator starting values of the 7 concrete layers ("to integers" form:
// 2^52 + the 32-bit halves of (rc - kMagicAdj) mod p).
struct MonolithTab {
    double k[7][2][12];
};
constexpr MonolithTab make_monolith_tab() {
    MonolithTab t{};
    constexpr uint64_t rc[84] = {ZK_MONOLITH_RC_LIST};
    for (int rnd = 0; rnd < 7; rnd++)
        for (int r = 0; r < 12; r++) {
            const uint64_t m = cx_sub_mod(cx_canon(rc[12 * rnd + r]), kMagicAdj);
            t.k[rnd][0][r] = kMagic + (double)(m & 0xffffffffull);
            t.k[rnd][1][r] = kMagic + (double)(m >> 32);
        }
    return t;
}
__constant__ MonolithTab c_monolith = make_monolith_tab();
__device__ MonolithTab g_monolith = make_monolith_tab();

__device__ __forceinline__ void monolith_concrete(uint64_t s[12], const double (*k)[12]) {
    double a[12], lo[12], hi[12];
#pragma unroll
    for (int i = 0; i < 12; i++) a[i] = magic_in((uint32_t)s[i]);
    circ12_half<MonolithCirc>(a, lo, k[0]);
#pragma unroll
    for (int i = 0; i < 12; i++) a[i] = magic_in((uint32_t)(s[i] >> 32));
    circ12_half<MonolithCirc>(a, hi, k[1]);
#pragma unroll
    for (int r = 0; r < 12; r++) s[r] = pr_reduce_split_nc(magic_out(lo[r]), magic_out(hi[r]));
#pragma unroll
    for (int r = 0; r < 4; r++) s[r] = gl_canon(s[r]);
}

// Rotate every byte of x left by K (within the byte).
template <int K>
__device__ __forceinline__ uint32_t rotl_bytes(uint32_t x) {
    constexpr uint32_t low = 0x01010101u * ((1u << K) - 1u);  // the low K bits of each byte
    return ((x << K) & ~low) | ((x >> (8 - K)) & low);
}
__device__ __forceinline__ uint32_t monolith_bar32(uint32_t x) {
    return rotl_bytes<1>(x ^ (rotl_bytes<1>(~x) & rotl_bytes<2>(x) & rotl_bytes<3>(x)));
}

__device__ __forceinline__ void monolith_permute(uint64_t s[12], const MonolithTab &tab = c_monolith) {
    monolith_concrete(s, tab.k[0]);
#pragma unroll 1
    for (int rnd = 1; rnd <= 6; rnd++) {
#pragma unroll
        for (int i = 0; i < 4; i++)
            s[i] = ((uint64_t)monolith_bar32((uint32_t)(s[i] >> 32)) << 32) | monolith_bar32((uint32_t)s[i]);
#pragma unroll
        for (int i = 11; i > 0; i--) s[i] = pr_add_c(s[i], gl_mul(s[i - 1], s[i - 1]));
        monolith_concrete(s, tab.k[rnd]);
    }
}

// ---------------------------------------------------- Poseidon-BN128
// circomlib's Poseidon over the BN254 scalar field r, t = 5, 8 full and 60
// partial rounds in the optimised form (native/poseidon/poseidon_bn128.cu:
// 111-193), field arithmetic of element_bn128.cu: Montgomery form with
// R = 2^256, four 64-bit limbs, every result fully reduced.  The 12
// Goldilocks lanes become 4 field elements x_i = lane[3i+2] + lane[3i+1] 2^64
// + lane[3i] 2^128; the state is (0, x_0, .., x_3).  Output lane 3i + k is
// limb 2 - k of state element i, reduced mod p once.
struct BnTab {
    uint64_t c[100][4];  // round constants
    uint64_t s[540][4];  // sparse partial-round matrices, 9 values per round
    uint64_t m[25][4];   // MDS, m[5 j + i] multiplies state j into lane i
    uint64_t p[25][4];   // pre-sparse matrix (same indexing)
};
constexpr BnTab make_bn_tab() {
    BnTab t{};
    constexpr uint64_t c[400] = {ZK_BN128_C_LIST};
    constexpr uint64_t sp[2160] = {ZK_BN128_S_LIST};
    constexpr uint64_t m[100] = {ZK_BN128_M_LIST};
    constexpr uint64_t pm[100] = {ZK_BN128_P_LIST};
    for (int i = 0; i < 400; i++) t.c[i / 4][i % 4] = c[i];
    for (int i = 0; i < 2160; i++) t.s[i / 4][i % 4] = sp[i];
    for (int i = 0; i < 100; i++) t.m[i / 4][i % 4] = m[i];
    for (int i = 0; i < 100; i++) t.p[i / 4][i % 4] = pm[i];
    return t;
}
__constant__ BnTab c_bn128 = make_bn_tab();
__device__ BnTab g_bn128 = make_bn_tab();

struct Fr {
    uint64_t v[4];
};
__host__ __device__ constexpr uint64_t bn_r(int i) {  // the modulus r, little-endian limbs
    constexpr uint64_t r[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                               0x30644e72e131a029ull};
    return r[i];
}
constexpr uint64_t kBnNinv = 0xc2e1f593efffffffull;  // -r^-1 mod 2^64
constexpr uint64_t kBnR2[4] = {0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull, 0x8c49833d53bb8085ull,
                               0x0216d0b17f4e44a5ull};  // 2^512 mod r

// t - r if t >= r (t < 2r; `top` is bit 256 of t): one borrow chain.
__device__ __forceinline__ void bn_reduce_once(uint64_t t[4], uint64_t top) {
    uint64_t d0, d1, d2, d3;
    uint32_t bw;
    asm("sub.cc.u64  %0, %5, %9;\n\t"
        "subc.cc.u64 %1, %6, %10;\n\t"
        "subc.cc.u64 %2, %7, %11;\n\t"
        "subc.cc.u64 %3, %8, %12;\n\t"
        "subc.u32    %4, 0, 0;"
        : "=l"(d0), "=l"(d1), "=l"(d2), "=l"(d3), "=r"(bw)
        : "l"(t[0]), "l"(t[1]), "l"(t[2]), "l"(t[3]), "l"(bn_r(0)), "l"(bn_r(1)), "l"(bn_r(2)), "l"(bn_r(3)));
    const bool ge = top != 0 || bw == 0;
    t[0] = ge ? d0 : t[0];
    t[1] = ge ? d1 : t[1];
    t[2] = ge ? d2 : t[2];
    t[3] = ge ? d3 : t[3];
}
// x + y mod r for x, y < r: one carry chain, then bn_reduce_once.
__device__ __forceinline__ Fr bn_add(const Fr &x, const Fr &y) {
    Fr z;
    uint32_t c;
    asm("add.cc.u64  %0, %5, %9;\n\t"
        "addc.cc.u64 %1, %6, %10;\n\t"
        "addc.cc.u64 %2, %7, %11;\n\t"
        "addc.cc.u64 %3, %8, %12;\n\t"
        "addc.u32    %4, 0, 0;"
        : "=l"(z.v[0]), "=l"(z.v[1]), "=l"(z.v[2]), "=l"(z.v[3]), "=r"(c)
        : "l"(x.v[0]), "l"(x.v[1]), "l"(x.v[2]), "l"(x.v[3]), "l"(y.v[0]), "l"(y.v[1]), "l"(y.v[2]), "l"(y.v[3]));
    bn_reduce_once(z.v, c);
    return z;
}
// Montgomery product x y / 2^256 mod r: CIOS over eight 32-bit limbs, each
// row a pair of carry chains (low halves of the products, then high halves)
// for t += x y_i and for t += m r, m = t_0 (-r^-1) mod 2^32; the row ends by
// dropping the zero limb t_0.  t < 2r throughout; one conditional
// subtraction at the end.
// Not inlined: a permutation makes ~1050 of these products, and one shared
// copy of the code keeps the kernel inside the instruction cache (inlined,
// ncu showed warps waiting on instruction fetch ~3 cycles per issue).
constexpr uint32_t kBnNinv32 = 0xefffffffu;  // -r^-1 mod 2^32
__device__ __noinline__ Fr bn_mul(const Fr &x, const Fr &y) {
    uint32_t a[8], b[8], r[8];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        a[2 * i] = (uint32_t)x.v[i];
        a[2 * i + 1] = (uint32_t)(x.v[i] >> 32);
        b[2 * i] = (uint32_t)y.v[i];
        b[2 * i + 1] = (uint32_t)(y.v[i] >> 32);
        r[2 * i] = (uint32_t)bn_r(i);
        r[2 * i + 1] = (uint32_t)(bn_r(i) >> 32);
    }
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0, t9 = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t bi = b[i];
        // t += a * b_i
        asm("mad.lo.cc.u32  %0, %10, %18, %0;\n\t"
            "madc.lo.cc.u32 %1, %11, %18, %1;\n\t"
            "madc.lo.cc.u32 %2, %12, %18, %2;\n\t"
            "madc.lo.cc.u32 %3, %13, %18, %3;\n\t"
            "madc.lo.cc.u32 %4, %14, %18, %4;\n\t"
            "madc.lo.cc.u32 %5, %15, %18, %5;\n\t"
            "madc.lo.cc.u32 %6, %16, %18, %6;\n\t"
            "madc.lo.cc.u32 %7, %17, %18, %7;\n\t"
            "addc.cc.u32    %8, %8, 0;\n\t"
            "addc.u32       %9, %9, 0;\n\t"
            "mad.hi.cc.u32  %1, %10, %18, %1;\n\t"
            "madc.hi.cc.u32 %2, %11, %18, %2;\n\t"
            "madc.hi.cc.u32 %3, %12, %18, %3;\n\t"
            "madc.hi.cc.u32 %4, %13, %18, %4;\n\t"
            "madc.hi.cc.u32 %5, %14, %18, %5;\n\t"
            "madc.hi.cc.u32 %6, %15, %18, %6;\n\t"
            "madc.hi.cc.u32 %7, %16, %18, %7;\n\t"
            "madc.hi.cc.u32 %8, %17, %18, %8;\n\t"
            "addc.u32       %9, %9, 0;"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8), "+r"(t9)
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(bi));
        const uint32_t m = t0 * kBnNinv32;
        // t += m * r (t_0 becomes 0)
        asm("mad.lo.cc.u32  %0, %10, %18, %0;\n\t"
            "madc.lo.cc.u32 %1, %11, %18, %1;\n\t"
            "madc.lo.cc.u32 %2, %12, %18, %2;\n\t"
            "madc.lo.cc.u32 %3, %13, %18, %3;\n\t"
            "madc.lo.cc.u32 %4, %14, %18, %4;\n\t"
            "madc.lo.cc.u32 %5, %15, %18, %5;\n\t"
            "madc.lo.cc.u32 %6, %16, %18, %6;\n\t"
            "madc.lo.cc.u32 %7, %17, %18, %7;\n\t"
            "addc.cc.u32    %8, %8, 0;\n\t"
            "addc.u32       %9, %9, 0;\n\t"
            "mad.hi.cc.u32  %1, %10, %18, %1;\n\t"
            "madc.hi.cc.u32 %2, %11, %18, %2;\n\t"
            "madc.hi.cc.u32 %3, %12, %18, %3;\n\t"
            "madc.hi.cc.u32 %4, %13, %18, %4;\n\t"
            "madc.hi.cc.u32 %5, %14, %18, %5;\n\t"
            "madc.hi.cc.u32 %6, %15, %18, %6;\n\t"
            "madc.hi.cc.u32 %7, %16, %18, %7;\n\t"
            "madc.hi.cc.u32 %8, %17, %18, %8;\n\t"
            "addc.u32       %9, %9, 0;"
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8), "+r"(t9)
            : "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(m));
        t0 = t1, t1 = t2, t2 = t3, t3 = t4, t4 = t5, t5 = t6, t6 = t7, t7 = t8, t8 = t9, t9 = 0;
    }
    Fr z{{((uint64_t)t1 << 32) | t0, ((uint64_t)t3 << 32) | t2, ((uint64_t)t5 << 32) | t4,
          ((uint64_t)t7 << 32) | t6}};
    bn_reduce_once(z.v, t8);
    return z;
}
__device__ __forceinline__ Fr bn_load(const uint64_t (&a)[4]) { return Fr{{a[0], a[1], a[2], a[3]}}; }
__device__ __forceinline__ Fr bn_exp5(const Fr &x) {
    const Fr x2 = bn_mul(x, x);
    const Fr x4 = bn_mul(x2, x2);
    return bn_mul(x4, x);
}
// st <- M^T st (new_i = sum_j m[5 j + i] st_j)
__device__ __forceinline__ void bn_mix(Fr st[5], const uint64_t (*m)[4]) {
    Fr out[5];
#pragma unroll 1
    for (int i = 0; i < 5; i++) {
        Fr acc = bn_mul(bn_load(m[i]), st[0]);
#pragma unroll
        for (int j = 1; j < 5; j++) acc = bn_add(acc, bn_mul(bn_load(m[5 * j + i]), st[j]));
        out[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 5; i++) st[i] = out[i];
}

__device__ __forceinline__ void poseidon_bn128_permute(uint64_t s[12], const BnTab &tab = c_bn128) {
    Fr st[5];
    st[0] = Fr{{0, 0, 0, 0}};
    const Fr r2{{kBnR2[0], kBnR2[1], kBnR2[2], kBnR2[3]}};
#pragma unroll
    for (int i = 0; i < 4; i++) st[i + 1] = bn_mul(Fr{{s[3 * i + 2], s[3 * i + 1], s[3 * i], 0}}, r2);
#pragma unroll
    for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], bn_load(tab.c[i]));
#pragma unroll 1
    for (int r = 0; r < 4; r++) {  // full rounds 1-4: S-box, constants, M (P for the 4th)
#pragma unroll
        for (int i = 0; i < 5; i++) st[i] = bn_exp5(st[i]);
#pragma unroll
        for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], bn_load(tab.c[5 * (r + 1) + i]));
        bn_mix(st, r < 3 ? tab.m : tab.p);
    }
#pragma unroll 1
    for (int r = 0; r < 60; r++) {  // partial rounds with the sparse matrices
        st[0] = bn_add(bn_exp5(st[0]), bn_load(tab.c[25 + r]));
        const uint64_t (*sp)[4] = tab.s + 9 * r;
        Fr acc = bn_mul(bn_load(sp[0]), st[0]);
#pragma unroll
        for (int j = 1; j < 5; j++) acc = bn_add(acc, bn_mul(bn_load(sp[j]), st[j]));
#pragma unroll
        for (int k = 1; k < 5; k++) st[k] = bn_add(st[k], bn_mul(st[0], bn_load(sp[4 + k])));
        st[0] = acc;
    }
#pragma unroll 1
    for (int r = 0; r < 4; r++) {  // full rounds 5-8 (no constants in the last)
#pragma unroll
        for (int i = 0; i < 5; i++) st[i] = bn_exp5(st[i]);
        if (r < 3) {
#pragma unroll
            for (int i = 0; i < 5; i++) st[i] = bn_add(st[i], bn_load(tab.c[85 + 5 * r + i]));
        }
        bn_mix(st, tab.m);
    }
    const Fr one{{1, 0, 0, 0}};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const Fr v = bn_mul(st[i], one);  // out of Montgomery form
#pragma unroll
        for (int k = 0; k < 3; k++) s[3 * i + k] = gl_canon(v.v[2 - k]);
    }
}

// ------------------------------------------------------------ hashers
enum : int { kPoseidon = 0, kKeccak = 1, kPoseidonBN128 = 2, kPoseidon2 = 3, kMonolith = 4 };

// Leaf elements are reduced mod p when read (a no-op for canonical inputs).
template <int H, int W = 4>
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
            if constexpr (H == kPoseidon) poseidon_permute<W>(s);
            else if constexpr (H == kMonolith) monolith_permute(s);
            else if constexpr (H == kPoseidonBN128) poseidon_bn128_permute(s);
            else poseidon2_permute<W>(s);
        }
        out[0] = gl_canon(s[0]);
        out[1] = gl_canon(s[1]);
        out[2] = gl_canon(s[2]);
        out[3] = gl_canon(s[3]);
    }
}

template <int H>
struct TabOf;
template <>
struct TabOf<kPoseidon> {
    using type = PoseidonTab;
};
template <>
struct TabOf<kPoseidon2> {
    using type = Poseidon2Tab;
};
template <>
struct TabOf<kKeccak> {
    using type = KeccakTab;
};
template <>
struct TabOf<kMonolith> {
    using type = MonolithTab;
};
template <>
struct TabOf<kPoseidonBN128> {
    using type = BnTab;
};
template <int H>
__device__ __forceinline__ const typename TabOf<H>::type &const_tab() {
    if constexpr (H == kPoseidon) return c_poseidon;
    else if constexpr (H == kPoseidon2) return c_poseidon2;
    else if constexpr (H == kMonolith) return c_monolith;
    else if constexpr (H == kPoseidonBN128) return c_bn128;
    else return c_keccak_tab;
}

// The __device__ twin of a hasher's tables (source of shared-memory copies).
template <int H>
__device__ __forceinline__ const typename TabOf<H>::type *global_tab() {
    if constexpr (H == kPoseidon) return &g_poseidon;
    else if constexpr (H == kPoseidon2) return &g_poseidon2;
    else if constexpr (H == kMonolith) return &g_monolith;
    else if constexpr (H == kPoseidonBN128) return &g_bn128;
    else return nullptr;
}

// H(l || r) of two digests; W and tab choose the S-box width and the table copy.
template <int H, int W = 4>
__device__ __forceinline__ void hash_two(const uint64_t *l, const uint64_t *r, uint64_t *out,
                                         const typename TabOf<H>::type &tab = const_tab<H>()) {
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
        if constexpr (H == kPoseidon) poseidon_permute<W>(s, tab);
        else if constexpr (H == kMonolith) monolith_permute(s, tab);
        else if constexpr (H == kPoseidonBN128) poseidon_bn128_permute(s, tab);
        else poseidon2_permute<W>(s, tab);
        out[0] = gl_canon(s[0]);
        out[1] = gl_canon(s[1]);
        out[2] = gl_canon(s[2]);
        out[3] = gl_canon(s[3]);
    }
}

// ------------------------------------------- Poseidon on two threads
// For trees with too few leaves to fill the GPU one thread per hash, but
// enough that six threads per hash would be issue-bound: the permutation is
// split over the two threads of a lane pair (lanes 2k, 2k + 1; sixteen hashes
// per warp, no idle lanes).  Thread h owns state lanes 6h .. 6h + 5.  Each
// round: the S-box on the owned lanes (lane 0 only, on thread 0, in partial
// rounds); then the MDS with the 32-bit halves split between the pair (thread
// 0 takes the low halves of all 12 lanes, thread 1 the high halves: six
// 32-bit shuffles bring the partner's halves), the half-vector layer in FP64
// as in the one-thread path, and six 64-bit shuffles that hand each thread
// the other half of its own lanes' outputs.  The total work is about that
// of one thread per hash, spread over twice the threads.
__device__ __forceinline__ uint32_t shfl_xor32(uint32_t v) { return (uint32_t)__shfl_xor_sync(0xffffffffu, (int)v, 1); }
__device__ __forceinline__ double shfl_xor_d(double v) { return __shfl_xor_sync(0xffffffffu, v, 1); }

// s: lanes 6h .. 6h + 5 (partially reduced, in and out).  Every lane of the
// warp must call this (shuffles over the full warp).
__device__ __forceinline__ void poseidon_permute_duo(uint64_t s[6], uint32_t h, const PoseidonTab &tab) {
#pragma unroll
    for (int i = 0; i < 6; i++) s[i] = pr_add_c(s[i], tab.rc0[6 * h + i]);
#pragma unroll 1
    for (int rnd = 0; rnd < 30; rnd++) {
        if (rnd < 4 || rnd >= 26) {
#pragma unroll
            for (int i = 0; i < 6; i++) s[i] = pr_pow7(s[i]);
        } else if (h == 0) {
            s[0] = pr_pow7(s[0]);
        }
        // Half h of all 12 lanes: own lanes directly, the partner's through a shuffle.
        double a[12], o[12];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            const uint32_t lo = (uint32_t)s[i], hi = (uint32_t)(s[i] >> 32);
            const uint32_t got = shfl_xor32(h ? lo : hi);  // the partner wants the half it computes
            const uint32_t mine = h ? hi : lo;
            a[i] = magic_in(h ? got : mine);       // lanes 0-5: thread 0's own, thread 1's received
            a[i + 6] = magic_in(h ? mine : got);   // lanes 6-11: thread 1's own, thread 0's received
        }
        poseidon_mds_half(a, o, tab.mdsk.v[rnd][h]);
        // Thread 0 keeps the low outputs of lanes 0-5 and receives their high
        // outputs; thread 1 keeps the high outputs of lanes 6-11 and receives
        // their low outputs.
#pragma unroll
        for (int i = 0; i < 6; i++) {
            const double got = shfl_xor_d(h ? o[i] : o[i + 6]);
            const double lo = h ? got : o[i], hi = h ? o[i + 6] : got;
            s[i] = pr_reduce_split_nc(magic_out(lo), magic_out(hi));
        }
    }
}

// Sponge of n words on a lane pair (zeknox's hash_or_noop: n <= 4 copies and
// zero-pads); `active` pairs load and store, the others compute on zeros.
// n must be the same for all pairs of a warp.
__device__ __forceinline__ void poseidon_hash_one_duo(const uint64_t *in, uint32_t n, uint64_t *out, bool active,
                                                      uint32_t h, const PoseidonTab &tab) {
    if (n <= 4) {
        if (active && h == 0)
            for (uint32_t i = 0; i < 4; i++) out[i] = i < n ? in[i] : 0ull;
        return;
    }
    uint64_t s[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t idx = 0; idx < n; idx += 8) {
        const uint32_t len = n - idx < 8 ? n - idx : 8;
        if (active) {
#pragma unroll
            for (uint32_t i = 0; i < 6; i++) {
                const uint32_t lane = 6 * h + i;  // rate lanes 0..7 are overwritten
                if (lane < len) s[i] = gl_canon(in[idx + lane]);
            }
        }
        poseidon_permute_duo(s, h, tab);
    }
    if (active && h == 0)
#pragma unroll
        for (int i = 0; i < 4; i++) out[i] = gl_canon(s[i]);
}

// ------------------------------------------- Poseidon on six threads
// For the latency-bound parts (narrow tree levels, small trees) one
// permutation is spread over a group of six consecutive lanes of a warp
// (five groups per warp; lanes 30 and 31 compute on dummy data).  Group
// thread t owns lanes t and t + 6.  Each round: the S-box on the owned lanes
// (lane 0 only, on thread 0, in partial rounds), an all-gather of the 12
// lanes by shuffles (every shuffle reads one thread of the group, so all
// threads get the lanes in natural order), then thread t computes the MDS
// row pair (t, t + 6) of the split above: rows of A + B and A - B held in
// registers.  About a third of the single-thread path's instructions per
// thread, so about a third of its latency.
struct HexLanes {
    uint32_t t;     // thread within the group, 0..5 (lanes 30, 31: 0..1 of a dummy group)
    uint32_t base;  // warp lane of the group's thread 0
    __device__ __forceinline__ HexLanes() {
        const uint32_t lane = threadIdx.x & 31;
        const uint32_t g = lane < 30 ? lane / 6 : 0;
        t = lane < 30 ? lane % 6 : lane - 30;
        base = 6 * g;
    }
    // true for the lanes whose group is a real one (not lanes 30, 31)
    __device__ __forceinline__ bool real() const { return (threadIdx.x & 31) < 30; }
    __device__ __forceinline__ uint32_t group_in_warp() const { return base / 6; }
};
// Poseidon's group: its MDS rows in registers.  (The table argument gives the
// Poseidon and Poseidon2 group forms one constructor signature.)
struct HexGroup : HexLanes {
    double p2[6], q2[6];  // row t of A + B and A - B (with the diagonal term on row 0)
    double fix6;          // -2 d on thread 0 (lane 6 must not get the diagonal), else 0
    __device__ __forceinline__ explicit HexGroup(const PoseidonTab &) : HexLanes() {
#pragma unroll
        for (int k = 0; k < 6; k++) {
            p2[k] = (double)mds_p2((int)t, k);
            q2[k] = (double)mds_q2((int)t, k);
        }
        fix6 = t == 0 ? -2.0 * (double)mds_diag0() : 0.0;
    }
};

__device__ __forceinline__ uint64_t shfl64(uint64_t v, uint32_t src) {
    return (uint64_t)__shfl_sync(0xffffffffu, (long long)v, (int)src);
}

// o0, o1: lanes t and t + 6 of the state (partially reduced, in and out).
// Every lane of the warp must call this (shuffles over the full warp).
__device__ __forceinline__ void poseidon_permute_hex(uint64_t &o0, uint64_t &o1, const HexGroup &g,
                                                     const PoseidonTab &tab) {
    o0 = pr_add_c(o0, tab.rc0[g.t]);
    o1 = pr_add_c(o1, tab.rc0[g.t + 6]);
#pragma unroll 1
    for (int rnd = 0; rnd < 30; rnd++) {
        if (rnd < 4 || rnd >= 26) {
            o0 = pr_pow7(o0);
            o1 = pr_pow7(o1);
        } else {
            const uint64_t y = pr_pow7(o0);
            if (g.t == 0) o0 = y;
        }
        uint64_t x[12];
#pragma unroll
        for (int i = 0; i < 12; i++) x[i] = shfl64(i < 6 ? o0 : o1, g.base + (i % 6));
        double first[2], second[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double u[6], w[6], x6 = 0.0;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                const double a = magic_in(h ? (uint32_t)(x[i] >> 32) : (uint32_t)x[i]);
                const double b = magic_in(h ? (uint32_t)(x[i + 6] >> 32) : (uint32_t)x[i + 6]);
                const double tb = b - kMagic;
                if (i == 0) x6 = tb;
                w[i] = a - b;
                u[i] = fma(2.0, tb, w[i]);
            }
            double pa = g.p2[0] * u[0], qa = g.q2[0] * w[0];
#pragma unroll
            for (int k = 1; k < 6; k++) {
                pa = fma(g.p2[k], u[k], pa);
                qa = fma(g.q2[k], w[k], qa);
            }
            const double d = fma(g.fix6, x6, pa - qa);
            first[h] = fma(0.5, pa + qa, tab.mdsk.v[rnd][h][g.t]);
            second[h] = fma(0.5, d, tab.mdsk.v[rnd][h][g.t + 6]);
        }
        o0 = pr_reduce_split_nc(magic_out(first[0]), magic_out(first[1]));
        o1 = pr_reduce_split_nc(magic_out(second[0]), magic_out(second[1]));
    }
}

// ------------------------------------------- Poseidon2 on six threads
// The same group layout: thread t owns state lanes t and t + 6.
//
// External layer: output lane r is sum_b (1 + [b == r / 4]) (M4 x_b)[r % 4]
// over the three 4-lane blocks x_b.  Row c + 2 of M4 is row c rotated by two
// columns (M4[c + 2][d] = M4[c][d + 2], indices mod 4), and lane t + 6 has
// column (t + 2) % 4, so thread t needs only m = M4[t % 4]: lane t takes
// x_(4b + d) with m[d], lane t + 6 with m[(d + 2) % 4], and each lane weighs
// the three block sums by w in {1, 2}.  As in the one-thread layer, each
// 32-bit half runs in exact FP64 (every sum below 2^39), offset by 2^52.
//
// Internal layer (x_i <- x_i D_i + sum_j x_j + c_i): each thread adds its
// two lanes exactly (65 bits), the group all-gathers the six partial sums
// (96-bit total), and each thread forms its two lanes' products.
struct HexGroup2 : HexLanes {
    double m[4];          // row t % 4 of M4
    double w0[3], w1[3];  // block weights of lanes t and t + 6
    uint64_t d0, d1;      // internal diagonal of lanes t and t + 6
    __device__ __forceinline__ explicit HexGroup2(const Poseidon2Tab &tab) : HexLanes() {
        // M4 rows 0 and 1; rows 2 and 3 are these rotated by two columns.
        const uint32_t c = t & 3, r = c & 1, rot = c & 2;
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const uint32_t k = (d + rot) & 3;
            const double row0 = k == 0 ? 5.0 : k == 1 ? 7.0 : k == 2 ? 1.0 : 3.0;
            const double row1 = k == 0 ? 4.0 : k == 1 ? 6.0 : 1.0;
            m[d] = r ? row1 : row0;
        }
#pragma unroll
        for (uint32_t b = 0; b < 3; b++) {
            w0[b] = b == t / 4 ? 2.0 : 1.0;
            w1[b] = b == (t + 6) / 4 ? 2.0 : 1.0;
        }
        d0 = tab.diag[t];
        d1 = tab.diag[t + 6];
    }
};

// External layer on a group, plus the constants cm (adjusted for the magic
// offsets; nullptr: none).
__device__ __forceinline__ void poseidon2_external_hex(uint64_t &o0, uint64_t &o1, const HexGroup2 &g,
                                                       const uint64_t *cm) {
    uint64_t x[12];
#pragma unroll
    for (int i = 0; i < 12; i++) x[i] = shfl64(i < 6 ? o0 : o1, g.base + (i % 6));
    double first[2], second[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        double v[12];
#pragma unroll
        for (int i = 0; i < 12; i++) v[i] = magic_in(h ? (uint32_t)(x[i] >> 32) : (uint32_t)x[i]) - kMagic;
        double a0 = kMagic, a1 = kMagic;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            double y0 = g.m[0] * v[4 * b], y1 = g.m[2] * v[4 * b];
#pragma unroll
            for (int d = 1; d < 4; d++) {
                y0 = fma(g.m[d], v[4 * b + d], y0);
                y1 = fma(g.m[(d + 2) & 3], v[4 * b + d], y1);
            }
            a0 = fma(g.w0[b], y0, a0);
            a1 = fma(g.w1[b], y1, a1);
        }
        first[h] = a0;
        second[h] = a1;
    }
    o0 = pr_reduce_split(magic_out(first[0]), magic_out(first[1]), cm ? cm[g.t] : kMagicNeg);
    o1 = pr_reduce_split(magic_out(second[0]), magic_out(second[1]), cm ? cm[g.t + 6] : kMagicNeg);
}

// Internal layer on a group, plus the next round's constants c (unadjusted).
__device__ __forceinline__ void poseidon2_internal_hex(uint64_t &o0, uint64_t &o1, const HexGroup2 &g,
                                                       const uint64_t *c) {
    uint32_t p0, p1, p2;
    asm("add.cc.u32 %0, %3, %5;\n\t"
        "addc.cc.u32 %1, %4, %6;\n\t"
        "addc.u32 %2, 0, 0;"
        : "=r"(p0), "=r"(p1), "=r"(p2)
        : "r"((uint32_t)o0), "r"((uint32_t)(o0 >> 32)), "r"((uint32_t)o1), "r"((uint32_t)(o1 >> 32)));
    uint32_t s0 = 0, s1 = 0, s2 = 0;  // sum of the 12 lanes, below 12 * 2^64
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const uint32_t src = g.base + k;
        const uint32_t q0 = (uint32_t)__shfl_sync(0xffffffffu, (int)p0, (int)src);
        const uint32_t q1 = (uint32_t)__shfl_sync(0xffffffffu, (int)p1, (int)src);
        const uint32_t q2 = (uint32_t)__shfl_sync(0xffffffffu, (int)p2, (int)src);
        asm("add.cc.u32 %0, %0, %3;\n\t"
            "addc.cc.u32 %1, %1, %4;\n\t"
            "addc.u32 %2, %2, %5;"
            : "+r"(s0), "+r"(s1), "+r"(s2)
            : "r"(q0), "r"(q1), "r"(q2));
    }
    uint64_t lane[2] = {o0, o1};
    const uint64_t cc[2] = {c[g.t], c[g.t + 6]};
    const uint64_t dd[2] = {g.d0, g.d1};
#pragma unroll
    for (int j = 0; j < 2; j++) {
        uint32_t c0, c1, c2;
        asm("add.cc.u32 %0, %3, %6;\n\t"
            "addc.cc.u32 %1, %4, %7;\n\t"
            "addc.u32 %2, %5, 0;"
            : "=r"(c0), "=r"(c1), "=r"(c2)
            : "r"(s0), "r"(s1), "r"(s2), "r"((uint32_t)cc[j]), "r"((uint32_t)(cc[j] >> 32)));
        lane[j] = pr_mul_add(lane[j], dd[j], ((uint64_t)c1 << 32) | c0, c2);
    }
    o0 = lane[0];
    o1 = lane[1];
}

// The rounds of poseidon2_permute on a group.
__device__ __forceinline__ void poseidon2_permute_hex(uint64_t &o0, uint64_t &o1, const HexGroup2 &g,
                                                      const Poseidon2Tab &tab) {
    poseidon2_external_hex(o0, o1, g, &tab.rcm.v[0]);
#pragma unroll 1
    for (int rnd = 0; rnd < 4; rnd++) {
        o0 = pr_pow7(o0);
        o1 = pr_pow7(o1);
        poseidon2_external_hex(o0, o1, g, &tab.rcm.v[12 * (rnd + 1)]);
    }
#pragma unroll 1
    for (int rnd = 4; rnd < 26; rnd++) {
        const uint64_t y = pr_pow7(o0);
        if (g.t == 0) o0 = y;
        poseidon2_internal_hex(o0, o1, g, &tab.rc.v[12 * (rnd + 1)]);
    }
#pragma unroll 1
    for (int rnd = 26; rnd < 30; rnd++) {
        o0 = pr_pow7(o0);
        o1 = pr_pow7(o1);
        poseidon2_external_hex(o0, o1, g, rnd < 29 ? &tab.rcm.v[12 * (rnd + 1)] : nullptr);
    }
}

__device__ __forceinline__ void permute_hex(uint64_t &o0, uint64_t &o1, const HexGroup &g, const PoseidonTab &tab) {
    poseidon_permute_hex(o0, o1, g, tab);
}
__device__ __forceinline__ void permute_hex(uint64_t &o0, uint64_t &o1, const HexGroup2 &g, const Poseidon2Tab &tab) {
    poseidon2_permute_hex(o0, o1, g, tab);
}

// The group form of a hasher: HexOf<kPoseidon> or HexOf<kPoseidon2>.
template <int H>
using HexOf = typename std::conditional<H == kPoseidon, HexGroup, HexGroup2>::type;

// H(l || r) on a group: every lane calls; `active` groups load and store.
template <class G, class Tab>
__device__ __forceinline__ void hash_two_hex(const uint64_t *l, const uint64_t *r, uint64_t *out, bool active,
                                             const G &g, const Tab &tab) {
    uint64_t o0 = 0, o1 = 0;
    if (active) {
        o0 = gl_canon(g.t < 4 ? l[g.t] : r[g.t - 4]);
        if (g.t < 2) o1 = gl_canon(r[g.t + 2]);
    }
    permute_hex(o0, o1, g, tab);
    if (active && g.t < 4) out[g.t] = gl_canon(o0);
}

// Sponge of n words (zeknox's hash_or_noop: n <= 4 copies and zero-pads).
// n must be the same for all groups of a warp.
template <class G, class Tab>
__device__ __forceinline__ void hash_one_hex(const uint64_t *in, uint32_t n, uint64_t *out, bool active, const G &g,
                                             const Tab &tab) {
    if (n <= 4) {
        if (active && g.t < 4) out[g.t] = g.t < n ? in[g.t] : 0ull;
        return;
    }
    uint64_t o0 = 0, o1 = 0;
    for (uint32_t idx = 0; idx < n; idx += 8) {
        const uint32_t len = n - idx < 8 ? n - idx : 8;
        if (active) {
            if (g.t < len) o0 = gl_canon(in[idx + g.t]);
            if (g.t + 6 < len) o1 = gl_canon(in[idx + g.t + 6]);
        }
        permute_hex(o0, o1, g, tab);
    }
    if (active && g.t < 4) out[g.t] = gl_canon(o0);
}

}  // namespace zk
