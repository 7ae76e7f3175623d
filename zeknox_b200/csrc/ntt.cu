// Batched NTT / coset LDE / bit-reversing transpose for sm_100a.
//
// zeknox (native/ntt/ntt.cu:106-158, kernels.cu:14-392) runs one global
// radix-2 stage per launch plus bit-reversal, zero-extension, coset and
// normalisation passes.  Here a size-2^lg transform is split into P <= 3
// passes (lg = l_1 + ... + l_P, each l_p <= 12); every pass moves a group of
// lines (strided columns, or contiguous rows in the last pass) into shared
// memory, runs a 2^l_p-point transform there, applies the inter-pass twiddle
// and writes back, so the whole transform costs P reads and P writes of the
// data.  Zero-extension, the coset multiply and the 1/N scaling are folded
// into the first / last pass, and the last pass writes natural order directly
// (no bit-reversal pass).
//
// Decomposition (Cooley-Tukey over mixed radix): with N = N_1 * S_1,
//   X[k_1 + N_1 k'] = sum_r w_{S_1}^{r k'} [ w_N^{r k_1} sum_i x[i S_1 + r] w_{N_1}^{i k_1} ]
// pass 1 computes the bracket for every column r (stride S_1) in place, the
// remaining passes transform each contiguous block of S_1 elements the same
// way, and the last pass stores X at its natural index.
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>

#include "gl64.cuh"
#include "ntt.cuh"
#include "ntt_field.cuh"
#include "pdl.cuh"
#include "runtime.cuh"

namespace zk {

namespace {

using namespace ntf;

constexpr int kNttThreads = 256;
constexpr int kLinesElems = 1 << 13;  // elements per group held in shared memory

struct PassArgs {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t src_poly_stride;  // elements between consecutive polynomials
    uint64_t dst_poly_stride;
    uint32_t batches;
    uint32_t lg_n;      // log2 of the transform size N
    uint32_t l;         // log2 line length L of this pass
    uint32_t lg_s;      // log2 stride S of line elements (column pass); 0 in the last pass
    uint32_t lg_pre;    // log2 of the number of prefixes Q = N / (L * S)
    uint32_t lg_t;      // log2 lines per group T
    uint32_t l_first;   // log2 N_1 (digit split of the prefix, 3-pass last pass)
    uint32_t kind;      // 0 column pass, 1 last pass (rows), 2 single pass, 3 last pass to leaves
    // leaf layout output (kinds 2 and 3): element k of polynomial b goes to
    // dst[rev_lg(k) * leaf_stride + b] (the bit-reversing transpose, fused)
    uint32_t to_leaves;
    uint64_t leaf_stride;  // polynomials per leaf row (all of them, not just this chunk)
    // first pass: zero-extension and coset pre-multiply
    uint64_t n_valid;   // source elements per polynomial that are read (others are 0)
    const uint64_t *pre_lo, *pre_hi;  // coset powers (null: none)
    const uint64_t *pre_full;         // the same powers in one table (null: two-level only)
    uint32_t pre_h;
    // last pass: output scaling by coset^k * scale
    const uint64_t *post_lo, *post_hi;  // coset powers (null: none)
    const uint64_t *post_full;
    uint32_t post_h;
    uint64_t scale;     // 1 = none
    // twiddles
    const uint64_t *tw_lo, *tw_hi;  // omega_N powers (two-level)
    const uint64_t *tw_full;        // omega_N^e for every e < N (null above 2^20 points)
    uint32_t tw_h;
    const uint64_t *line_roots;     // omega_4096^j, j < 4096
    uint32_t inverse;               // direction of line_roots / tw (selects the DFT-8 constants)
};

__device__ __forceinline__ uint64_t pow2l(const uint64_t *lo, const uint64_t *hi, uint32_t h, uint64_t e) {
    return nt_mul(__ldg(lo + (e & ((1ull << h) - 1))), __ldg(hi + (e >> h)));
}
// b^e from the one-load table when there is one, else from the two-level table.
__device__ __forceinline__ uint64_t pow_at(const uint64_t *full, const uint64_t *lo, const uint64_t *hi, uint32_t h,
                                           uint64_t e) {
    return full ? __ldg(full + e) : pow2l(lo, hi, h, e);
}

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

// 8-byte asynchronous global -> shared copy (cp.async, no register staging),
// so a thread's loads of a tile are all in flight at once.
__device__ __forceinline__ void cp_async8(uint64_t *smem_dst, const uint64_t *gmem_src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// In-place DIF stages over T interleaved lines of length L = 2^l in shared
// memory (element e of line t at e * tp + t), from half-span 2^s_top down to
// 1: natural order in, bit-reversed out.  Stages are taken three at a time as
// mixed-radix Cooley-Tukey steps: a sub-transform of size M = 8q splits into
// 8-point DFTs over the elements o + j q (j < 8) followed by the twiddles
// omega_M^(o * rev3(j)) on output j, then q-point sub-transforms; one
// shared-memory round trip per step.  The 8-point DFTs multiply only by
// powers of two (dft8), so a step costs 7 general products per 8 elements
// instead of the 12 of three radix-2 stages, and the last step (q = 1) none.
// A radix-4 or radix-2 tail ends odd stage counts.  tw[e] = omega_L^e.
__device__ __forceinline__ void smem_dif(uint64_t *sm, const uint64_t *tw, uint32_t l, int s_top, uint32_t lg_t,
                                         uint32_t tp, bool inv) {
    const uint32_t T = 1u << lg_t;
    int s = s_top;
    while (s >= 2) {  // spans 4q, 2q, q with q = 2^(s-2); unit = 8 elements at stride q
        __syncthreads();
        const uint32_t lq = s - 2, q = 1u << lq;
        const uint32_t units = T << (l - 3);
        const uint32_t sh8 = l - 1 - s;  // omega_{8q}^j = tw[j << sh8]
        for (uint32_t u = threadIdx.x; u < units; u += blockDim.x) {
            const uint32_t t = u & (T - 1), w = u >> lg_t;
            const uint32_t o = w & (q - 1), e0 = ((w >> lq) << (lq + 3)) + o;
            uint64_t x[8];
#pragma unroll
            for (int k = 0; k < 8; k++) x[k] = sm[(e0 + k * q) * tp + t];
            dft8(x, inv);
            if (o != 0) {
                constexpr uint32_t rev3[8] = {0, 4, 2, 6, 1, 5, 3, 7};
#pragma unroll
                for (int j = 1; j < 8; j++) x[j] = nt_mul(x[j], tw[(o * rev3[j]) << sh8]);
            }
#pragma unroll
            for (int k = 0; k < 8; k++) sm[(e0 + k * q) * tp + t] = x[k];
        }
        s -= 3;
    }
    __syncthreads();
    if (s == 1) {  // spans 2 and 1: radix-4 units (the 4th root is +-2^48)
        const uint32_t units = T << (l - 2);
        for (uint32_t u = threadIdx.x; u < units; u += blockDim.x) {
            const uint32_t t = u & (T - 1), e0 = (u >> lg_t) << 2;
            const uint64_t x0 = sm[e0 * tp + t], x1 = sm[(e0 + 1) * tp + t], x2 = sm[(e0 + 2) * tp + t],
                           x3 = sm[(e0 + 3) * tp + t];
            const uint64_t a0 = nt_add(x0, x2), a2 = nt_sub(x0, x2), a1 = nt_add(x1, x3);
            const uint64_t a3 = inv ? gl_mul2_48(nt_sub(x3, x1)) : gl_mul2_48(nt_sub(x1, x3));
            sm[e0 * tp + t] = nt_add(a0, a1);
            sm[(e0 + 1) * tp + t] = nt_sub(a0, a1);
            sm[(e0 + 2) * tp + t] = nt_add(a2, a3);
            sm[(e0 + 3) * tp + t] = nt_sub(a2, a3);
        }
        __syncthreads();
    } else if (s == 0) {  // span 1
        const uint32_t units = T << (l - 1);
        for (uint32_t u = threadIdx.x; u < units; u += blockDim.x) {
            const uint32_t t = u & (T - 1), e0 = (u >> lg_t) << 1;
            uint64_t x0 = sm[e0 * tp + t], x1 = sm[(e0 + 1) * tp + t];
            bfly1(x0, x1);
            sm[e0 * tp + t] = x0;
            sm[(e0 + 1) * tp + t] = x1;
        }
        __syncthreads();
    }
}

// smem_dif with the line length (2^LG_L), the lines per block (2^LG_T), the
// first half-span (S) and the direction fixed at compile time: the unit loops
// unroll and every index but the thread's own folds to a constant.  Same
// steps and synchronisation as smem_dif.
template <int LG_L, int LG_T, int S, bool INV>
__device__ __forceinline__ void smem_dif_fixed(uint64_t *sm, const uint64_t *tw) {
    constexpr uint32_t T = 1u << LG_T, TP = T > 1 ? T + 1 : 1;
    if constexpr (S >= 2) {
        constexpr uint32_t LQ = S - 2, Q = 1u << LQ, SH8 = LG_L - 1 - S;
        constexpr uint32_t UNITS = T << (LG_L - 3);
        __syncthreads();
#pragma unroll
        for (uint32_t it = 0; it < (UNITS + kNttThreads - 1) / kNttThreads; it++) {
            const uint32_t u = threadIdx.x + it * kNttThreads;
            if (UNITS % kNttThreads == 0 || u < UNITS) {
                const uint32_t t = u & (T - 1), w = u >> LG_T;
                const uint32_t o = w & (Q - 1), e0 = ((w >> LQ) << (LQ + 3)) + o;
                uint64_t *b = sm + e0 * TP + t;
                uint64_t x[8];
#pragma unroll
                for (int k = 0; k < 8; k++) x[k] = b[k * Q * TP];
                dft8(x, INV);
                if constexpr (LQ > 0) {
                    if (o != 0) {
                        constexpr uint32_t rev3[8] = {0, 4, 2, 6, 1, 5, 3, 7};
#pragma unroll
                        for (int j = 1; j < 8; j++) x[j] = nt_mul(x[j], tw[(o * rev3[j]) << SH8]);
                    }
                }
#pragma unroll
                for (int k = 0; k < 8; k++) b[k * Q * TP] = x[k];
            }
        }
        smem_dif_fixed<LG_L, LG_T, S - 3, INV>(sm, tw);
    } else {
        __syncthreads();
        if constexpr (S == 1) {  // spans 2 and 1: radix-4 units
            constexpr uint32_t UNITS = T << (LG_L - 2);
#pragma unroll
            for (uint32_t it = 0; it < (UNITS + kNttThreads - 1) / kNttThreads; it++) {
                const uint32_t u = threadIdx.x + it * kNttThreads;
                if (UNITS % kNttThreads == 0 || u < UNITS) {
                    uint64_t *b = sm + ((u >> LG_T) << 2) * TP + (u & (T - 1));
                    const uint64_t x0 = b[0], x1 = b[TP], x2 = b[2 * TP], x3 = b[3 * TP];
                    const uint64_t a0 = nt_add(x0, x2), a2 = nt_sub(x0, x2), a1 = nt_add(x1, x3);
                    const uint64_t a3 = INV ? gl_mul2_48(nt_sub(x3, x1)) : gl_mul2_48(nt_sub(x1, x3));
                    b[0] = nt_add(a0, a1);
                    b[TP] = nt_sub(a0, a1);
                    b[2 * TP] = nt_add(a2, a3);
                    b[3 * TP] = nt_sub(a2, a3);
                }
            }
            __syncthreads();
        } else if constexpr (S == 0) {  // span 1
            constexpr uint32_t UNITS = T << (LG_L - 1);
#pragma unroll
            for (uint32_t it = 0; it < (UNITS + kNttThreads - 1) / kNttThreads; it++) {
                const uint32_t u = threadIdx.x + it * kNttThreads;
                if (UNITS % kNttThreads == 0 || u < UNITS) {
                    uint64_t *b = sm + ((u >> LG_T) << 1) * TP + (u & (T - 1));
                    uint64_t x0 = b[0], x1 = b[TP];
                    bfly1(x0, x1);
                    b[0] = x0;
                    b[TP] = x1;
                }
            }
            __syncthreads();
        }
    }
}

__host__ __device__ constexpr uint32_t brev_const(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

template <bool INV>
__global__ void __launch_bounds__(kNttThreads) ntt_pass_kernel(PassArgs a) {
    extern __shared__ uint64_t smem[];
    const uint32_t l = a.l, L = 1u << l;
    const uint32_t T = 1u << a.lg_t;
    const uint32_t tp = T > 1 ? T + 1 : 1;
    uint64_t *tw = smem;  // omega_L^e, e < L
    uint64_t *sm = smem + L;
    for (uint32_t j = threadIdx.x; j < L; j += blockDim.x) tw[j] = __ldg(a.line_roots + (j << (kLineLgMax - l)));
    pdl_wait();  // the previous pass's output (launch_after) is read and overwritten only from here on
    const uint64_t g = blockIdx.x;

    if (a.kind == 0) {
        // ---- column pass: lines r0 + t (t < T) of prefix q, elements at stride S
        const uint32_t lg_s = a.lg_s;
        const uint64_t S = 1ull << lg_s;
        const uint64_t groups_per_prefix = S >> a.lg_t;
        const uint64_t groups_per_poly = groups_per_prefix << a.lg_pre;
        const uint64_t poly = g / groups_per_poly;
        const uint64_t rem = g % groups_per_poly;
        const uint64_t q = rem / groups_per_prefix;
        const uint64_t r0 = (rem % groups_per_prefix) << a.lg_t;
        const uint64_t base = q << (l + lg_s);  // prefix block start within the polynomial
        const uint64_t *src = a.src + poly * a.src_poly_stride;
        uint64_t *dst = a.dst + poly * a.dst_poly_stride;
        // Only the first Lv = 2^lv elements of a line can be non-zero (zero
        // extension): the first l - lv DIF stages then reduce to writing block
        // b of the line as x_e * omega_L^(e * brev(b)), e < Lv.
        uint32_t lv = l;
        if (a.n_valid < ((uint64_t)L << lg_s) && base == 0) {
            const uint64_t nz = (a.n_valid + S - 1) >> lg_s;  // non-zero prefix of every line
            lv = nz <= 1 ? 0 : 64 - __clzll(nz - 1);
        }
        const uint32_t rr = l - lv;
        __syncthreads();
        if (rr >= 2) {
            // Stage the inputs (block 1 of the line) and their coset powers
            // (block 2) with asynchronous copies, so all of a thread's loads are
            // in flight together; each thread reads back only the slots it
            // staged, before its own replication overwrites them.
            for (uint32_t idx = threadIdx.x; idx < (T << lv); idx += blockDim.x) {
                const uint32_t t = idx & (T - 1), e = idx >> a.lg_t;
                const uint64_t i = base + ((uint64_t)e << lg_s) + r0 + t;
                if (i < a.n_valid) {
                    cp_async8(&sm[((1u << lv) + e) * tp + t], src + i);
                    if (a.pre_full) cp_async8(&sm[((2u << lv) + e) * tp + t], a.pre_full + i);
                }
            }
            cp_async_wait_all();
        }
        for (uint32_t idx = threadIdx.x; idx < (T << lv); idx += blockDim.x) {
            const uint32_t t = idx & (T - 1), e = idx >> a.lg_t;
            const uint64_t i = base + ((uint64_t)e << lg_s) + r0 + t;  // index within the polynomial
            uint64_t v = 0;
            if (i < a.n_valid) {
                if (rr >= 2) {
                    v = nt_canon(sm[((1u << lv) + e) * tp + t]);
                    if (a.pre_full) v = nt_mul(v, sm[((2u << lv) + e) * tp + t]);
                    else if (a.pre_lo) v = nt_mul(v, pow2l(a.pre_lo, a.pre_hi, a.pre_h, i));
                } else {
                    v = nt_canon(src[i]);
                    if (a.pre_lo) v = nt_mul(v, pow_at(a.pre_full, a.pre_lo, a.pre_hi, a.pre_h, i));
                }
            }
            sm[e * tp + t] = v;
            for (uint32_t b = 1; b < (1u << rr); b++)
                sm[((b << lv) + e) * tp + t] = nt_mul(v, tw[(e * brev_bits(b, rr)) & (L - 1)]);
        }
        smem_dif(sm, tw, l, (int)lv - 1, a.lg_t, tp, INV);
        // store with the inter-pass twiddle w_N^((r0 + t) k Q): one table load
        // each, or (no one-load table) stepped by k with a second product
        const uint32_t t = threadIdx.x & (T - 1);
        const uint32_t k0 = threadIdx.x >> a.lg_t, dk = blockDim.x >> a.lg_t;
        const uint64_t r = r0 + t;
        const uint64_t nmask = (1ull << a.lg_n) - 1;  // w_N has order N
        if (a.tw_full) {
            for (uint32_t k = k0; k < L; k += dk) {
                const uint64_t tw_k = __ldg(a.tw_full + (((r * k) << a.lg_pre) & nmask));
                dst[base + ((uint64_t)k << lg_s) + r] = nt_mul(sm[brev_bits(k, l) * tp + t], tw_k);
            }
            return;
        }
        uint64_t twk = pow2l(a.tw_lo, a.tw_hi, a.tw_h, ((r * k0) << a.lg_pre) & nmask);
        const uint64_t step = pow2l(a.tw_lo, a.tw_hi, a.tw_h, ((r * dk) << a.lg_pre) & nmask);
        for (uint32_t k = k0; k < L; k += dk) {
            const uint64_t v = nt_mul(sm[brev_bits(k, l) * tp + t], twk);
            dst[base + ((uint64_t)k << lg_s) + r] = v;
            twk = nt_mul(twk, step);
        }
        return;
    }

    // ---- row passes: T lines, each a contiguous run of L elements
    const uint64_t Q = 1ull << a.lg_pre;  // prefixes per polynomial (1 for a single pass)
    uint64_t poly0, c0;
    uint32_t nlines = T;
    if (a.kind == 1) {
        const uint64_t groups_per_poly = Q >> a.lg_t;
        poly0 = g / groups_per_poly;
        c0 = (g % groups_per_poly) << a.lg_t;  // first digit-reversed prefix of the group
    } else {
        poly0 = g << a.lg_t;
        c0 = 0;
        if (poly0 + T > a.batches) nlines = (uint32_t)(a.batches - poly0);
    }
    auto line_src = [&](uint32_t t) -> uint64_t {  // element offset of line t's start in src
        if (a.kind == 2) return (poly0 + t) * a.src_poly_stride;
        const uint64_t krev = c0 + t;  // k_1 + N_1 k_2 (3 passes) or k_1 (2 passes)
        const uint64_t mask1 = (1ull << a.l_first) - 1;
        const uint64_t kpos = ((krev & mask1) << (a.lg_pre - a.l_first)) | (krev >> a.l_first);
        return poly0 * a.src_poly_stride + (kpos << l);
    };
    for (uint32_t idx = threadIdx.x; idx < T * L; idx += blockDim.x) {
        const uint32_t e = idx & (L - 1), t = idx >> l;
        uint64_t v = 0;
        if (t < nlines) {
            if (a.kind == 2) {
                if (e < a.n_valid) {
                    v = nt_canon(a.src[line_src(t) + e]);
                    if (a.pre_lo) v = nt_mul(v, pow_at(a.pre_full, a.pre_lo, a.pre_hi, a.pre_h, e));
                }
            } else {
                cp_async8(&sm[e * tp + t], a.src + line_src(t) + e);
                continue;
            }
        }
        sm[e * tp + t] = v;
    }
    cp_async_wait_all();
    smem_dif(sm, tw, l, (int)l - 1, a.lg_t, tp, INV);
    if (a.kind == 1) {
        // natural index of line t's element k: krev + Q * k
        uint64_t *dst = a.dst + poly0 * a.dst_poly_stride;
        for (uint32_t idx = threadIdx.x; idx < T * L; idx += blockDim.x) {
            const uint32_t t = idx & (T - 1), k = idx >> a.lg_t;
            uint64_t v = sm[brev_bits(k, l) * tp + t];
            const uint64_t o = c0 + t + ((uint64_t)k << a.lg_pre);
            if (a.post_lo) v = nt_mul(v, pow_at(a.post_full, a.post_lo, a.post_hi, a.post_h, o));
            if (a.scale != 1) v = nt_mul(v, a.scale);
            dst[o] = v;
        }
    } else if (a.to_leaves) {
        // leaves[rev(k)][poly0 + t]: consecutive threads write consecutive polynomials
        for (uint32_t idx = threadIdx.x; idx < T * L; idx += blockDim.x) {
            const uint32_t t = idx & (T - 1), k = idx >> a.lg_t;
            if (t >= nlines) continue;
            const uint64_t v = sm[brev_bits(k, l) * tp + t];
            a.dst[(uint64_t)brev_bits(k, l) * a.leaf_stride + poly0 + t] = v;
        }
    } else {
        for (uint32_t idx = threadIdx.x; idx < T * L; idx += blockDim.x) {
            const uint32_t k = idx & (L - 1), t = idx >> l;
            if (t >= nlines) continue;
            uint64_t v = sm[brev_bits(k, l) * tp + t];
            if (a.post_lo) v = nt_mul(v, pow_at(a.post_full, a.post_lo, a.post_hi, a.post_h, k));
            if (a.scale != 1) v = nt_mul(v, a.scale);
            a.dst[(poly0 + t) * a.dst_poly_stride + k] = v;
        }
    }
}

// Last pass of a multi-pass transform writing the leaf layout: a block takes
// the same prefix (line krev) of 2^lg_t consecutive polynomials, so that every
// leaf row receives 2^lg_t contiguous elements.  Element k of line krev has
// natural index o = krev + Q k and goes to dst[rev_lg(o) * leaf_stride + b].
template <bool INV>
__global__ void __launch_bounds__(kNttThreads) ntt_last_pass_leaves(PassArgs a) {
    extern __shared__ uint64_t smem[];
    const uint32_t l = a.l, L = 1u << l;
    // Row pitch as pass_smem sizes it (one polynomial: no padding column).
    const uint32_t P = 1u << a.lg_t, tp = P > 1 ? P + 1 : 1;
    uint64_t *tw = smem;
    uint64_t *sm = smem + L;
    for (uint32_t j = threadIdx.x; j < L; j += blockDim.x) tw[j] = __ldg(a.line_roots + (j << (kLineLgMax - l)));
    pdl_wait();  // the previous pass's output is read only from here on
    const uint64_t Q = 1ull << a.lg_pre;
    const uint64_t krev = blockIdx.x % Q, pg = blockIdx.x / Q;
    const uint64_t p0 = pg << a.lg_t;  // first polynomial of the group (within the chunk)
    const uint32_t np = (uint32_t)min((uint64_t)P, a.batches - p0);
    const uint64_t mask1 = (1ull << a.l_first) - 1;
    const uint64_t kpos = ((krev & mask1) << (a.lg_pre - a.l_first)) | (krev >> a.l_first);
    for (uint32_t idx = threadIdx.x; idx < P * L; idx += blockDim.x) {
        const uint32_t e = idx & (L - 1), p = idx >> l;
        if (p < np) cp_async8(&sm[e * tp + p], a.src + (p0 + p) * a.src_poly_stride + (kpos << l) + e);
        else sm[e * tp + p] = 0ull;
    }
    cp_async_wait_all();
    smem_dif(sm, tw, l, (int)l - 1, a.lg_t, tp, INV);
    const uint32_t lg = a.lg_n;
    for (uint32_t idx = threadIdx.x; idx < P * L; idx += blockDim.x) {
        const uint32_t p = idx & (P - 1), k = idx >> a.lg_t;
        if (p >= np) continue;
        const uint64_t o = krev + ((uint64_t)k << a.lg_pre);
        const uint64_t row = __brevll(o) >> (64 - lg);
        a.dst[row * a.leaf_stride + p0 + p] = sm[brev_bits(k, l) * tp + p];
    }
}


using PassKernel = void (*)(PassArgs);

// The column pass (kind 0) of ntt_pass_kernel with the line length (2^LG_L),
// lines per block (2^LG_T) and non-zero prefix of every line (2^LV, LV ==
// LG_L: no zero extension) fixed at compile time, for launches with the
// one-load twiddle table and, when there is a coset, the one-load coset table
// (transforms of up to 2^20 points).  Thread t's elements are t + 256 j: its
// line (t mod T) is fixed, and its element and output positions step by
// constants.
template <int LG_L, int LG_T, int LV, bool INV>
__global__ void __launch_bounds__(kNttThreads) ntt_column_fixed(PassArgs a) {
    constexpr uint32_t L = 1u << LG_L, T = 1u << LG_T, TP = T > 1 ? T + 1 : 1, RR = LG_L - LV;
    static_assert(RR == 0 || RR >= 2, "a one-stage zero extension takes the generic pass");
    static_assert(T <= kNttThreads && (T << LG_L) % kNttThreads == 0, "block elements: a multiple of the threads");
    extern __shared__ uint64_t smem[];
    uint64_t *tw = smem;  // omega_L^e, e < L
    uint64_t *sm = smem + L;
    for (uint32_t j = threadIdx.x; j < L; j += kNttThreads) tw[j] = __ldg(a.line_roots + (j << (kLineLgMax - LG_L)));
    pdl_wait();
    const uint32_t lg_s = a.lg_s, lg_gpp = lg_s - LG_T;  // groups per prefix: 2^lg_gpp
    const uint64_t g = blockIdx.x;
    const uint64_t poly = g >> (lg_gpp + a.lg_pre);
    const uint64_t rem = g & ((1ull << (lg_gpp + a.lg_pre)) - 1);
    const uint64_t base = (rem >> lg_gpp) << (LG_L + lg_s);  // prefix block start within the polynomial
    const uint32_t t = threadIdx.x & (T - 1);
    const uint64_t r = ((rem & ((1ull << lg_gpp) - 1)) << LG_T) + t;  // this thread's line
    const uint64_t *src = a.src + poly * a.src_poly_stride + base + r;  // element e of the line: src[e << lg_s]
    uint64_t *dst = a.dst + poly * a.dst_poly_stride + base + r;
    const uint64_t i0 = base + r;  // index within the polynomial of the line's element 0
    const uint32_t e0 = threadIdx.x >> LG_T;
    constexpr uint32_t DE = kNttThreads >> LG_T;  // element step between j and j + 1
    const uint64_t *pre = a.pre_full;
    __syncthreads();  // the twiddle table, read by the replication below
    if constexpr (RR >= 2) {
        // inputs (line block 1) and coset powers (line block 2) staged with asynchronous copies;
        // each thread reads back only the slots it staged, before its replication overwrites them
        constexpr uint32_t NE = (T << LV) < kNttThreads ? 1 : (T << LV) / kNttThreads;
        if ((T << LV) >= kNttThreads || threadIdx.x < (T << LV)) {
#pragma unroll
            for (uint32_t j = 0; j < NE; j++) {
                const uint32_t e = e0 + j * DE;
                const uint64_t i = i0 + ((uint64_t)e << lg_s);
                if (i < a.n_valid) {
                    cp_async8(&sm[((1u << LV) + e) * TP + t], src + ((uint64_t)e << lg_s));
                    if (pre) cp_async8(&sm[((2u << LV) + e) * TP + t], pre + i);
                }
            }
        }
        cp_async_wait_all();
        if ((T << LV) >= kNttThreads || threadIdx.x < (T << LV)) {
#pragma unroll
            for (uint32_t j = 0; j < NE; j++) {
                const uint32_t e = e0 + j * DE;
                const uint64_t i = i0 + ((uint64_t)e << lg_s);
                uint64_t v = 0;
                if (i < a.n_valid) {
                    v = nt_canon(sm[((1u << LV) + e) * TP + t]);
                    if (pre) v = nt_mul(v, sm[((2u << LV) + e) * TP + t]);
                }
                sm[e * TP + t] = v;
#pragma unroll
                for (uint32_t b = 1; b < (1u << RR); b++)
                    sm[((b << LV) + e) * TP + t] = nt_mul(v, tw[(e * brev_const(b, RR)) & (L - 1)]);
            }
        }
    } else {
#pragma unroll
        for (uint32_t j = 0; j < (T << LG_L) / kNttThreads; j++) {
            const uint32_t e = e0 + j * DE;
            const uint64_t i = i0 + ((uint64_t)e << lg_s);
            uint64_t v = 0;
            if (i < a.n_valid) {
                v = nt_canon(src[(uint64_t)e << lg_s]);
                if (pre) v = nt_mul(v, __ldg(pre + i));
            }
            sm[e * TP + t] = v;
        }
    }
    smem_dif_fixed<LG_L, LG_T, (int)LV - 1, INV>(sm, tw);
    // store with the inter-pass twiddle w_N^(r k Q), one table load each (the
    // table has N <= 2^20 entries, so exponents wrap mod 2^32 harmlessly)
    const uint32_t nmask = (uint32_t)((1ull << a.lg_n) - 1);
    const uint32_t krt = __brev(e0) >> (32 - LG_L);  // rev(k) of the first k = e0
    const uint32_t rk0 = (uint32_t)r * e0, rdk = (uint32_t)r * DE;
    const uint32_t lg_pre = a.lg_pre;
    const uint64_t *twf = a.tw_full;
#pragma unroll
    for (uint32_t m = 0; m < (T << LG_L) / kNttThreads; m++) {
        const uint32_t k = e0 + m * DE;
        const uint32_t kr = krt | brev_const(m * DE, LG_L);
        const uint64_t tw_k = __ldg(twf + (((rk0 + m * rdk) << lg_pre) & nmask));
        dst[(uint64_t)k << lg_s] = nt_mul(sm[kr * TP + t], tw_k);
    }
}

// The compiled (line length, lines per block, non-zero prefix) triples of
// ntt_column_fixed, per direction.
template <bool INV>
PassKernel column_fixed_kernel(uint32_t l, uint32_t lg_t, uint32_t lv) {
#define ZK_COLUMN_CASES(LG_L, LG_T)                                                        \
    case ((LG_L) << 8 | (LG_T) << 4 | 0): return ntt_column_fixed<LG_L, LG_T, LG_L, INV>;      \
    case ((LG_L) << 8 | (LG_T) << 4 | 2): return ntt_column_fixed<LG_L, LG_T, LG_L - 2, INV>;  \
    case ((LG_L) << 8 | (LG_T) << 4 | 3): return ntt_column_fixed<LG_L, LG_T, LG_L - 3, INV>;
    if (lv > l) return nullptr;
    switch (l << 8 | lg_t << 4 | (l - lv)) {
        ZK_COLUMN_CASES(7, 5) ZK_COLUMN_CASES(8, 5) ZK_COLUMN_CASES(9, 4) ZK_COLUMN_CASES(10, 3)
        ZK_COLUMN_CASES(11, 2) ZK_COLUMN_CASES(12, 1)
        ZK_COLUMN_CASES(7, 4) ZK_COLUMN_CASES(8, 4) ZK_COLUMN_CASES(9, 3) ZK_COLUMN_CASES(10, 2)
        ZK_COLUMN_CASES(11, 1) ZK_COLUMN_CASES(12, 0)
        default: return nullptr;
    }
#undef ZK_COLUMN_CASES
}

// The last pass of a multi-pass transform writing rows (kind 1 of
// ntt_pass_kernel) with the line length (2^LG_L) and lines per block (2^LG_T)
// fixed at compile time.  Line t of the block is prefix krev = c0 + t; its
// element k has natural index c0 + t + Q k.  Thread t's elements are
// t + 256 j, so the output column (t mod T) is fixed and k = t / T + j * 256 / T.
template <int LG_L, int LG_T, bool INV>
__global__ void __launch_bounds__(kNttThreads) ntt_rows_fixed(PassArgs a) {
    constexpr uint32_t L = 1u << LG_L, T = 1u << LG_T, TP = T > 1 ? T + 1 : 1;
    constexpr uint32_t PER = T * L / kNttThreads;  // elements per thread
    static_assert(T * L % kNttThreads == 0 && T <= kNttThreads, "block elements: a multiple of the threads");
    extern __shared__ uint64_t smem[];
    uint64_t *tw = smem;
    uint64_t *sm = smem + L;
    for (uint32_t j = threadIdx.x; j < L; j += kNttThreads) tw[j] = __ldg(a.line_roots + (j << (kLineLgMax - LG_L)));
    pdl_wait();  // the previous pass's output is read only from here on
    const uint32_t lg_pre = a.lg_pre, lg_gpp = lg_pre - LG_T;  // groups per polynomial: 2^lg_gpp
    const uint64_t g = blockIdx.x, poly0 = g >> lg_gpp, c0 = (g & ((1ull << lg_gpp) - 1)) << LG_T;
    const uint64_t mask1 = (1ull << a.l_first) - 1;
    const uint64_t *src = a.src + poly0 * a.src_poly_stride;
#pragma unroll
    for (uint32_t j = 0; j < PER; j++) {
        uint32_t e, t;  // element t + 256 j: line position e of line t
        if constexpr (LG_L >= 8) {
            e = threadIdx.x + kNttThreads * (j & (L / kNttThreads - 1));
            t = j / (L / kNttThreads);
        } else {
            e = threadIdx.x & (L - 1);
            t = (threadIdx.x >> LG_L) + j * (kNttThreads >> LG_L);
        }
        const uint64_t krev = c0 + t;  // k_1 + N_1 k_2 (3 passes) or k_1 (2 passes)
        const uint64_t kpos = ((krev & mask1) << (lg_pre - a.l_first)) | (krev >> a.l_first);
        cp_async8(&sm[e * TP + t], src + (kpos << LG_L) + e);
    }
    cp_async_wait_all();
    smem_dif_fixed<LG_L, LG_T, LG_L - 1, INV>(sm, tw);
    constexpr uint32_t DK = kNttThreads >> LG_T;  // step of k between j and j + 1
    const uint32_t t = threadIdx.x & (T - 1), kt = threadIdx.x >> LG_T;
    const uint32_t krt = __brev(kt) >> (32 - LG_L);
    const uint64_t o0 = c0 + t + ((uint64_t)kt << lg_pre);  // natural index of this thread's first element
    uint64_t *dst = a.dst + poly0 * a.dst_poly_stride + o0;
    const uint64_t *col = sm + t;
#pragma unroll
    for (uint32_t j = 0; j < PER; j++) {
        const uint32_t kr = krt | brev_const(j * DK, LG_L);
        const uint64_t step = (uint64_t)(j * DK) << lg_pre;
        uint64_t v = col[kr * TP];
        if (a.post_lo) v = nt_mul(v, pow_at(a.post_full, a.post_lo, a.post_hi, a.post_h, o0 + step));
        if (a.scale != 1) v = nt_mul(v, a.scale);
        dst[step] = v;
    }
}

// The compiled (line length, lines per block) pairs of ntt_rows_fixed, per direction.
template <bool INV>
PassKernel rows_fixed_kernel(uint32_t l, uint32_t lg_t) {
#define ZK_ROWS_CASE(LG_L, LG_T) \
    case ((LG_L) << 4 | (LG_T)): return ntt_rows_fixed<LG_L, LG_T, INV>;
    switch (l << 4 | lg_t) {
        ZK_ROWS_CASE(6, 5) ZK_ROWS_CASE(7, 5) ZK_ROWS_CASE(8, 5) ZK_ROWS_CASE(9, 4) ZK_ROWS_CASE(10, 3)
        ZK_ROWS_CASE(11, 2) ZK_ROWS_CASE(12, 1)
        default: return nullptr;
    }
#undef ZK_ROWS_CASE
}

// ntt_last_pass_leaves with the line length (2^LG_L) and polynomials per
// block (2^LG_P) fixed at compile time, for blocks whose P * L elements are a
// multiple of the thread count: thread t's elements are t + 256 i, so their
// polynomial, line position and leaf row split into a part of t, computed
// once, and a part of i, a constant.  A line element k goes to the leaf row
// rev_lg(krev + Q k) = (rev_lg_pre(krev) << LG_L) | rev_LG_L(k).
template <int LG_L, int LG_P>
__global__ void __launch_bounds__(kNttThreads) ntt_leaves_fixed(PassArgs a) {
    constexpr uint32_t L = 1u << LG_L, P = 1u << LG_P, TP = P > 1 ? P + 1 : 1;
    constexpr uint32_t PER = P * L / kNttThreads;  // elements per thread
    static_assert(P * L % kNttThreads == 0 && LG_P <= 8, "block elements: a multiple of the thread count");
    extern __shared__ uint64_t smem[];
    uint64_t *tw = smem;
    uint64_t *sm = smem + L;
    for (uint32_t j = threadIdx.x; j < L; j += kNttThreads) tw[j] = __ldg(a.line_roots + (j << (kLineLgMax - LG_L)));
    pdl_wait();  // the previous pass's output is read only from here on
    const uint32_t lg_pre = a.lg_pre;
    // With 16 or more polynomial groups (leaf rows of at least 16 runs written
    // by different blocks), consecutive blocks take the groups of one set of
    // leaf rows, so each row's sectors are completed while they are in L2
    // (135 x 2^15 -> 2^18, 17 groups: 0.613 -> 0.604 ms); with fewer groups,
    // consecutive blocks take consecutive rows of one group (that order
    // measured 0.3-4 % faster there).
    const uint32_t ngroups = (uint32_t)((a.batches + P - 1) >> LG_P);
    uint64_t krev, p0;
    if (ngroups >= 16) {
        krev = blockIdx.x / ngroups;
        p0 = (uint64_t)(blockIdx.x - krev * ngroups) << LG_P;
    } else {
        krev = blockIdx.x & ((1ull << lg_pre) - 1);
        p0 = (uint64_t)(blockIdx.x >> lg_pre) << LG_P;
    }
    const uint32_t np = (uint32_t)min((uint64_t)P, a.batches - p0);
    const uint64_t mask1 = (1ull << a.l_first) - 1;
    const uint64_t kpos = ((krev & mask1) << (lg_pre - a.l_first)) | (krev >> a.l_first);
    const uint64_t stride = a.src_poly_stride;
    const uint64_t *src = a.src + p0 * stride + (kpos << LG_L);
#pragma unroll
    for (uint32_t i = 0; i < PER; i++) {
        uint32_t e, p;  // element t + 256 i: line position e of polynomial p
        if constexpr (LG_L >= 8) {
            e = threadIdx.x + kNttThreads * (i & (L / kNttThreads - 1));
            p = i / (L / kNttThreads);
        } else {
            e = threadIdx.x & (L - 1);
            p = (threadIdx.x >> LG_L) + i * (kNttThreads >> LG_L);
        }
        if (p < np) cp_async8(&sm[e * TP + p], src + p * stride + e);
        else sm[e * TP + p] = 0ull;
    }
    cp_async_wait_all();
    smem_dif_fixed<LG_L, LG_P, LG_L - 1, false>(sm, tw);
    // stores: element t + 256 i is polynomial p = t mod P at line position
    // k = t / P + i * (256 / P), whose bit-reversal is rev(t / P) | rev(i * 256 / P)
    const uint32_t p = threadIdx.x & (P - 1);
    if (p >= np) return;
    const uint32_t kt = threadIdx.x >> LG_P;
    const uint32_t krt = __brev(kt) >> (32 - LG_L);
    const uint64_t ls = a.leaf_stride;
    uint64_t *dst = a.dst + p0 + p + (((uint64_t)brev_bits((uint32_t)krev, lg_pre) << LG_L) | krt) * ls;
    const uint64_t *col = sm + p;
#pragma unroll
    for (uint32_t i = 0; i < PER; i++) {
        constexpr uint32_t KS = 8 - LG_P;  // log2 of the step of k between i and i + 1
        const uint32_t kri = brev_const(i << KS, LG_L);  // a constant for each i
        dst[(uint64_t)kri * ls] = col[(krt | kri) * TP];
    }
}

// The compiled (line length, polynomials per block) pairs of ntt_leaves_fixed.
#define ZK_LEAVES_CASE(LG_L, LG_P) \
    case ((LG_L) << 4 | (LG_P)): return ntt_leaves_fixed<LG_L, LG_P>;
PassKernel leaves_fixed_kernel(uint32_t l, uint32_t lg_t) {
    switch (l << 4 | lg_t) {
        ZK_LEAVES_CASE(6, 2) ZK_LEAVES_CASE(6, 3) ZK_LEAVES_CASE(6, 4)
        ZK_LEAVES_CASE(7, 1) ZK_LEAVES_CASE(7, 2) ZK_LEAVES_CASE(7, 3) ZK_LEAVES_CASE(7, 4)
        ZK_LEAVES_CASE(8, 0) ZK_LEAVES_CASE(8, 1) ZK_LEAVES_CASE(8, 2) ZK_LEAVES_CASE(8, 3) ZK_LEAVES_CASE(8, 4)
        ZK_LEAVES_CASE(9, 0) ZK_LEAVES_CASE(9, 1) ZK_LEAVES_CASE(9, 2) ZK_LEAVES_CASE(9, 3) ZK_LEAVES_CASE(9, 4)
        ZK_LEAVES_CASE(10, 0) ZK_LEAVES_CASE(10, 1) ZK_LEAVES_CASE(10, 2) ZK_LEAVES_CASE(10, 3)
        ZK_LEAVES_CASE(11, 0) ZK_LEAVES_CASE(11, 1) ZK_LEAVES_CASE(11, 2)
        ZK_LEAVES_CASE(12, 0) ZK_LEAVES_CASE(12, 1)
        default: return nullptr;
    }
}
#undef ZK_LEAVES_CASE

// out[rev(k) * B + b] = in[b * N + k] (zeknox kernels.cu:94-135).  A block
// takes kTrK consecutive k of a chunk of up to kTrMaxPolys polynomials
// (reads: kTrK contiguous words per polynomial) and writes each of the kTrK
// output rows as one contiguous run of the chunk's words, so a chunk holding
// every polynomial writes whole leaf rows.  The shared tile is [k][poly] with
// an odd row pitch (no bank conflicts on either side).
constexpr int kTrK = 32;
constexpr uint32_t kTrMaxPolys = 192;
template <bool VEC>
__global__ void __launch_bounds__(256) transpose_rev_kernel(uint64_t *__restrict__ out, const uint64_t *__restrict__ in,
                                                            uint32_t lg_n, uint32_t batches, uint32_t chunk) {
    extern __shared__ uint64_t tile[];
    const uint64_t N = 1ull << lg_n;
    const uint32_t K = N < (uint64_t)kTrK ? (uint32_t)N : kTrK;
    const uint64_t k0 = (uint64_t)blockIdx.x * K;
    const uint32_t b0 = blockIdx.y * chunk;
    const uint32_t nb = min(chunk, batches - b0);
    const uint32_t pitch = nb | 1;
    if (VEC && K == kTrK) {  // 16-byte loads of two consecutive k (k0 is a multiple of 32)
        constexpr uint32_t H = kTrK / 2;
#pragma unroll 4
        for (uint32_t idx = threadIdx.x; idx < nb * H; idx += blockDim.x) {
            const uint32_t bl = idx / H, kl = 2 * (idx % H);
            const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(in + (uint64_t)(b0 + bl) * N + k0 + kl);
            tile[kl * pitch + bl] = v.x;
            tile[(kl + 1) * pitch + bl] = v.y;
        }
    } else {
        for (uint32_t idx = threadIdx.x; idx < nb * K; idx += blockDim.x) {
            const uint32_t bl = idx / K, kl = idx % K;
            tile[kl * pitch + bl] = in[(uint64_t)(b0 + bl) * N + k0 + kl];
        }
    }
    __syncthreads();
#pragma unroll 4
    for (uint32_t idx = threadIdx.x; idx < nb * K; idx += blockDim.x) {
        const uint32_t kl = idx / nb, bl = idx % nb;
        const uint64_t k = k0 + kl;
        const uint64_t r = lg_n ? (__brevll(k) >> (64 - lg_n)) : 0;
        out[r * batches + b0 + bl] = tile[kl * pitch + bl];
    }
}

// Salt rows: uniform field elements from a counter-based SplitMix64 stream.
__global__ void salt_kernel(uint64_t *out, uint64_t count, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t ctr = i, z;
        do {
            z = seed + (ctr + 1) * 0x9E3779B97F4A7C15ull;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            ctr += count;
        } while (z >= ZK_P);
        out[i] = z;
    }
}

struct Plan {
    int passes;
    uint32_t l[3];
};

// to_leaves: the last pass writes each leaf row in runs of 8 polynomials only
// while its lines are at most 2^9 points (shared memory); with two passes the
// runs shrink to 4 words at 2^20-2^21, 2 at 2^22-2^23 and 1 at 2^24.  Measured
// (B200, LDE to leaves): three passes win from 2^22 on (2^22 x 48 polys 7.5 ->
// 6.7 ms, 2^23 x 24 8.4 -> 6.8 ms, 2^24 x 12 12.0 -> 8.7 ms) and lose below
// (2^20 x 64 1.7 -> 2.4 ms), so transforms of 2^22..2^24 points take three.
Plan make_plan(uint32_t lg, bool to_leaves = false) {
    Plan p{};
    if (to_leaves && lg >= 22 && lg <= 24) {
        p.passes = 3;
        p.l[0] = (lg + 2) / 3;
        p.l[1] = (lg - p.l[0] + 1) / 2;
        p.l[2] = lg - p.l[0] - p.l[1];
        return p;
    }
    if (lg <= 12) {
        p.passes = 1;
        p.l[0] = lg;
    } else if (lg <= 24) {
        p.passes = 2;
        p.l[0] = (lg + 1) / 2;
        p.l[1] = lg - p.l[0];
    } else {
        p.passes = 3;
        p.l[0] = (lg + 2) / 3;
        p.l[1] = (lg - p.l[0] + 1) / 2;
        p.l[2] = lg - p.l[0] - p.l[1];
    }
    return p;
}

uint32_t ilog2_floor(uint64_t x) { return 63 - __builtin_clzll(x); }

size_t pass_smem(uint32_t l, uint32_t lg_t) {
    const uint64_t T = 1ull << lg_t, tp = T > 1 ? T + 1 : 1;
    const uint64_t L = 1ull << l;
    return (size_t)(L + L * tp) * sizeof(uint64_t);
}

// after_pass: the previous launch on `s` is the pass before this one of the
// same transform, so this pass may start while it drains (pdl.cuh).
// ZK_NTT_GENERIC_PASSES=1 keeps the runtime-shaped pass kernels for every
// shape (same outputs; for comparing the two forms).
bool fixed_passes_enabled() {
    static const bool on = [] {
        const char *e = getenv("ZK_NTT_GENERIC_PASSES");
        return !(e && e[0] == '1');
    }();
    return on;
}

// The 160 KB dynamic shared memory attribute, once per (kernel, device): a
// fixed table (no host allocation on the launch path, which the
// allocation-free LDE shares), one device bit mask per kernel.
void set_smem_attr(PassKernel kern) {
    constexpr int kSlots = 512;
    static std::mutex mu;
    static PassKernel keys[kSlots];
    static uint64_t devs[kSlots];
    const int dev = current_device();
    std::lock_guard<std::mutex> g(mu);
    int i = (int)(((uintptr_t)kern >> 4) % kSlots);
    for (int n = 0; n < kSlots && keys[i] && keys[i] != kern; n++) i = (i + 1) % kSlots;
    const bool known = keys[i] == kern && dev < 64 && (devs[i] >> dev & 1);
    if (known) return;
    ZK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    if (!keys[i] || keys[i] == kern) {  // remembered unless the table is full (then set on every launch)
        keys[i] = kern;
        if (dev < 64) devs[i] |= 1ull << dev;
    }
}

// The transform's direction is a template parameter of the pass kernels (the
// 8-point DFT's root multiplies differ), so each compiled kernel holds one form.
void launch_pass(const PassArgs &a, uint64_t groups, cudaStream_t s, bool after_pass) {
    const size_t smem = pass_smem(a.l, a.lg_t);
    static std::atomic<uint64_t> attr_set{0};  // one bit per device
    const int dev = current_device();
    if (dev < 64 && !(attr_set.load() & (1ull << dev))) {
        ZK_CUDA(cudaFuncSetAttribute(ntt_pass_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        ZK_CUDA(cudaFuncSetAttribute(ntt_pass_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        attr_set.fetch_or(1ull << dev);
    }
    require(groups < (1ull << 31), "transform too large for one launch");
    PassKernel kern = a.inverse ? ntt_pass_kernel<true> : ntt_pass_kernel<false>;
    if (a.kind == 0 && a.tw_full && (a.pre_full || !a.pre_lo) && fixed_passes_enabled()) {
        // the compile-time column pass, when this shape has one (lv as the kernel computes it)
        const uint64_t S = 1ull << a.lg_s, L = 1ull << a.l;
        uint32_t lv = a.l;
        if (a.n_valid < (L << a.lg_s) && a.lg_pre == 0) {
            const uint64_t nz = (a.n_valid + S - 1) >> a.lg_s;
            lv = nz <= 1 ? 0 : 64 - __builtin_clzll(nz - 1);
        }
        PassKernel fixed = a.inverse ? column_fixed_kernel<true>(a.l, a.lg_t, lv)
                                     : column_fixed_kernel<false>(a.l, a.lg_t, lv);
        if (fixed) {
            set_smem_attr(fixed);
            kern = fixed;
        }
    }
    if (a.kind == 1 && fixed_passes_enabled()) {
        PassKernel fixed = a.inverse ? rows_fixed_kernel<true>(a.l, a.lg_t) : rows_fixed_kernel<false>(a.l, a.lg_t);
        if (fixed) {
            set_smem_attr(fixed);
            kern = fixed;
        }
    }
    if (after_pass) {
        launch_after(kern, (unsigned)groups, kNttThreads, smem, s, a);
        return;
    }
    kern<<<(unsigned)groups, kNttThreads, smem, s>>>(a);
    ZK_CHECK_LAUNCH();
}

void launch_leaves_pass(const PassArgs &a, uint64_t groups, cudaStream_t s) {
    const size_t smem = pass_smem(a.l, a.lg_t);
    PassKernel fixed = fixed_passes_enabled() ? leaves_fixed_kernel(a.l, a.lg_t) : nullptr;
    PassKernel kern = fixed ? fixed : ntt_last_pass_leaves<false>;
    set_smem_attr(kern);
    require(groups < (1ull << 31), "transform too large for one launch");
    require(!a.inverse, "the leaf layout is written by forward transforms only");
    launch_after(kern, (unsigned)groups, kNttThreads, smem, s, a);  // always after a pass
}

}  // namespace

// ---- autotuning of the LDE -> leaves stage ----
// Per (transform size, batch-size class): the number of passes (2 or 3) and
// the polynomials per block of the leaves pass (2^lg_t), chosen by timing the
// candidates on the device (ntt_autotune_leaves).  Untuned shapes use the
// static choice of make_plan and 8 polynomials per block.
struct LeavesChoice {
    uint8_t passes = 0;  // 0: no entry
    uint8_t lg_t = 0;
};
std::mutex g_tune_mu;
std::map<uint64_t, LeavesChoice> g_tune;
thread_local const LeavesChoice *t_tune_override = nullptr;  // set while the tuner times a candidate

uint64_t tune_key(uint32_t lg, uint64_t batches) {
    const uint64_t cls = 64 - __builtin_clzll(batches);  // batch-size class: bit length
    return ((uint64_t)lg << 8) | cls;
}

LeavesChoice leaves_choice(uint32_t lg, uint64_t batches) {
    if (t_tune_override) return *t_tune_override;
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(tune_key(lg, batches));
    return it == g_tune.end() ? LeavesChoice{} : it->second;
}

Plan plan_with_passes(uint32_t lg, int passes) {
    Plan p{};
    p.passes = passes;
    if (passes == 2) {
        p.l[0] = (lg + 1) / 2;
        p.l[1] = lg - p.l[0];
    } else {
        p.l[0] = (lg + 2) / 3;
        p.l[1] = (lg - p.l[0] + 1) / 2;
        p.l[2] = lg - p.l[0] - p.l[1];
    }
    return p;
}

// Leaves-pass block of 2^lg_t polynomials over lines of 2^l points fits the
// 160 KB of dynamic shared memory the pass launches with.
bool leaves_fits(uint32_t l, uint32_t lg_t) { return pass_smem(l, lg_t) <= 160 * 1024; }

// Arguments shared by every pass of one transform: the direction's tables
// (roots: omega_N powers, two-level plus the one-load table when there is
// one; line_roots_dev: omega_4096^j), coset tables and scale of the job.
static PassArgs transform_args(const NttJob &j, const PowTable &roots, const uint64_t *line_roots_dev) {
    PassArgs base{};
    base.lg_n = j.lg;
    base.tw_lo = roots.lo();
    base.tw_hi = roots.hi();
    base.tw_h = roots.h;
    base.tw_full = roots.full;
    base.line_roots = line_roots_dev;
    base.inverse = j.inverse ? 1u : 0u;
    base.scale = j.scale;
    base.batches = (uint32_t)j.batches;
    if (j.pre_coset) {
        base.pre_lo = j.pre_coset->lo();
        base.pre_hi = j.pre_coset->hi();
        base.pre_h = j.pre_coset->h;
        base.pre_full = j.pre_coset->full;
    }
    if (j.post_coset) {
        base.post_lo = j.post_coset->lo();
        base.post_hi = j.post_coset->hi();
        base.post_h = j.post_coset->h;
        base.post_full = j.post_coset->full;
    }
    return base;
}

// Launches the passes of `plan` for job j (every transform of this file goes
// through here): one pass, or per chunk of polynomials the column passes into
// j.scratch and the last pass (rows, or the leaf layout with `tuned`'s
// polynomials per block when it names one).
static void launch_plan(const NttJob &j, const PassArgs &base, const Plan &plan, const LeavesChoice &tuned,
                 cudaStream_t s) {
    const uint32_t lg = j.lg;
    const uint64_t N = 1ull << lg;
    if (plan.passes == 1) {
        PassArgs a = base;
        a.kind = 2;
        a.l = lg;
        a.lg_pre = 0;
        a.lg_t = std::min<uint32_t>(ilog2_floor(kLinesElems) - lg, 6);
        a.src = j.src;
        a.dst = j.dst;
        a.src_poly_stride = j.src_stride;
        a.dst_poly_stride = j.dst_stride;
        a.n_valid = j.n_valid;
        if (j.to_leaves) {
            a.to_leaves = 1;
            a.leaf_stride = j.leaf_stride ? j.leaf_stride : j.batches;
            a.lg_t = std::min<uint32_t>(a.lg_t, 4);
        }
        const uint64_t groups = (j.batches + (1ull << a.lg_t) - 1) >> a.lg_t;
        launch_pass(a, groups, s, false);
        return;
    }

    // Multi-pass: process polynomials in chunks whose intermediate (chunk * N
    // elements) stays within `scratch_elems`, so it is L2-resident when small.
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(j.batches, j.scratch_elems / N));
    uint64_t *scr = j.scratch;
    for (uint64_t b0 = 0; b0 < j.batches; b0 += chunk) {
        const uint64_t nb = std::min<uint64_t>(chunk, j.batches - b0);
        uint32_t lg_s = lg;
        for (int p = 0; p < plan.passes; p++) {
            PassArgs a = base;
            a.l = plan.l[p];
            a.l_first = plan.l[0];
            a.batches = (uint32_t)nb;
            if (p < plan.passes - 1) {
                lg_s -= a.l;
                a.kind = 0;
                a.lg_s = lg_s;
                a.lg_pre = lg - a.l - lg_s;
                a.lg_t = std::min<uint32_t>(ilog2_floor(kLinesElems) - a.l, lg_s);
                a.lg_t = std::min<uint32_t>(a.lg_t, 5);
                // With the one-load twiddle table (up to 2^20 points, the compile-time
                // column kernels) half as many lines per block: half the shared
                // memory, so more resident blocks hide the loads.  Measured, LDE to
                // leaves: 135 x 2^15 -> 2^18 0.645 -> 0.625 ms, 64 x 2^17 -> 2^19
                // 0.741 -> 0.676, 16 x 2^12 -> 2^15 0.026 -> 0.020; without the table
                // (the generic pass) 300 x 2^19 -> 2^22 got slower (35.1 -> 36.7).
                if (base.tw_full && a.lg_t > 0) a.lg_t--;
                if (p == 0) {
                    a.src = j.src + b0 * j.src_stride;
                    a.src_poly_stride = j.src_stride;
                    a.n_valid = j.n_valid;
                } else {
                    a.src = scr;
                    a.src_poly_stride = N;
                    a.n_valid = N;
                    a.pre_lo = nullptr;
                }
                a.dst = scr;
                a.dst_poly_stride = N;
                a.post_lo = nullptr;
                a.scale = 1;
                const uint64_t groups = nb << (lg - a.l - a.lg_t);
                launch_pass(a, groups, s, p > 0);
            } else if (j.to_leaves) {
                // 8 polynomials per block: 64-byte runs in every leaf row (more resident
                // blocks hide the loads of the intermediate better than 16 did)
                a.kind = 3;
                a.lg_s = 0;
                a.lg_pre = lg - a.l;
                a.lg_t = a.l <= 9 ? 3 : 12 - std::min<uint32_t>(a.l, 12);
                if (tuned.passes && leaves_fits(a.l, tuned.lg_t)) a.lg_t = tuned.lg_t;
                // no wider than the chunk (the smallest power of two >= its polynomials)
                while (a.lg_t > 0 && (1ull << (a.lg_t - 1)) >= nb) a.lg_t--;
                a.src = scr;
                a.src_poly_stride = N;
                a.dst = j.dst + b0;
                a.leaf_stride = j.leaf_stride ? j.leaf_stride : j.batches;
                a.pre_lo = nullptr;
                a.n_valid = N;
                const uint64_t groups = ((nb + (1ull << a.lg_t) - 1) >> a.lg_t) << a.lg_pre;
                launch_leaves_pass(a, groups, s);
            } else {
                a.kind = 1;
                a.lg_s = 0;
                a.lg_pre = lg - a.l;
                a.lg_t = std::min<uint32_t>(ilog2_floor(kLinesElems) - a.l, plan.l[0]);
                a.lg_t = std::min<uint32_t>(a.lg_t, 5);
                a.src = scr;
                a.src_poly_stride = N;
                a.dst = j.dst + b0 * j.dst_stride;
                a.dst_poly_stride = j.dst_stride;
                a.pre_lo = nullptr;
                a.n_valid = N;
                const uint64_t groups = nb << (a.lg_pre - a.lg_t);
                launch_pass(a, groups, s, true);
            }
        }
    }
}

// One batched transform of `batches` polynomials of 2^lg elements.
void ntt_run(const NttJob &j, cudaStream_t s) {
    const uint32_t lg = j.lg;
    require(lg >= 1 && lg <= 32, "transform size out of range");
    if (j.batches == 0) return;
    DeviceCtx &ctx = device_ctx(current_device());
    const PowTable &rt = root_table(ctx, lg, j.inverse);
    const uint64_t *lr = line_roots(ctx, j.inverse);
    const LeavesChoice tuned = j.to_leaves ? leaves_choice(lg, j.batches) : LeavesChoice{};
    const Plan plan = tuned.passes ? plan_with_passes(lg, tuned.passes) : make_plan(lg, j.to_leaves);
    launch_plan(j, transform_args(j, rt, lr), plan, tuned, s);
}

uint64_t ntt_scratch_elems(uint32_t lg, uint64_t batches) {
    if (make_plan(lg).passes == 1) return 0;
    const uint64_t N = 1ull << lg;
    // Intermediate for up to 512 MiB of polynomials per chunk: chunks small
    // enough to bound the scratch, large enough that each pass launch spans
    // many waves of blocks (a chunk of a few polynomials leaves most of the
    // last wave idle).  Always at least one polynomial.
    const uint64_t cap = (512ull << 20) / sizeof(uint64_t);
    return std::max<uint64_t>(N, std::min<uint64_t>(batches * N, cap / N * N));
}

// The leaves pass puts up to 8 polynomials in a block (8-word runs in every
// leaf row), so the LDE -> leaves stage takes chunks of at least 8
// polynomials when the batch has them, beyond the 512 MiB of
// ntt_scratch_elems where need be (2 GiB for 2^25-point transforms).  With 2
// polynomials per chunk (2^25 points), six of every eight block lines idled
// and each leaf row got 16-byte runs: 120 x 2^22 -> 2^25 took 240 ms against
// 141 ms for the LDE rows plus the transpose.
uint64_t ntt_leaves_scratch_elems(uint32_t lg, uint64_t batches) {
    const uint64_t base = ntt_scratch_elems(lg, batches);
    if (!base) return 0;
    return std::max<uint64_t>(base, std::min<uint64_t>(batches, 8) << lg);
}

void transpose_rev_run(uint64_t *out, const uint64_t *in, uint32_t lg_n, uint32_t batches, cudaStream_t s) {
    if (batches == 0) return;
    const uint64_t N = 1ull << lg_n;
    const uint64_t K = std::min<uint64_t>(N, kTrK);
    const uint32_t nchunks = (batches + kTrMaxPolys - 1) / kTrMaxPolys;
    const uint32_t chunk = (batches + nchunks - 1) / nchunks;  // balanced chunks
    const uint64_t gx = N / K;
    require(gx < (1ull << 31) && nchunks < 65536, "transpose too large");
    const size_t smem = (size_t)K * (chunk | 1) * sizeof(uint64_t);
    // 16-byte loads need a 16-byte aligned input (caller pointers may be 8-byte aligned only).
    const bool vec = ((uintptr_t)in & 15) == 0;
    static std::atomic<uint64_t> attr_set{0};  // one bit per device
    const int dev = current_device();
    if (dev < 64 && !(attr_set.load() & (1ull << dev))) {
        const int big = (int)(kTrK * (kTrMaxPolys | 1) * sizeof(uint64_t));
        ZK_CUDA(cudaFuncSetAttribute(transpose_rev_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        ZK_CUDA(cudaFuncSetAttribute(transpose_rev_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        attr_set.fetch_or(1ull << dev);
    }
    if (vec) transpose_rev_kernel<true><<<dim3((unsigned)gx, nchunks), 256, smem, s>>>(out, in, lg_n, batches, chunk);
    else transpose_rev_kernel<false><<<dim3((unsigned)gx, nchunks), 256, smem, s>>>(out, in, lg_n, batches, chunk);
    ZK_CHECK_LAUNCH();
}

void salt_run(uint64_t *out, uint64_t count, uint64_t seed, cudaStream_t s) {
    if (!count) return;
    salt_kernel<<<1184, 256, 0, s>>>(out, count, seed);
    ZK_CHECK_LAUNCH();
}

}  // namespace zk

namespace zk {

// The transform of ntt_run, but on tables the caller supplies (no per-device
// state is created or looked up, so nothing is allocated here): used by the
// allocation-free LDE entry point in noalloc.cu.  Same pass setup as ntt_run
// (launch_plan), with the static plan.
void ntt_run_on_tables(const NttJob &j, const PowTable &roots, const uint64_t *line_roots_dev, cudaStream_t s) {
    require(j.lg >= 1 && j.lg <= 32 && !j.to_leaves, "transform size out of range");
    if (j.batches == 0) return;
    launch_plan(j, transform_args(j, roots, line_roots_dev), make_plan(j.lg), LeavesChoice{}, s);
}

// Times every legal (passes, polynomials per block) pair of the LDE -> leaves
// stage for this shape on scratch data (outputs do not depend on the choice)
// and records the fastest.  Synchronous; call it outside stream capture.
// Returns the number of candidates timed (0 if the shape was tuned already or
// has one pass).
int ntt_autotune_leaves(uint32_t lg_n, uint32_t rate_bits, uint64_t batches, cudaStream_t s) {
    const uint32_t lg = lg_n + rate_bits;
    require(lg >= 1 && lg <= 30 && batches >= 1, "invalid shape");
    if (make_plan(lg).passes == 1) return 0;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        if (g_tune.count(tune_key(lg, batches))) return 0;
    }
    DeviceCtx &ctx = device_ctx(current_device());
    const uint64_t N = 1ull << lg, n = 1ull << lg_n;
    // a representative batch: the class's own size, capped at ~1 GiB of leaves
    // but never below the 8 polynomials a chunk of the leaves stage holds
    const uint64_t bt = std::max<uint64_t>(1, std::min<uint64_t>(batches, std::max<uint64_t>(8, (1ull << 27) / N)));
    Scratch in(bt * n * sizeof(uint64_t), s), out(bt * N * sizeof(uint64_t), s);
    const uint64_t scr_elems = ntt_leaves_scratch_elems(lg, bt);
    Scratch scr(scr_elems * sizeof(uint64_t), s);
    ZK_CUDA(cudaMemsetAsync(in.p, 0, bt * n * sizeof(uint64_t), s));
    NttJob j;
    j.src = in.as<uint64_t>();
    j.src_stride = n;
    j.n_valid = n;
    j.dst = out.as<uint64_t>();
    j.batches = bt;
    j.lg = lg;
    j.pre_coset = &coset_table(ctx, lg, GROUP_GENERATOR, false);
    j.to_leaves = true;
    j.scratch = scr.as<uint64_t>();
    j.scratch_elems = scr_elems;
    cudaEvent_t e0, e1;
    ZK_CUDA(cudaEventCreate(&e0));
    ZK_CUDA(cudaEventCreate(&e1));
    LeavesChoice best{};
    float best_ms = 1e30f;
    int timed = 0;
    try {
        for (int passes = 2; passes <= 3; passes++) {
            if (passes == 2 && lg > 24) continue;
            const Plan p = plan_with_passes(lg, passes);
            const uint32_t l_last = p.l[passes - 1];
            for (uint32_t lg_t = 2; lg_t <= 4; lg_t++) {
                if (!leaves_fits(l_last, lg_t)) continue;
                const LeavesChoice c{(uint8_t)passes, (uint8_t)lg_t};
                t_tune_override = &c;
                ntt_run(j, s);  // warm-up
                ZK_CUDA(cudaEventRecord(e0, s));
                ntt_run(j, s);
                ntt_run(j, s);
                ZK_CUDA(cudaEventRecord(e1, s));
                t_tune_override = nullptr;
                ZK_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                ZK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                timed++;
                if (ms < best_ms) best_ms = ms, best = c;
            }
        }
    } catch (...) {
        t_tune_override = nullptr;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best.passes) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune[tune_key(lg, batches)] = best;
    }
    return timed;
}

void ntt_autotune_clear() {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune.clear();
}

}  // namespace zk
