// FRI commit-phase folding over the quadratic extension GF(p^2).
//
// The commitment's FRI prover (the consumer of zeknox's LDE and Merkle trees in
// the OKX Plonky2 fork, which calls the wrappers of native/lib.h:21-51) commits
// a polynomial P over GF(p^2) = GF(p)[X] / (X^2 - 7), given by its
// coefficients, in rounds.  Round i with arity a = 2^arity_bits:
//
//   1. evaluate P_i on the coset s_i * <w_(N_i)> (N_i = n_i * 2^rate_bits
//      points), reverse the order of the evaluations by bit reversal, and
//      commit rows of a consecutive evaluations (2a base elements each) as
//      the leaves of a Merkle tree;
//   2. draw the challenge beta_i from the tree's cap (Fiat-Shamir, done by the
//      caller);
//   3. fold: P_(i+1)(y) = sum_(t<a) beta_i^t Q_t(y), where P_i(x) =
//      sum_(t<a) x^t Q_t(x^a), i.e. coefficient j of P_(i+1) is
//      sum_(t<a) beta_i^t c_(j a + t);  s_(i+1) = s_i^a.
//
// Step 1 is the coset LDE written in the leaf layout (ntt.cu, to_leaves) on
// two polynomials (real and X parts of the coefficients), whose leaf rows are
// exactly the interleaved extension values in bit-reversed order; step 3 is
// the kernel below.  Coefficients live in the split layout: row 0 = real
// parts, row 1 = X parts, n elements each (the `batches = 2` layout of the
// LDE entry points).  The first fold may read interleaved pairs instead (the
// in-memory form of an array of GF(p^2) elements).
#include <stdint.h>

#include "fri.cuh"
#include "gl64.cuh"
#include "runtime.cuh"

namespace zk {

namespace {

struct FoldArgs {
    uint64_t p0[kFriMaxArity];  // real part of beta^t
    uint64_t p1[kFriMaxArity];  // X part of beta^t
    uint64_t q1[kFriMaxArity];  // 7 * (X part of beta^t)
};

// out[j] = sum_(t<a) beta^t * in[j a + t] in GF(p^2), for j < n_out.  The a
// products of one output are independent (the powers of beta come from the
// host), so a thread has 4a field products in flight instead of a Horner chain.
template <bool kInterleaved>
__global__ void __launch_bounds__(256) fri_fold_kernel(uint64_t *__restrict__ out, const uint64_t *__restrict__ in,
                                                       uint64_t in_stride, uint64_t n_out, uint64_t out_stride,
                                                       uint32_t lg_a, FoldArgs args) {
    const uint32_t a = 1u << lg_a;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n_out; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r0 = 0, r1 = 0;
        const uint64_t base = j << lg_a;
#pragma unroll 4
        for (uint32_t t = 0; t < a; t++) {
            uint64_t c0, c1;
            if (kInterleaved) {
                const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2 *>(in) + base + t);
                c0 = v.x;
                c1 = v.y;
            } else {
                c0 = __ldg(in + base + t);
                c1 = __ldg(in + in_stride + base + t);
            }
            // (c0 + c1 X)(p0 + p1 X) = c0 p0 + 7 c1 p1 + (c0 p1 + c1 p0) X
            r0 = gl_add(r0, gl_add(gl_mul(c0, args.p0[t]), gl_mul(c1, args.q1[t])));
            r1 = gl_add(r1, gl_add(gl_mul(c0, args.p1[t]), gl_mul(c1, args.p0[t])));
        }
        out[j] = r0;
        out[out_stride + j] = r1;
    }
}

// Host GF(p^2) product, W = 7.
void ext_mul_host(uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1, uint64_t &c0, uint64_t &c1) {
    const uint64_t x = h_mul(a0, b0), y = h_mul(h_mul(a1, b1), 7);
    c0 = (uint64_t)(((unsigned __int128)x + y) % P_HOST);
    c1 = (uint64_t)(((unsigned __int128)h_mul(a0, b1) + h_mul(a1, b0)) % P_HOST);
}

}  // namespace

void fri_fold_run(uint64_t *out, const uint64_t *in, uint64_t n_in, uint32_t arity_bits, uint64_t beta0,
                  uint64_t beta1, bool in_interleaved, cudaStream_t s) {
    require(arity_bits >= 1 && (1u << arity_bits) <= kFriMaxArity, "FRI arity_bits must be in 1..6");
    require(n_in >= (1ull << arity_bits) && (n_in & (n_in - 1)) == 0, "FRI fold: n_in must be a power of two >= arity");
    require(beta0 < P_HOST && beta1 < P_HOST, "FRI fold: beta must be canonical");
    require(out != in, "FRI fold cannot run in place");
    require(!in_interleaved || ((uintptr_t)in & 15) == 0, "FRI fold: interleaved input must be 16-byte aligned");
    FoldArgs args{};
    uint64_t w0 = 1, w1 = 0;  // beta^t
    for (uint32_t t = 0; t < (1u << arity_bits); t++) {
        args.p0[t] = w0;
        args.p1[t] = w1;
        args.q1[t] = h_mul(w1, 7);
        ext_mul_host(w0, w1, beta0, beta1, w0, w1);
    }
    const uint64_t n_out = n_in >> arity_bits;
    const uint64_t blocks = std::min<uint64_t>((n_out + 255) / 256, 148ull * 16);
    if (in_interleaved)
        fri_fold_kernel<true><<<(unsigned)blocks, 256, 0, s>>>(out, in, 0, n_out, n_out, arity_bits, args);
    else
        fri_fold_kernel<false><<<(unsigned)blocks, 256, 0, s>>>(out, in, n_in, n_out, n_out, arity_bits, args);
    ZK_CHECK_LAUNCH();
}

}  // namespace zk
