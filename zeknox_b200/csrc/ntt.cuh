// Host interface of the NTT engine (ntt.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "runtime.cuh"

namespace zk {

// One batched transform X[k] = sum_i x[i] w^(ik) over `batches` polynomials of
// N = 2^lg elements, w = omega_N (forward) or omega_N^-1 (inverse), natural
// order in and out.  Element i of polynomial b is read from
// src[b * src_stride + i] when i < n_valid (0 otherwise: zero-extension), and
// optionally multiplied by pre_coset^i first; the output element k goes to
// dst[b * dst_stride + k], optionally multiplied by post_coset^k and by `scale`.
// src may equal dst.  `scratch` holds scratch_elems >= ntt_scratch_elems(..)
// elements when the transform needs more than one pass.
struct NttJob {
    const uint64_t *src = nullptr;
    uint64_t *dst = nullptr;
    uint64_t src_stride = 0, dst_stride = 0;
    uint64_t batches = 0;
    uint32_t lg = 0;
    bool inverse = false;
    uint64_t n_valid = 0;
    const PowTable *pre_coset = nullptr;
    const PowTable *post_coset = nullptr;
    uint64_t scale = 1;
    uint64_t *scratch = nullptr;
    uint64_t scratch_elems = 0;
    // Write the leaf layout instead: element k of polynomial b goes to
    // dst[rev_lg(k) * batches + b] (forward transforms without post_coset/scale).
    bool to_leaves = false;
    // Words per leaf row when the polynomials are a column slice of a wider
    // leaf matrix (dst then points at the slice's first column); 0 = batches.
    uint64_t leaf_stride = 0;
};

void ntt_run(const NttJob &job, cudaStream_t s);
uint64_t ntt_scratch_elems(uint32_t lg, uint64_t batches);
// Scratch of the LDE -> leaves stage (to_leaves): chunks of at least 8 polynomials.
uint64_t ntt_leaves_scratch_elems(uint32_t lg, uint64_t batches);
void transpose_rev_run(uint64_t *out, const uint64_t *in, uint32_t lg_n, uint32_t batches, cudaStream_t s);
void salt_run(uint64_t *out, uint64_t count, uint64_t seed, cudaStream_t s);
// Autotuning of the LDE -> leaves stage per (size, batch-size class); see ntt.cu.
int ntt_autotune_leaves(uint32_t lg_n, uint32_t rate_bits, uint64_t batches, cudaStream_t s);
void ntt_autotune_clear();

}  // namespace zk

namespace zk {
// ntt_run on caller-supplied tables (roots: powers of omega_N for this
// direction, two-level; line_roots: omega_4096^j, j < 4096, this direction).
// Creates no per-device state and allocates nothing.
void ntt_run_on_tables(const NttJob &job, const PowTable &roots, const uint64_t *line_roots, cudaStream_t s);
}  // namespace zk
