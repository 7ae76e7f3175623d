// Host interface of the FRI folding kernel (fri.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace zk {

constexpr uint32_t kFriMaxArity = 64;  // arity_bits <= 6

// out (split layout, 2 rows of n_in >> arity_bits) = the fold of in (split
// layout, 2 rows of n_in; or n_in interleaved GF(p^2) pairs) by beta.
void fri_fold_run(uint64_t *out, const uint64_t *in, uint64_t n_in, uint32_t arity_bits, uint64_t beta0,
                  uint64_t beta1, bool in_interleaved, cudaStream_t s);

}  // namespace zk
