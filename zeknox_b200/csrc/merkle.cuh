// Host interface of the Merkle builder (merkle.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace zk {

// Sizes as in zeknox's fill_digests_buf_linear_* (native/merkle/merkle.h:30-62):
// counts of 4-element digests and of leaves; all pointers on the device.
struct MerkleJob {
    uint64_t *digests = nullptr;
    uint64_t *cap = nullptr;
    const uint64_t *leaves = nullptr;
    uint64_t n_digests = 0, n_caps = 0, n_leaves = 0, leaf_size = 0, cap_height = 0, hash_type = 0;
};

bool merkle_hash_supported(uint64_t hash_type);
void merkle_validate(const MerkleJob &job);  // throws zk::Error
void merkle_run(const MerkleJob &job, cudaStream_t s);
// Threads-per-hash autotuner for Poseidon leaves: times the six-, two- and
// one-thread leaf kernels on a zero tree of this shape (n_leaves <= 2^16,
// leaf_size > 4; other shapes and hashers return 0) and keeps the fastest for
// its class (log2 of the leaf count, permutations per leaf).  Returns the
// number of candidates timed (0: already tuned or not tunable).  Outputs do
// not depend on the choice.
int merkle_autotune_leaves(uint64_t n_leaves, uint64_t leaf_size, uint64_t hash_type, cudaStream_t s);
void merkle_autotune_clear();
// Leaf rows and sibling paths of n_queries leaves (all pointers on the device).
void merkle_open(const uint64_t *leaves, const uint64_t *digests, uint64_t n_leaves, uint64_t leaf_size,
                 uint64_t cap_height, const uint64_t *idx, uint64_t n_queries, uint64_t *out_leaves,
                 uint64_t *out_siblings, cudaStream_t s);

}  // namespace zk
