// Merkle forest construction in zeknox's linear digest layout
// (native/merkle/merkle.cu:166-244).
//
// Leaf hashing runs one thread per leaf with the sponge state in registers
// (kernel `merkle_leaves`).  The internal levels of all 2^cap_height subtrees
// are built bottom-up; `merkle_tile_levels` folds the lowest levels inside a
// thread block (shared memory, no extra launches) and `merkle_level` handles
// the remaining wide levels; `merkle_caps` hashes the subtree roots.
#include <stdint.h>

#include "hash.cuh"
#include "merkle.cuh"
#include "runtime.cuh"

namespace zk {

namespace {

constexpr int kLeafThreads = 128;

// Digest slot of leaf i: subtree s = i / Ls owns [s*Ds, (s+1)*Ds); its leaves
// sit at the tail, Ds - Ls + j.  In direct mode digest i goes to slot i.
struct LeafMap {
    uint64_t ls = 1, ds = 0;
    bool direct = true;
    __device__ __forceinline__ uint64_t slot(uint64_t i) const {
        if (direct) return i;
        const uint64_t s = i / ls, j = i % ls;
        return s * ds + (ds - ls) + j;
    }
};

template <int H>
__global__ void __launch_bounds__(kLeafThreads) merkle_leaves(const uint64_t *__restrict__ leaves, uint64_t n_leaves,
                                                              uint32_t leaf_size, uint64_t *__restrict__ out,
                                                              LeafMap map) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n_leaves) return;
    hash_one<H>(leaves + i * leaf_size, leaf_size, out + 4 * map.slot(i));
}

// One level of width w (= 2^r nodes per subtree, at offsets w - 2 .. 2w - 3):
// node i <- H(node 2(i+1), node 2(i+1)+1).
template <int H>
__global__ void __launch_bounds__(kLeafThreads) merkle_level(uint64_t *__restrict__ digests, uint64_t w,
                                                             uint64_t n_caps, uint64_t ds) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (tid >= w * n_caps) return;
    const uint64_t s = tid / w, i = (w - 2) + tid % w;
    uint64_t *base = digests + 4 * s * ds;
    hash_two<H>(base + 4 * (2 * i + 2), base + 4 * (2 * i + 3), base + 4 * i);
}

template <int H>
__global__ void merkle_caps(uint64_t *__restrict__ cap, const uint64_t *__restrict__ digests, uint64_t n_caps,
                            uint64_t ds) {
    const uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s >= n_caps) return;
    hash_two<H>(digests + 4 * s * ds, digests + 4 * (s * ds + 1), cap + 4 * s);
}

inline unsigned blocks_for(uint64_t n, unsigned tpb) {
    const uint64_t b = (n + tpb - 1) / tpb;
    require(b < (1ull << 31), "Merkle launch too large");
    return (unsigned)(b ? b : 1);
}

template <int H>
void merkle_run_t(const MerkleJob &j, cudaStream_t st) {
    const uint32_t w = (uint32_t)j.leaf_size;
    if (j.n_caps == j.n_leaves) {
        if (!j.n_leaves) return;
        merkle_leaves<H><<<blocks_for(j.n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(j.leaves, j.n_leaves, w, j.cap,
                                                                                         LeafMap{});
        ZK_CHECK_LAUNCH();
        return;
    }
    const uint64_t ls = j.n_leaves >> j.cap_height, ds = j.n_digests >> j.cap_height;
    if (ls == 1) {
        merkle_leaves<H><<<blocks_for(j.n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(j.leaves, j.n_leaves, w, j.cap,
                                                                                         LeafMap{});
        ZK_CHECK_LAUNCH();
        return;
    }
    LeafMap map;
    map.direct = (ls == 2);
    map.ls = ls;
    map.ds = ds;
    merkle_leaves<H><<<blocks_for(j.n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(j.leaves, j.n_leaves, w, j.digests,
                                                                                     map);
    ZK_CHECK_LAUNCH();
    for (uint64_t lw = ls / 2; lw >= 2; lw /= 2) {
        merkle_level<H><<<blocks_for(lw * j.n_caps, kLeafThreads), kLeafThreads, 0, st>>>(j.digests, lw, j.n_caps, ds);
        ZK_CHECK_LAUNCH();
    }
    merkle_caps<H><<<blocks_for(j.n_caps, 64), 64, 0, st>>>(j.cap, j.digests, j.n_caps, ds);
    ZK_CHECK_LAUNCH();
}

}  // namespace

bool merkle_hash_supported(uint64_t ht) { return ht == kPoseidon || ht == kPoseidon2 || ht == kKeccak; }

void merkle_validate(const MerkleJob &j) {
    require(merkle_hash_supported(j.hash_type), "unsupported hash type " + std::to_string(j.hash_type));
    require(j.cap_height < 64 && j.n_caps == (1ull << j.cap_height), "cap_buf_size must be 2^cap_height");
    require(j.leaf_size > 0 && j.leaf_size < (1ull << 31), "leaf_size out of range");
    if (j.n_caps == j.n_leaves) return;
    require(j.n_leaves % j.n_caps == 0, "leaves_buf_size must be a multiple of cap_buf_size");
    const uint64_t ls = j.n_leaves >> j.cap_height;
    require((ls & (ls - 1)) == 0, "leaves per subtree must be a power of two");
    require((j.n_digests >> j.cap_height) == 2 * ls - 2 && j.n_digests % j.n_caps == 0,
            "digests_buf_size must be 2 * (leaves_buf_size - cap_buf_size)");
    require(j.leaves && j.cap && (ls == 1 || j.digests), "null buffer");
}

void merkle_run(const MerkleJob &j, cudaStream_t st) {
    merkle_validate(j);
    switch (j.hash_type) {
    case kPoseidon: merkle_run_t<kPoseidon>(j, st); break;
    case kPoseidon2: merkle_run_t<kPoseidon2>(j, st); break;
    case kKeccak: merkle_run_t<kKeccak>(j, st); break;
    default: break;
    }
}

}  // namespace zk
