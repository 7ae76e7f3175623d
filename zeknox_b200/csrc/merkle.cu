// Merkle forest construction in zeknox's linear digest layout
// (native/merkle/merkle.cu:166-244).
//
// zeknox launches one kernel for the leaves, one per tree level and one for
// the cap (merkle.cu:215-243).  Here `merkle_tile` gives each block a tile of
// 128 consecutive leaves of one subtree: every thread runs its leaf's sponge
// with the state in registers, then the block folds the tile's 7 lowest
// levels through shared memory, writing every digest on the way.  The levels
// above the tiles (fewer than 2^cap_height * L/128 nodes) are finished by
// `merkle_top`, one block per subtree, which also writes the cap.  The
// special shapes (cap == leaves, 1 or 2 leaves per subtree, Keccak leaves
// shorter than a digest) use the one-thread-per-hash kernels
// `merkle_leaves` / `merkle_caps`.
#include <stdint.h>

#include <algorithm>

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

constexpr int kTile = 128;

// Level of width w (nodes per subtree) starts at offset w - 2 of the subtree's
// digest block; width 1 is the subtree root, which is the cap entry.
__device__ __forceinline__ uint64_t *node_ptr(uint64_t *sub, uint64_t w, uint64_t i) { return sub + 4 * (w - 2 + i); }

// Block = tile of blockDim.x (<= 128, a power of two) consecutive leaves of one
// subtree.  Hashes the leaves, then folds log2(blockDim.x) levels.  For the
// Poseidon hashers a node is the sponge of its two children's 8 words (the
// same state as hash_two), so leaves and nodes go through one call site of
// the permutation: one copy of its code in the kernel, which keeps the
// instruction working set of the resident warps small.
template <int H>
__global__ void __launch_bounds__(kTile) merkle_tile(const uint64_t *__restrict__ leaves, uint32_t leaf_size,
                                                     uint64_t *__restrict__ digests, uint64_t *__restrict__ cap,
                                                     uint64_t ls, uint64_t ds) {
    __shared__ uint64_t sm[kTile * 4];
    const uint32_t t = threadIdx.x, T = blockDim.x;
    const uint64_t leaf = blockIdx.x * (uint64_t)T + t;
    const uint64_t sub = leaf / ls, j0 = (blockIdx.x * (uint64_t)T) % ls;
    uint64_t *base = digests + 4 * sub * ds;
    if constexpr (H == kKeccak) {
        uint64_t d[4];
        hash_one<H>(leaves + leaf * leaf_size, leaf_size, d);
        uint64_t *dst = base + 4 * (ds - ls + j0 + t);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            dst[k] = d[k];
            sm[4 * t + k] = d[k];
        }
        uint64_t w = ls;
        for (uint32_t active = T >> 1; active >= 1; active >>= 1) {
            w >>= 1;
            __syncthreads();
            uint64_t h[4];
            if (t < active) hash_two<H>(&sm[8 * t], &sm[8 * t + 4], h);
            __syncthreads();
            if (t < active) {
                const uint64_t i = (j0 >> (__ffs(T / active) - 1)) + t;  // index in the level of width w
                uint64_t *o = w >= 2 ? node_ptr(base, w, i) : cap + 4 * sub;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    o[k] = h[k];
                    sm[4 * t + k] = h[k];
                }
            }
        }
    } else {
        const uint64_t *src = leaves + leaf * leaf_size;
        uint32_t n = leaf_size, active = T, lvl = 0;
        for (;;) {
            uint64_t h[4];
            if (t < active) hash_one<H>(src, n, h);
            if (lvl) __syncthreads();  // every child in sm has been read
            if (t < active) {
                const uint64_t w = ls >> lvl;  // width of this level
                uint64_t *o = lvl == 0 ? base + 4 * (ds - ls + j0 + t)
                                       : (w >= 2 ? node_ptr(base, w, (j0 >> lvl) + t) : cap + 4 * sub);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    o[k] = h[k];
                    sm[4 * t + k] = h[k];
                }
            }
            active >>= 1;
            if (!active) break;
            __syncthreads();
            src = &sm[8 * t];
            n = 8;
            lvl++;
        }
    }
}

// One block per subtree: the levels above the tiles, from width w0 down to the
// root (written to cap[sub]).
template <int H>
__global__ void __launch_bounds__(256) merkle_top(uint64_t *__restrict__ digests, uint64_t *__restrict__ cap,
                                                  uint64_t ds, uint64_t w0) {
    const uint64_t sub = blockIdx.x;
    uint64_t *base = digests + 4 * sub * ds;
    for (uint64_t w = w0; w > 1; w >>= 1) {
        const uint64_t wn = w >> 1;
        for (uint64_t i = threadIdx.x; i < wn; i += blockDim.x) {
            uint64_t h[4];
            hash_two<H>(node_ptr(base, w, 2 * i), node_ptr(base, w, 2 * i + 1), h);
            uint64_t *o = wn >= 2 ? node_ptr(base, wn, i) : cap + 4 * sub;
#pragma unroll
            for (int k = 0; k < 4; k++) o[k] = h[k];
        }
        __syncthreads();
    }
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
    if (ls == 2 || (H == kKeccak && w < 4)) {
        // zeknox's one-thread-per-hash structure (merkle.cu:193-243); Keccak
        // leaves shorter than a digest keep the words they do not write.
        LeafMap map;
        map.direct = (ls == 2);
        map.ls = ls;
        map.ds = ds;
        merkle_leaves<H><<<blocks_for(j.n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(j.leaves, j.n_leaves, w,
                                                                                         j.digests, map);
        ZK_CHECK_LAUNCH();
        for (uint64_t lw = ls / 2; lw >= 2; lw /= 2) {
            merkle_level<H><<<blocks_for(lw * j.n_caps, kLeafThreads), kLeafThreads, 0, st>>>(j.digests, lw, j.n_caps,
                                                                                              ds);
            ZK_CHECK_LAUNCH();
        }
        merkle_caps<H><<<blocks_for(j.n_caps, 64), 64, 0, st>>>(j.cap, j.digests, j.n_caps, ds);
        ZK_CHECK_LAUNCH();
        return;
    }
    const uint32_t T = (uint32_t)std::min<uint64_t>(kTile, ls);
    merkle_tile<H><<<blocks_for(j.n_leaves, T), T, 0, st>>>(j.leaves, w, j.digests, j.cap, ls, ds);
    ZK_CHECK_LAUNCH();
    if (ls > (uint64_t)kTile) {
        require(j.n_caps < (1ull << 31), "too many subtrees");
        merkle_top<H><<<(unsigned)j.n_caps, 256, 0, st>>>(j.digests, j.cap, ds, ls / kTile);
        ZK_CHECK_LAUNCH();
    }
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
