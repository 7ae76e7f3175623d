// Merkle forest construction in zeknox's linear digest layout
// (native/merkle/merkle.cu:166-244).
//
// One launch hashes every leaf (one thread per leaf, sponge state in
// registers), then one launch per tree level hashes that level's nodes across
// all subtrees, and a last one the narrow top and the cap: the structure of
// zeknox's kernels (merkle.cu:215-243).  For Poseidon and Poseidon2, the
// latency-bound parts (small trees, narrow levels, the top) spread each
// permutation over six threads (Poseidon also over two) instead (hash.cuh),
// with thresholds set by measurement.
// Fusing the lower levels into the leaf kernel (a block folding its tile of
// leaves through shared memory) measured slower on B200: a block then holds
// its registers through the serial, mostly idle fold levels, which costs more
// than re-reading the children from L2.
#include <stdint.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "hash.cuh"
#include "merkle.cuh"
#include "pdl.cuh"
#include "runtime.cuh"

namespace zk {

namespace {

constexpr int kLeafThreads = 128;

// The level and top kernels are launched with launch_after (pdl.cuh): each
// loads its round tables, waits for the previous level, and releases its
// dependents once its block has stored its nodes.

// Digest slot of leaf i: subtree s = i / Ls owns [s*Ds, (s+1)*Ds); its leaves
// sit at the tail, Ds - Ls + j.  In direct mode digest i goes to slot i.
struct LeafMap {
    uint32_t lg_ls = 0;  // Ls = 2^lg_ls
    uint64_t ds = 0;
    bool direct = true;
    __device__ __forceinline__ uint64_t slot(uint64_t i) const {
        if (direct) return i;
        const uint64_t ls = 1ull << lg_ls;
        return (i >> lg_ls) * ds + (ds - ls) + (i & (ls - 1));
    }
};

template <int H>
__global__ void __launch_bounds__(kLeafThreads) merkle_leaves(const uint64_t *__restrict__ leaves, uint64_t n_leaves,
                                                              uint32_t leaf_size, uint64_t *__restrict__ out,
                                                              LeafMap map) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n_leaves) return;
    // S-box width: all 12 lanes at once measured faster for Poseidon; for
    // Poseidon2 the larger loop body costs more in instruction fetch.
    hash_one<H, H == kPoseidon ? 12 : 4>(leaves + i * leaf_size, leaf_size, out + 4 * map.slot(i));
    pdl_release();
}

// One level of width w = 2^lg_w nodes per subtree (at offsets w - 2 .. 2w - 3
// of each subtree's block): node i <- H(node 2(i+1), node 2(i+1)+1).
template <int H, int W>
__global__ void __launch_bounds__(kLeafThreads) merkle_level(uint64_t *__restrict__ digests, uint32_t lg_w,
                                                             uint64_t n_caps, uint64_t ds) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t w = 1ull << lg_w;
    if (tid >= (n_caps << lg_w)) return;
    const uint64_t s = tid >> lg_w, i = (w - 2) + (tid & (w - 1));
    uint64_t *base = digests + 4 * s * ds;
    pdl_wait();
    hash_two<H, W>(base + 4 * (2 * i + 2), base + 4 * (2 * i + 3), base + 4 * i);
    pdl_release();
}

// One block per subtree: the levels of width w_top, w_top/2, ..., 1 (the cap),
// one node per thread, __syncthreads between levels.  These levels are few
// nodes each, so every one costs about one permutation's latency: the block
// copies its hasher's round tables into shared memory first and uses the
// 12-lanes-at-once S-box.
template <int H>
__global__ void __launch_bounds__(256) merkle_top(uint64_t *__restrict__ digests, uint64_t *__restrict__ cap,
                                                   uint64_t ds, uint32_t w_top) {
    using Tab = typename TabOf<H>::type;
    __shared__ __align__(16) unsigned char tab_raw[sizeof(Tab)];
    Tab &tab = *reinterpret_cast<Tab *>(tab_raw);
    if constexpr (sizeof(Tab) >= 8) {
        const uint64_t *g = reinterpret_cast<const uint64_t *>(global_tab<H>());
        uint64_t *d = reinterpret_cast<uint64_t *>(tab_raw);
        for (uint32_t k = threadIdx.x; k < sizeof(Tab) / 8; k += blockDim.x) d[k] = g[k];
    }
    __syncthreads();
    const uint64_t sub = blockIdx.x;
    uint64_t *base = digests + 4 * sub * ds;
    pdl_wait();
    for (uint32_t w = w_top; w >= 1; w >>= 1) {
        const uint32_t i = threadIdx.x;
        if (i < w) {
            const uint64_t *c = base + 4 * (2 * w - 2 + 2 * i);  // children 2i, 2i+1 of the level of width 2w
            uint64_t *o = w >= 2 ? base + 4 * (w - 2 + i) : cap + 4 * sub;
            if constexpr (sizeof(Tab) >= 8) hash_two<H, 12>(c, c + 4, o, tab);
            else hash_two<H, 12>(c, c + 4, o);
        }
        __syncthreads();
    }
}

// Copies a hasher's round tables into shared memory (all threads of the block).
template <int H>
__device__ __forceinline__ void load_tab(typename TabOf<H>::type &dst) {
    const uint64_t *g = reinterpret_cast<const uint64_t *>(global_tab<H>());
    uint64_t *d = reinterpret_cast<uint64_t *>(&dst);
    for (uint32_t k = threadIdx.x; k < sizeof(dst) / 8; k += blockDim.x) d[k] = g[k];
    __syncthreads();
}

// Poseidon on two threads per hash (a lane pair): sixteen hashes per warp.
constexpr int kDuoThreads = 128;

__global__ void __launch_bounds__(kDuoThreads) merkle_leaves_duo(const uint64_t *__restrict__ leaves,
                                                                 uint64_t n_leaves, uint32_t leaf_size,
                                                                 uint64_t *__restrict__ out, LeafMap map) {
    __shared__ PoseidonTab tab;  // per-thread table indices: shared memory, not the constant bank
    load_tab<kPoseidon>(tab);
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t first = (t >> 5) << 4;  // the warp's first hash
    if (first >= n_leaves) return;         // whole warp
    const uint32_t h = threadIdx.x & 1;
    const uint64_t i = t >> 1;
    const bool active = i < n_leaves;
    const uint64_t ii = active ? i : 0;
    poseidon_hash_one_duo(leaves + ii * leaf_size, leaf_size, out + 4 * map.slot(ii), active, h, tab);
    pdl_release();
}

// Poseidon and Poseidon2 on six threads per hash (HexGroup, HexGroup2): five
// hashes per warp.  For the latency-bound cases: few leaves, narrow levels,
// the top of the tree.
constexpr int kHexThreads = 128;  // 4 warps = 20 hashes per block
constexpr uint64_t kHexPerBlock = 20;

template <int H>
__global__ void __launch_bounds__(kHexThreads) merkle_leaves_hex(const uint64_t *__restrict__ leaves,
                                                                 uint64_t n_leaves, uint32_t leaf_size,
                                                                 uint64_t *__restrict__ out, LeafMap map) {
    __shared__ typename TabOf<H>::type tab;
    load_tab<H>(tab);
    const HexOf<H> g(tab);
    const uint64_t first = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * 5;
    if (first >= n_leaves) return;  // whole warp
    const uint64_t i = first + g.group_in_warp();
    const bool active = g.real() && i < n_leaves;
    const uint64_t ii = active ? i : 0;
    hash_one_hex(leaves + ii * leaf_size, leaf_size, out + 4 * map.slot(ii), active, g, tab);
    pdl_release();
}

template <int H>
__global__ void __launch_bounds__(kHexThreads) merkle_level_hex(uint64_t *__restrict__ digests, uint32_t lg_w,
                                                                uint64_t n_caps, uint64_t ds) {
    __shared__ typename TabOf<H>::type tab;
    load_tab<H>(tab);
    const HexOf<H> g(tab);
    const uint64_t w = 1ull << lg_w;
    const uint64_t first = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * 5;
    if (first >= (n_caps << lg_w)) return;  // whole warp
    const uint64_t tid = first + g.group_in_warp();
    const bool active = g.real() && tid < (n_caps << lg_w);
    const uint64_t tt = active ? tid : 0;
    const uint64_t sub = tt >> lg_w, i = (w - 2) + (tt & (w - 1));
    uint64_t *base = digests + 4 * sub * ds;
    pdl_wait();
    hash_two_hex(base + 4 * (2 * i + 2), base + 4 * (2 * i + 3), base + 4 * i, active, g, tab);
    pdl_release();
}

// One block per subtree: levels of width w_top (<= 32) .. 1, then the cap.
template <int H>
__global__ void __launch_bounds__(224) merkle_top_hex(uint64_t *__restrict__ digests, uint64_t *__restrict__ cap,
                                                       uint64_t ds, uint32_t w_top) {
    __shared__ typename TabOf<H>::type tab;
    load_tab<H>(tab);
    const HexOf<H> g(tab);
    const uint64_t sub = blockIdx.x;
    uint64_t *base = digests + 4 * sub * ds;
    const uint32_t node = (threadIdx.x >> 5) * 5 + g.group_in_warp();
    pdl_wait();
    for (uint32_t w = w_top; w >= 1; w >>= 1) {
        if ((threadIdx.x >> 5) * 5 < w) {  // warps with at least one node of this level
            const bool active = g.real() && node < w;
            const uint32_t i = active ? node : 0;
            const uint64_t *c = base + 4 * (2 * w - 2 + 2 * i);  // children 2i, 2i+1 of the level of width 2w
            uint64_t *o = w >= 2 ? base + 4 * (w - 2 + i) : cap + 4 * sub;
            hash_two_hex(c, c + 4, o, active, g, tab);
        }
        __syncthreads();
    }
}

inline unsigned hex_blocks(uint64_t hashes) {
    const uint64_t b = (hashes + kHexPerBlock - 1) / kHexPerBlock;
    require(b < (1ull << 31), "Merkle launch too large");
    return (unsigned)(b ? b : 1);
}

inline unsigned blocks_for(uint64_t n, unsigned tpb) {
    const uint64_t b = (n + tpb - 1) / tpb;
    require(b < (1ull << 31), "Merkle launch too large");
    return (unsigned)(b ? b : 1);
}


// Threads per Poseidon hash for a tree's leaves: 6 (HexGroup), 2 (lane
// pairs) or 1.  Static thresholds, measured on trees of 135-word leaves:
// whole trees, six- vs one-threaded leaves, 8192 leaves 0.48 vs 0.65 ms,
// 16384 leaves 0.80 vs 0.68 ms, 32768 leaves 1.43 vs 0.87 ms; two threads per
// hash win between the two, 16384 leaves 0.59 ms (4096: 0.47, 8192: 0.49,
// 32768: 0.97, 65536: 1.54 vs 1.46 one-threaded).  merkle_autotune_leaves
// replaces them by measurement per (tree size, permutations per leaf).
constexpr uint64_t kHexLeaves = 1 << 13, kDuoLeaves = 1 << 14;
constexpr uint64_t kLayoutTuneMax = 1 << 16;  // larger trees: one thread per hash, by a wide margin
std::mutex g_layout_mu;
std::map<uint64_t, uint8_t> g_layout;  // layout_key -> threads per hash

uint64_t layout_key(uint64_t n_leaves, uint64_t leaf_size) {
    const uint64_t lg = 63 - __builtin_clzll(n_leaves);
    return (lg << 32) | ((leaf_size + 7) / 8);  // permutations per leaf
}
uint8_t leaf_layout(uint64_t n_leaves, uint64_t leaf_size) {
    if (n_leaves <= kLayoutTuneMax && leaf_size > 4) {
        std::lock_guard<std::mutex> g(g_layout_mu);
        auto it = g_layout.find(layout_key(n_leaves, leaf_size));
        if (it != g_layout.end()) return it->second;
    }
    return n_leaves <= kHexLeaves ? 6 : n_leaves <= kDuoLeaves ? 2 : 1;
}
void launch_poseidon_leaves(const uint64_t *leaves, uint64_t n_leaves, uint32_t w, uint64_t *out, LeafMap map,
                            uint8_t layout, cudaStream_t st) {
    if (layout == 6)
        merkle_leaves_hex<kPoseidon><<<hex_blocks(n_leaves), kHexThreads, 0, st>>>(leaves, n_leaves, w, out, map);
    else if (layout == 2)
        merkle_leaves_duo<<<blocks_for(2 * n_leaves, kDuoThreads), kDuoThreads, 0, st>>>(leaves, n_leaves, w, out, map);
    else
        merkle_leaves<kPoseidon><<<blocks_for(n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(leaves, n_leaves, w, out,
                                                                                              map);
    ZK_CHECK_LAUNCH();
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
    // Leaves into their digest slots (Keccak leaves shorter than a digest
    // keep the words they do not write, as in zeknox), then the levels.
    LeafMap map;
    map.direct = (ls == 2);
    map.lg_ls = (uint32_t)__builtin_ctzll(ls);
    map.ds = ds;
    if constexpr (H == kPoseidon || H == kPoseidon2) {
        // Latency-bound parts on several threads per hash: the leaves of
        // small trees (leaf_layout for Poseidon; Poseidon2 has the six-thread
        // form only, up to kHexLeaves), levels of fewer than kHexNodes nodes,
        // and the top (<= 32 nodes per subtree, so that one SM per subtree
        // stays latency- rather than issue-bound) in one launch.  Measured
        // per Poseidon level: 16384 nodes 46 us six-threaded vs 40 us
        // one-threaded (issue bound: six threads do twice the instructions of
        // one); 4096 nodes 20 us vs 40 us.
        constexpr uint64_t kHexNodes = 1 << 14;
        if constexpr (H == kPoseidon) {
            launch_poseidon_leaves(j.leaves, j.n_leaves, w, j.digests, map, leaf_layout(j.n_leaves, w), st);
        } else {
            if (j.n_leaves <= kHexLeaves)
                merkle_leaves_hex<H><<<hex_blocks(j.n_leaves), kHexThreads, 0, st>>>(j.leaves, j.n_leaves, w,
                                                                                     j.digests, map);
            else
                merkle_leaves<H><<<blocks_for(j.n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(j.leaves, j.n_leaves,
                                                                                                 w, j.digests, map);
            ZK_CHECK_LAUNCH();
        }
        uint32_t lg_top = 0;
        while (lg_top + 1 < map.lg_ls && lg_top < 5 && (j.n_caps << (lg_top + 1)) < kHexNodes) lg_top++;
        // Wide levels: the 12-lane S-box for Poseidon (measured 15 us faster
        // per tree of 2^18), the 4-lane one for Poseidon2 (as in its leaves).
        constexpr int kWideW = H == kPoseidon ? 12 : 4;
        for (uint32_t lg_w = map.lg_ls - 1; lg_w > lg_top; lg_w--) {
            const uint64_t nodes = j.n_caps << lg_w;
            if (nodes >= kHexNodes)
                launch_after(merkle_level<H, kWideW>, blocks_for(nodes, kLeafThreads), kLeafThreads, 0, st, j.digests,
                             lg_w, j.n_caps, ds);
            else
                launch_after(merkle_level_hex<H>, hex_blocks(nodes), kHexThreads, 0, st, j.digests, lg_w, j.n_caps,
                             ds);
        }
        require(j.n_caps < (1ull << 31), "too many subtrees");
        const uint32_t w_top = 1u << lg_top;
        launch_after(merkle_top_hex<H>, (unsigned)j.n_caps, 32 * ((w_top + 4) / 5), 0, st, j.digests, j.cap, ds,
                     w_top);
        return;
    }
    merkle_leaves<H><<<blocks_for(j.n_leaves, kLeafThreads), kLeafThreads, 0, st>>>(j.leaves, j.n_leaves, w, j.digests,
                                                                                     map);
    ZK_CHECK_LAUNCH();
    // Wide levels: one launch each, one node per thread.  The narrow top
    // (fewer than kNarrow nodes in all, at most 256 per subtree) goes to
    // merkle_top in one launch.
    constexpr uint64_t kNarrow = 1 << 14;
    uint32_t lg_top = 0;
    while (lg_top + 1 < map.lg_ls && lg_top < 8 && (j.n_caps << (lg_top + 1)) < kNarrow) lg_top++;
    for (uint32_t lg_w = map.lg_ls - 1; lg_w > lg_top; lg_w--)
        launch_after(merkle_level<H, 4>, blocks_for(j.n_caps << lg_w, kLeafThreads), kLeafThreads, 0, st, j.digests,
                     lg_w, j.n_caps, ds);
    require(j.n_caps < (1ull << 31), "too many subtrees");
    const uint32_t w_top = 1u << lg_top;
    launch_after(merkle_top<H>, (unsigned)j.n_caps, std::max<uint32_t>(32, w_top), 0, st, j.digests, j.cap, ds,
                 w_top);
}

}  // namespace

namespace {

// Opening proofs on a resident forest.  Leaf rows: one thread per (query, word).
__global__ void merkle_open_leaves(const uint64_t *__restrict__ leaves, uint64_t n_leaves, uint64_t leaf_size,
                                   const uint64_t *__restrict__ idx, uint64_t n_queries, uint64_t *__restrict__ out) {
    const uint64_t total = n_queries * leaf_size;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t q = t / leaf_size, k = t - q * leaf_size, i = idx[q];
        out[t] = i < n_leaves ? leaves[i * leaf_size + k] : ~0ull;
    }
}

// Siblings: one thread per (query, level).  Level lvl of leaf j (in its
// subtree) is the level of width w = Ls >> lvl at offset w - 2; the sibling of
// node j >> lvl is node (j >> lvl) ^ 1.
__global__ void merkle_open_paths(const uint64_t *__restrict__ digests, uint64_t n_leaves, uint32_t lg_ls, uint64_t ds,
                                  const uint64_t *__restrict__ idx, uint64_t n_queries, uint64_t *__restrict__ out) {
    const uint64_t total = n_queries * lg_ls;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t q = t / lg_ls, lvl = t - q * lg_ls, i = idx[q];
        uint64_t *o = out + 4 * t;
        if (i >= n_leaves) {
#pragma unroll
            for (int k = 0; k < 4; k++) o[k] = ~0ull;
            continue;
        }
        const uint64_t ls = 1ull << lg_ls, s = i >> lg_ls, j = i & (ls - 1);
        const uint64_t w = ls >> lvl;
        const uint64_t *d = digests + 4 * (s * ds + (w - 2) + ((j >> lvl) ^ 1));
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = d[k];
    }
}

unsigned grid_for(uint64_t n) {
    const uint64_t b = (n + 255) / 256;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 32));
}

}  // namespace

void merkle_open(const uint64_t *leaves, const uint64_t *digests, uint64_t n_leaves, uint64_t leaf_size,
                 uint64_t cap_height, const uint64_t *idx, uint64_t n_queries, uint64_t *out_leaves,
                 uint64_t *out_siblings, cudaStream_t st) {
    require(cap_height < 64 && n_leaves >= (1ull << cap_height) && n_leaves % (1ull << cap_height) == 0,
            "n_leaves must be a multiple of 2^cap_height");
    const uint64_t ls = n_leaves >> cap_height;
    require((ls & (ls - 1)) == 0, "leaves per subtree must be a power of two");
    require(leaf_size > 0, "leaf_size out of range");
    if (n_queries == 0) return;
    require(idx && leaves && out_leaves, "null buffer");
    const uint32_t lg_ls = (uint32_t)__builtin_ctzll(ls);
    merkle_open_leaves<<<grid_for(n_queries * leaf_size), 256, 0, st>>>(leaves, n_leaves, leaf_size, idx, n_queries,
                                                                       out_leaves);
    ZK_CHECK_LAUNCH();
    if (lg_ls == 0) return;
    require(digests && out_siblings, "null buffer");
    merkle_open_paths<<<grid_for(n_queries * lg_ls), 256, 0, st>>>(digests, n_leaves, lg_ls, 2 * ls - 2, idx, n_queries,
                                                                   out_siblings);
    ZK_CHECK_LAUNCH();
}

int merkle_autotune_leaves(uint64_t n_leaves, uint64_t leaf_size, uint64_t hash_type, cudaStream_t s) {
    if (hash_type != kPoseidon || leaf_size <= 4 || n_leaves < 2 || n_leaves > kLayoutTuneMax) return 0;
    require(leaf_size < (1ull << 31), "invalid leaf size");
    const uint64_t key = layout_key(n_leaves, leaf_size);
    {
        std::lock_guard<std::mutex> g(g_layout_mu);
        if (g_layout.count(key)) return 0;
    }
    // Zero leaves (canonical) of the class's own shape; digests in direct order.
    uint64_t *leaves = nullptr, *out = nullptr;
    ZK_CUDA(cudaMallocAsync((void **)&leaves, n_leaves * leaf_size * sizeof(uint64_t), s));
    ZK_CUDA(cudaMallocAsync((void **)&out, n_leaves * 4 * sizeof(uint64_t), s));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    uint8_t best = 1;
    float best_ms = 1e30f;
    int timed = 0;
    try {
        ZK_CUDA(cudaMemsetAsync(leaves, 0, n_leaves * leaf_size * sizeof(uint64_t), s));
        ZK_CUDA(cudaEventCreate(&e0));
        ZK_CUDA(cudaEventCreate(&e1));
        const LeafMap direct{};
        for (uint8_t layout : {6, 2, 1}) {
            launch_poseidon_leaves(leaves, n_leaves, (uint32_t)leaf_size, out, direct, layout, s);  // warm-up
            ZK_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < 3; r++)
                launch_poseidon_leaves(leaves, n_leaves, (uint32_t)leaf_size, out, direct, layout, s);
            ZK_CUDA(cudaEventRecord(e1, s));
            ZK_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            ZK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            timed++;
            if (ms < best_ms) best_ms = ms, best = layout;
        }
    } catch (...) {
        cudaStreamSynchronize(s);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFreeAsync(leaves, s);
        cudaFreeAsync(out, s);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ZK_CUDA(cudaFreeAsync(leaves, s));
    ZK_CUDA(cudaFreeAsync(out, s));
    std::lock_guard<std::mutex> g(g_layout_mu);
    g_layout[key] = best;
    return timed;
}

void merkle_autotune_clear() {
    std::lock_guard<std::mutex> g(g_layout_mu);
    g_layout.clear();
}

bool merkle_hash_supported(uint64_t ht) {
    return ht == kPoseidon || ht == kPoseidon2 || ht == kKeccak || ht == kMonolith || ht == kPoseidonBN128;
}

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
    case kMonolith: merkle_run_t<kMonolith>(j, st); break;
    case kPoseidonBN128: merkle_run_t<kPoseidonBN128>(j, st); break;
    default: break;
    }
}

}  // namespace zk
