// zk_lde_noalloc: the coset LDE with no device allocation.
//
// Who needs it: callers that cannot call cudaMalloc where they run the LDE.
// Provers that run inside a fixed, pre-reserved memory budget or their own
// arena must not let a library grow the CUDA memory pool behind their back
// (the regular entry points allocate the NTT intermediate and the twiddle /
// coset tables on demand, and the pool keeps that memory); embedders with
// hard latency limits forbid allocation calls on their hot path, because
// cudaMalloc can synchronise the device and take milliseconds.  This entry
// point keeps its intermediate and tables in one file-scope device array of
// fixed size instead.
//
// Limits and sharing rules:
//  * the array holds 2^22 elements of NTT intermediate (32 MiB) plus the
//    tables (96 KiB); every GPU that loads this part of the library keeps it
//    until the process exits;
//  * transforms up to 2^22 points (lg_n + rate_bits <= 22) are accepted;
//    larger ones are rejected with code cudaErrorMemoryAllocation (2) and a
//    NULL message (the message is not allocated either);
//  * every call reuses the same array and leaves its contents behind (its
//    tables are rewritten by each call, and its intermediate is fully written
//    before it is read); calls whose work overlaps on the GPU (different
//    streams, or different host threads) race on it and must be serialised by
//    the caller;
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress, which also loads this module on that device); make
//    that first call before any stream capture on the device;
//  * the coset is the one the device's coset LDEs use: generator 7, or the one
//    init_coset installed last;
//  * a CUDA failure inside the transform (a launch error) is raised and caught
//    internally; that path allocates host memory for the error text, which
//    zk_last_error() then returns.  Argument and size errors allocate nothing.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/zeknox.h"
#include "gl64.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

namespace {

constexpr uint32_t kMaxLg = 22;
constexpr uint64_t kScratchElems = 1ull << kMaxLg;
constexpr uint64_t kLineElems = 1ull << zk::kLineLgMax;  // omega_4096^j
constexpr uint64_t kPowElems = 2ull << ((kMaxLg + 1) / 2);  // two-level table, lg <= 22
constexpr uint64_t kTotalElems = kScratchElems + kLineElems + 2 * kPowElems;
constexpr int kMaxDevices = 64;

// The whole working set of the entry point.  Host code must not use this name
// as an address (it is a host-side stand-in); it uses the pointer resolved by
// cudaGetSymbolAddress below.
static __device__ __align__(256) uint64_t g_noalloc[kTotalElems];

std::mutex g_mu;
uint64_t *g_base[kMaxDevices] = {};

// b^e for e < 2^bits by square-and-multiply.
__device__ uint64_t dev_pow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = zk::gl_mul(r, b);
        b = zk::gl_mul(b, b);
        e >>= 1;
    }
    return r;
}

// Fill one table: dst[j] = base^j for j < n_lo, then dst[n_lo + j] =
// base^(j * n_lo) for j < n_hi (n_hi = 0: single-level table).
__global__ void fill_pow_table(uint64_t *dst, uint64_t base, uint64_t n_lo, uint64_t n_hi) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n_lo + n_hi;
         j += (uint64_t)gridDim.x * blockDim.x)
        dst[j] = j < n_lo ? dev_pow(base, j) : dev_pow(base, (j - n_lo) * n_lo);
}

RustError err(int code) { return RustError{code, nullptr}; }

}  // namespace

extern "C" RustError zk_lde_noalloc(void *d_output, const void *d_input, uint32_t lg_n, uint32_t rate_bits,
                                   uint32_t batches, uint32_t inv, uint32_t with_coset, void *stream) {
    const uint32_t lg = lg_n + rate_bits;
    if (lg_n == 0 || rate_bits == 0 || !d_output || !d_input || batches > (1u << 30))
        return err((int)cudaErrorInvalidValue);
    if (lg > kMaxLg || lg < lg_n) return err((int)cudaErrorMemoryAllocation);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return err(-(int)e);
    if (dev < 0 || dev >= kMaxDevices) return err((int)cudaErrorInvalidDevice);
    uint64_t *base;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (!g_base[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc);
            if (e != cudaSuccess) return err(-(int)e);
            g_base[dev] = (uint64_t *)p;
        }
        base = g_base[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t *scratch = base, *line = base + kScratchElems, *roots_dev = line + kLineElems,
             *coset_dev = roots_dev + kPowElems;

    // Tables for this call: the same values as the cached tables of the regular
    // path, coset generator included.
    const bool inverse = inv != 0;
    const uint64_t gen = zk::installed_coset_generator(dev);
    uint64_t w4096 = zk::h_omega(zk::kLineLgMax), wn = zk::h_omega(lg);
    if (inverse) {
        w4096 = zk::h_inv(w4096);
        wn = zk::h_inv(wn);
    }
    zk::PowTable roots, cos;
    roots.dev = roots_dev;
    roots.bits = lg;
    roots.h = (lg + 1) / 2;
    roots.base = wn;
    cos.dev = coset_dev;
    cos.bits = lg;
    cos.h = (lg + 1) / 2;
    cos.base = gen;
    const uint64_t lo_n = 1ull << roots.h, hi_n = 1ull << (lg - roots.h);
    // Each launch is checked and counted like every other launch of the library.
    auto launched = [] {
        const cudaError_t le = cudaGetLastError();
        if (le == cudaSuccess) zk::note_launch();
        return le;
    };
    fill_pow_table<<<16, 256, 0, s>>>(line, w4096, kLineElems, 0);
    if ((e = launched()) != cudaSuccess) return err(-(int)e);
    fill_pow_table<<<8, 256, 0, s>>>(roots_dev, wn, lo_n, hi_n);
    if ((e = launched()) != cudaSuccess) return err(-(int)e);
    if (with_coset) {
        fill_pow_table<<<8, 256, 0, s>>>(coset_dev, gen, lo_n, hi_n);
        if ((e = launched()) != cudaSuccess) return err(-(int)e);
    }

    zk::NttJob j;
    j.src = (const uint64_t *)d_input;
    j.src_stride = 1ull << lg_n;
    j.n_valid = 1ull << lg_n;
    j.dst = (uint64_t *)d_output;
    j.dst_stride = 1ull << lg;
    j.batches = batches;
    j.lg = lg;
    j.inverse = inverse;
    if (with_coset) (inverse ? j.post_coset : j.pre_coset) = &cos;
    if (inverse) j.scale = zk::h_inv(1ull << lg);
    j.scratch = scratch;
    j.scratch_elems = kScratchElems;
    try {
        zk::ntt_run_on_tables(j, roots, line, s);
    } catch (const zk::Error &ex) {
        zk::record_last_error(ex.code, ex.what());
        return err(ex.code);
    } catch (const std::exception &ex) {
        zk::record_last_error(-(int)cudaErrorUnknown, ex.what());
        return err(-(int)cudaErrorUnknown);
    }
    return err(0);
}
