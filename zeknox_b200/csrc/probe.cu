// Measurement aids for the benchmark (libzkprobe.so, not part of the C ABI):
//  * the INT32 multiply-add issue rate of the current GPU, the denominator of
//    the integer roofline of the hash kernels: each thread runs 8 independent
//    mad.lo.u32 chains; the rate is (threads * 8 * iterations) / elapsed,
//    timed with CUDA events;
//  * the field operations of the NTT and hash kernels, one kernel each, for
//    counting their instructions with ncu (zk_probe_field_ops).
#include <cuda_runtime.h>
#include <stdint.h>

#include "gl64.cuh"
#include "ntt_field.cuh"

namespace {

__global__ void imad_chains(uint32_t *out, uint32_t iters, uint32_t seed) {
    uint32_t a0 = threadIdx.x ^ seed, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
             a7 = a0 + 7;
    const uint32_t m = 0x9E3779B1u | seed, c = blockIdx.x;
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            asm volatile(
                "mad.lo.u32 %0, %0, %8, %9;\n\t"
                "mad.lo.u32 %1, %1, %8, %9;\n\t"
                "mad.lo.u32 %2, %2, %8, %9;\n\t"
                "mad.lo.u32 %3, %3, %8, %9;\n\t"
                "mad.lo.u32 %4, %4, %8, %9;\n\t"
                "mad.lo.u32 %5, %5, %8, %9;\n\t"
                "mad.lo.u32 %6, %6, %8, %9;\n\t"
                "mad.lo.u32 %7, %7, %8, %9;\n\t"
                : "+r"(a0), "+r"(a1), "+r"(a2), "+r"(a3), "+r"(a4), "+r"(a5), "+r"(a6), "+r"(a7)
                : "r"(m), "r"(c));
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
}

}  // namespace

// Returns INT32 IMAD operations per second (best of `reps`), or a negative
// CUDA error code.
extern "C" __attribute__((visibility("default"))) double zk_probe_imad_ops_per_s(int reps) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256, blocks = sms * 8;
    const uint32_t iters = 2048;
    uint32_t *out = nullptr;
    if (cudaMalloc(&out, sizeof(uint32_t) * threads * blocks) != cudaSuccess) return -2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0;
    imad_chains<<<blocks, threads>>>(out, 64, 1);  // warm-up
    for (int r = 0; r < reps; r++) {
        cudaEventRecord(e0);
        imad_chains<<<blocks, threads>>>(out, iters, (uint32_t)r);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = (double)threads * blocks * iters * 16 * 8;
        if (ms > 0 && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return err == cudaSuccess ? best : -(double)err;
}

// ---- field operations, one warp each: `iters` dependent applications of one
// operation (a <- op(a, b); b <- b ^ a), so that ncu's instruction count of
// the kernel minus probe_base's, divided by iters, is the instructions of one
// application (probe_dft8 against probe_dft8_base: eight 64-bit adds).
namespace {
using namespace zk;
using namespace zk::ntf;

#define ZK_PROBE_OP(name, ...)                                                   \
    __global__ void name(uint64_t *out, uint64_t a0, uint64_t b0, int iters) {     \
        uint64_t a = (a0 + threadIdx.x) % ZK_P, b = (b0 ^ threadIdx.x) % ZK_P;       \
        _Pragma("unroll 1") for (int i = 0; i < iters; i++) { __VA_ARGS__; }       \
        out[threadIdx.x] = a ^ b;                                                  \
    }
ZK_PROBE_OP(probe_base, a = a + b; b = b ^ a)
ZK_PROBE_OP(probe_nt_add, a = nt_add(a, b); b = b ^ a)
ZK_PROBE_OP(probe_nt_sub, a = nt_sub(a, b); b = b ^ a)
ZK_PROBE_OP(probe_nt_mul, a = nt_mul(a, b); b = b ^ a)
ZK_PROBE_OP(probe_mul2_24, a = gl_mul2_24(a); b = b ^ a)
ZK_PROBE_OP(probe_mul2_48, a = gl_mul2_48(a); b = b ^ a)
ZK_PROBE_OP(probe_mul2_72, a = gl_mul2_72(a); b = b ^ a)
ZK_PROBE_OP(probe_pr_mul, a = pr_mul(a, b); b = b ^ a)
ZK_PROBE_OP(probe_pr_sqr, a = pr_sqr(a); b = b ^ a)
ZK_PROBE_OP(probe_pr_pow7, a = pr_pow7(a); b = b ^ a)
#undef ZK_PROBE_OP

__global__ void probe_dft8(uint64_t *out, uint64_t a0, uint64_t, int iters) {
    uint64_t x[8];
    for (int k = 0; k < 8; k++) x[k] = (a0 * (k + 1) + threadIdx.x) % ZK_P;
#pragma unroll 1
    for (int i = 0; i < iters; i++) dft8(x, false);
    uint64_t r = 0;
    for (int k = 0; k < 8; k++) r ^= x[k];
    out[threadIdx.x] = r;
}
__global__ void probe_dft8_base(uint64_t *out, uint64_t a0, uint64_t, int iters) {
    uint64_t x[8];
    for (int k = 0; k < 8; k++) x[k] = (a0 * (k + 1) + threadIdx.x) % ZK_P;
#pragma unroll 1
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = x[k] + x[(k + 1) & 7];
    }
    uint64_t r = 0;
    for (int k = 0; k < 8; k++) r ^= x[k];
    out[threadIdx.x] = r;
}
}  // namespace

// Launches every field-operation kernel once (one warp, `iters` applications
// each); returns 0 or a negative CUDA error code.
extern "C" __attribute__((visibility("default"))) int zk_probe_field_ops(int iters) {
    uint64_t *out = nullptr;
    if (cudaMalloc(&out, 32 * sizeof(uint64_t)) != cudaSuccess) return -2;
    void (*ops[])(uint64_t *, uint64_t, uint64_t, int) = {
        probe_base, probe_nt_add, probe_nt_sub, probe_nt_mul, probe_mul2_24, probe_mul2_48, probe_mul2_72,
        probe_pr_mul, probe_pr_sqr, probe_pr_pow7, probe_dft8_base, probe_dft8};
    for (auto k : ops) k<<<1, 32>>>(out, 0x123456789abcdefull, 0xfedcba9876543210ull, iters);
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(out);
    return e == cudaSuccess ? 0 : -(int)e;
}
