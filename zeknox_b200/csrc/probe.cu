// Measurement aid for the benchmark (libzkprobe.so, not part of the C ABI):
// the INT32 multiply-add issue rate of the current GPU, the denominator of
// the integer roofline of the hash kernels.
//
// Each thread runs 8 independent mad.lo.u32 chains; the rate is
// (threads * 8 * iterations) / elapsed, timed with CUDA events.
#include <cuda_runtime.h>
#include <stdint.h>

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
