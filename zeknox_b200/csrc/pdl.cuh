// Programmatic dependent launch (sm_90 and later).  A kernel launched with
// launch_after may start while the kernel before it on the stream drains: it
// first does what does not depend on that kernel (round tables, twiddles into
// shared memory), then waits with pdl_wait() until the previous grid has
// completed and its writes are visible.  Every read of the previous kernel's
// output and every write comes after that wait.  A kernel may call
// pdl_release() once its block has stored its outputs, to let the dependent
// grid launch before it fully exits (otherwise that happens at its exit).
// Both instructions are no-ops in a kernel launched without the attribute.
// launch_after is only used where the previous operation on the stream is a
// kernel of the same chain (a transform's earlier pass, the tree's previous
// level).
#pragma once
#include <cuda_runtime.h>

#include "runtime.cuh"

namespace zk {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... P, typename... A>
void launch_after(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    ZK_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
    ZK_CHECK_LAUNCH();
}

}  // namespace zk
