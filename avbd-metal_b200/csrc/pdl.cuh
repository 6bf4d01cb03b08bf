// pdl.cuh — programmatic dependent launch for the iteration loop, a chain
// of ~100-300 dependent kernels per frame.  Each kernel lets the next one be
// scheduled as soon as all of its own blocks are running, and waits for the
// previous grid to complete (and its writes to be visible) before touching
// solver state.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace avbd {

__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_prologue() {
    pdl_trigger();
    pdl_wait();
}


template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kernel)(KArgs...), uint32_t blocks, uint32_t threads, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace avbd
