// launch.cuh — programmatic dependent launch (PDL) for the chained kernels
// of one batch (bitmaps -> query prep -> seeding pass -> merge -> main pass
// -> merge -> re-rank).
//
// A kernel launched with launch_pdl may begin (its CTAs scheduled, their
// shared-memory / tensor-memory setup run) while the previous kernel on the
// stream is still finishing; it must call pdl_wait() before its first
// access to global memory, which returns once the previous grid has
// completed and its writes are visible. Each kernel calls pdl_trigger()
// once its own CTAs are all resident, which lets the next kernel's CTAs
// launch into the SMs that free up. After a copy, a fill or a kernel
// launched without the attribute, pdl_wait() returns at once and the
// ordinary stream order holds.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace pv {

__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace pv
