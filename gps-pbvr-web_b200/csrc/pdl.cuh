// Kernel launches with programmatic stream serialisation (programmatic dependent launch): the
// launched kernel's CTAs may start while the previous kernel on the stream is finishing, so their
// set-up overlaps its tail. Such a kernel executes griddepcontrol.wait (which returns once the
// previous grid has completed and its memory operations are visible) before it reads anything
// earlier work wrote or writes anything earlier work reads, and griddepcontrol.launch_dependents
// once its own dependents may be scheduled. Captured into a CUDA graph the dependency becomes a
// programmatic edge.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace gpsb {

template <typename... Params, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace gpsb
