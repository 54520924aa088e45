// pdl.cuh — programmatic dependent launch of the kernels of a step
// (DIMGPU_PDL, dim_launch.h).  A kernel launched with programmatic stream
// serialization may be scheduled while its predecessor in the stream
// drains.  Every such kernel calls pdl_enter() first: griddepcontrol.wait
// (the predecessor has completed and its writes are visible) before it
// touches anything, so each kernel still completes after its predecessor,
// then griddepcontrol.launch_dependents, which lets its own successor be
// scheduled early.  A kernel launched plainly passes through pdl_enter()
// at once.
#pragma once

#include <cuda_runtime.h>

#include <utility>

#include "dim_launch.h"

namespace dimgpu {

template<bool On>
__device__ __forceinline__ void pdl_enter_if()
{
    if (On) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }
}

__device__ __forceinline__ void pdl_enter() { pdl_enter_if<DIMGPU_PDL>(); }

// Launch with programmatic stream serialization when On (plainly otherwise).
template<bool On, typename... KArgs, typename... Args>
cudaError_t launch_chained(void (*kern)(KArgs...), unsigned blocks, unsigned threads, size_t smem, cudaStream_t s,
                           Args&&... args)
{
    if (!On) {
        kern<<<blocks, threads, smem, s>>>(std::forward<Args>(args)...);
        return cudaSuccess;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template<typename... KArgs, typename... Args>
cudaError_t launch_stage_smem(void (*kern)(KArgs...), unsigned blocks, unsigned threads, size_t smem, cudaStream_t s,
                              Args&&... args)
{
    return launch_chained<DIMGPU_PDL>(kern, blocks, threads, smem, s, std::forward<Args>(args)...);
}

template<typename... KArgs, typename... Args>
cudaError_t launch_stage_dims(void (*kern)(KArgs...), unsigned blocks, unsigned threads, cudaStream_t s,
                              Args&&... args)
{
    return launch_chained<DIMGPU_PDL>(kern, blocks, threads, 0, s, std::forward<Args>(args)...);
}

template<typename... KArgs, typename... Args>
cudaError_t launch_stage(void (*kern)(KArgs...), unsigned blocks, cudaStream_t s, Args&&... args)
{
    return launch_chained<DIMGPU_PDL>(kern, blocks, 256u, 0, s, std::forward<Args>(args)...);
}

}  // namespace dimgpu
