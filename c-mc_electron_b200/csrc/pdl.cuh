// pdl.cuh -- programmatic dependent launch for the kernels of a step.
//
// A kernel launched with launch_pdl may be scheduled before the kernel
// ahead of it on the stream has finished: its launch overlaps the
// predecessor's tail instead of following its completion.  Every such
// kernel calls pdl_wait() before it reads or writes anything its
// predecessor touches; the wait returns once the predecessor grid has
// completed and its memory is visible (and at once when the kernel was
// launched the ordinary way, or after a memset or an event wait).
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace mcb200 {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace mcb200
