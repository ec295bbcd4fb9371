// pdl.cuh -- programmatic dependent launch for the library's kernels.
//
// A kernel launched with launch_pdl may have its launch processed while the
// previous kernel on the stream is finishing (from the moment that kernel's
// blocks have exited, instead of after the grid's completion has been
// handled).  Every such kernel calls pdl_wait() before touching global
// memory: it returns once the previous grid has completed and its writes are
// visible, and it is a no-op for a launch without a programmatic dependency.
#pragma once
#include <cuda_runtime.h>

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

template <typename... Exp, typename... Act>
cudaError_t launch_pdl(void (*kernel)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Act&&... args) {
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
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<Act&&>(args)...);
}
