// Kernel launch with programmatic stream serialisation (programmatic dependent launch): the kernel may be scheduled
// while the previous kernel in the stream is still running, and must call pdl_enter() (kernel_util.cuh) before it
// reads anything that kernel wrote.  Captured into CUDA graphs as programmatic edges.  Used by the chains of small
// dependent kernels (the MLs groups), where the launch latency between kernels, not their work, sets the time.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace pty {

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
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

}  // namespace pty
