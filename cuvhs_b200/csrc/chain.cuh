// Programmatic dependent launch for the decode's kernel chain (sm_90+).
//
// A kernel launched with launch_chained() is launched as soon as every CTA of
// the kernel before it on the stream has exited, without waiting for that
// kernel's completion to be processed; each chained kernel calls chain_wait()
// before its first global-memory access, which returns once the previous
// kernel has completed and its writes are visible (griddepcontrol.wait).  The
// stream's ordering is unchanged; only the launch latency between the two
// kernels is hidden.  No kernel triggers its dependents early
// (griddepcontrol.launch_dependents): dependents made resident during the
// previous kernel's last wave measured slower on the decode.  Before any other
// stream operation (copy, event, a kernel launched the ordinary way) the usual
// serialisation holds.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace cuvhs {

__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... P, typename... A>
inline cudaError_t launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                  A&&... args) {
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
  // callers that ignore the result see a failed launch in their cudaGetLastError check
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace cuvhs
