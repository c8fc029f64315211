// Programmatic dependent launch of the streamed line passes.
//
// A pass is launched with cudaLaunchAttributeProgrammaticStreamSerialization,
// which lets its CTAs start while the kernel before it in the stream (the
// previous pass) runs its last CTAs: launch, scheduling and the shared-memory
// set-up overlap that kernel's tail instead of following it. Every CTA then
// waits, before its first access of global memory, until the kernel before it
// has completed and its writes are visible, and lets the kernel after it
// start early in turn. Both instructions are no-ops when the kernel was
// launched without the attribute or follows no kernel; the waits end when
// the kernel before ends, so nothing here waits on a condition of its own.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <utility>

#include "common.cuh"

namespace qpb {

// Blocks the calling thread until the kernel this one depends on has
// completed and its memory operations are visible.
__device__ __forceinline__ void wait_for_prior_kernel() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Allows the kernel after this one to be scheduled (it still waits for this
// kernel's completion before touching memory).
__device__ __forceinline__ void allow_next_kernel() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// kernel<<<grid, block, smem, stream>>>(args...) with the attribute above.
template <class... Params, class... Args>
void launch_dependent(void (*kernel)(Params...), dim3 grid, dim3 block, std::size_t smem,
                      cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t config{};
  config.gridDim = grid;
  config.blockDim = block;
  config.dynamicSmemBytes = smem;
  config.stream = stream;
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  config.attrs = &attr;
  config.numAttrs = 1;
  QPB_CHECK(cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...));
}

}  // namespace qpb
