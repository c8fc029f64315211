// Register-resident line passes for power-of-two lengths (fast_pass.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "line_pass.cuh"

namespace qpb {

// True when a register-resident kernel exists for this pass: L a power of two
// in 16..1024 and whole CTAs of lines that never span two starts.
bool fast_pass_supports(const PassParams& p);

void launch_fast_pass(Mode mode, const PassParams& p, cudaStream_t stream);

// False when the environment sets QPB_GENERIC_PASSES=1 (every pass then runs
// the generic kernels; used to compare the two implementations).
bool fast_passes_enabled();

// Lines per CTA of the register-resident kernel for this pass (0: not used).
int fast_pass_lines(const PassParams& p);

// Raises the dynamic shared-memory limit of the kernels that need more than
// 48 KiB; once per device, outside stream capture.
void configure_fast_passes();

}  // namespace qpb
