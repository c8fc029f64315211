// Column line passes whose tiles move by TMA tensor copies (column_pass.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "line_pass.cuh"

namespace qpb {

// False when the environment sets QPB_COLUMN_PASSES=0 (column passes then run
// the register-resident kernels of fast_pass.cu; used to compare the two).
bool column_passes_enabled();

// Lines per CTA of the TMA column pass for `mode` with these parameters, or 0
// when it does not take the pass: strided lines (S > 1) of 64, 128, 256 or 512
// points, CTAs of 8 adjacent columns that never span two starts, modes kMod
// (p.amp_tiled == kAmpTiledLines: the amplitude tiled line-major in this
// pass's CTA order), kFwd and kInv.
int column_pass_lines(const PassParams& p, Mode mode);

// True where the TMA column pass is the one to run on this column axis: it can
// (column_pass_lines) and its lines have 128, 256 or 512 points. At 256 it is the
// faster pass (the 256^2 benchmark's modulus pass: 14.2 against 14.6 us, its
// step 12.2 against 12.8 ms); at 128 the 128^3 crystal's whole iteration runs
// 2.6% faster with it (36.6 k against 35.6 k start-iterations/s), although
// its y-axis passes alone take about 2 us longer than the register-resident
// ones; at 512 its modulus pass takes 109 against 128 us (64 starts). Lines
// of 64 points run the register-resident column pass.
bool column_pass_preferred(const PassParams& p, Mode mode);

void launch_column_pass(Mode mode, const PassParams& p, cudaStream_t stream);

// The tensor map of a complex64 wave that column tiles of 8 lines move:
// p.w as {S, L, p.lines / S} elements, box [1][L][8], 64-byte swizzle.
CUtensorMap column_wave_map(const PassParams& p);

// Raises the dynamic shared-memory limit where needed; once per device,
// outside stream capture.
void configure_column_passes();

}  // namespace qpb
