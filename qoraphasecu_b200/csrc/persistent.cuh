// The persistent schedule: a chunk of iterations of every start of a 2D
// solver as ONE kernel launch (persistent.cu).
#pragma once

#include <cuda_runtime.h>

#include "line_pass.cuh"

namespace qpb {

// Device words of one launch's work list, zeroed before every launch: the
// next item to claim, the items finished, an abort flag, then per start the
// column (modulus) tiles and the row (update) tiles completed so far.
inline constexpr int kPersistentHead = 4;
inline int persistent_work_words(int starts) { return kPersistentHead + 2 * starts; }

// True for 2D problems whose sides are 64, 128 or 256 points, with the
// modulus pass on the TMA column tiles of 8 lines (the amplitude tiled
// line-major) and complex64 storage.
bool persistent_supports(int ndim, int d1, int d2);

// `iterations` iterations of all starts: `mod` is the modulus pass along y
// (columns), `upd` the update pass along x (rows), both for all starts;
// `work` holds persistent_work_words(starts) zeroed words. Error rows follow
// the control block's counter of mod.group, which the launch advances by
// `iterations`; the update coefficients come from the control block.
void launch_persistent(const PassParams& mod, const PassParams& upd, int starts, int iterations,
                       unsigned* work, cudaStream_t stream);

// CTAs of one launch (for reporting): every SM times the resident CTAs.
int persistent_grid(int d1, int d2);

void configure_persistent();

}  // namespace qpb
