// Resident iteration kernel: whole iterations of square 2D problems (side 64,
// 128 or 256) with each start's iterate, wave and support held in the shared
// memory of a thread-block cluster for a whole chunk of iterations.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "line_pass.cuh"

namespace qpb {

struct ResidentParams {
  float2* x;                     // [starts][n] iterate, FFT order (read at start, written at end)
  float2* w;                     // [starts][n] x-axis transform of x (written at end)
  const void* amp;               // signed amplitude (-1 masked), FFT order, [n], amp_storage type
  long long amp_stride;          // elements between problems' amplitudes (0: one problem)
  int starts_per_problem;
  const std::uint8_t* support;   // [starts][n]
  Ctrl* ctrl;                    // coefficients, error rows, counters[group] = first error row
  const float2* twiddle;         // stage-major table of the N-point transform (stage_table.hpp)
  int group;
  int start0;                    // first global start of the launch (error column)
  int starts_total;              // error row width
  int iterations;                // iterations this launch runs
  float scale;                   // 1/N (= 1/sqrt(n))
  AmpStorage amp_storage;
};

// Side lengths with a resident kernel (square 2D problems only): 64, 128, 256.
bool resident_supports(int ndim, int d1, int d2);

// CTAs per start (the cluster size) for side N.
int resident_cluster(int side);

// Clusters of the side-N kernel that the current device runs at once.
int resident_max_clusters(int side);

// Enqueues `p.iterations` iterations of `starts` starts of an N x N problem, then
// advances ctrl->counters[group] by that count.
void launch_resident(const ResidentParams& p, int side, int starts, cudaStream_t stream);

// Raises the shared-memory limits of the resident kernels on the current device
// (once per device, outside stream capture).
void configure_resident();

}  // namespace qpb
