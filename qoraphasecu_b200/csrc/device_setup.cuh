// Problem set-up from arrays already on the device.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "line_pass.cuh"

namespace qpb {

struct ProblemView;
struct Dims3;

// make_problem (src/core/problem.cpp:40-70) on device arrays, centre-origin:
// amplitude = sqrt(max(I, 0)), mask and support as 0/1, a NULL support
// replaced by the autocorrelation support at `support_threshold` (computed on
// the device). Enqueued on `stream`; returns after it, raising
// InvalidArgument for non-finite intensities or a mask that covers everything.
// Works in the calling device's set-up arena (no allocation once it has grown
// to the problem's size).
void make_problem_device(const float* intensity, int ndim, const long long* shape,
                         const std::uint8_t* support, const std::uint8_t* mask,
                         float support_threshold, float* amplitude_out, std::uint8_t* mask_out,
                         std::uint8_t* support_out, cudaStream_t stream);

// The autocorrelation support (problem.cpp:72-88) of a centre-origin host
// intensity, computed on the calling device in its set-up arena: the
// intensity goes up, the 0/1 support comes back.
void autocorrelation_support_host(const float* intensity, int ndim, const long long* shape,
                                  float threshold, std::uint8_t* out);

// Device bytes of `scratch` that prepare_problem_device needs for n elements
// (a multiple of 256).
std::size_t prepare_scratch_bytes(long long n);

// One problem's solver inputs from its device arrays (centre-origin): the FFT-
// order FP32 amplitude, the signed amplitude (-1 masked) in `storage` written
// to `signed_out` in the modulus pass's CTA order when `lines` > 0 and S > 1
// (tiles of `lines` lines, line-major inside a tile when `line_major`),
// the FFT-order 0/1 support, and the usable energy (sum of A^2 over unmasked
// pixels, in one fixed order: the same bits on every call) into the device
// double `energy`. With `peak` (a device float) the amplitude is first
// divided by its peak, which `peak` receives (fp16 wave storage). Enqueued on
// `stream`, which it does not synchronise. `scratch`:
// prepare_scratch_bytes(n) device bytes, in use until the work ends.
void prepare_problem_device(const ProblemView& q, Dims3 d, AmpStorage storage, int L, int S,
                            int lines, bool line_major, float* amp_fft, void* signed_out,
                            std::uint8_t* support_fft, void* scratch, double* energy,
                            float* peak, cudaStream_t stream);

}  // namespace qpb
