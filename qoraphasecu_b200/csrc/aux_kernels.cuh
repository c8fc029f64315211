// Element-wise kernels around the iteration: random starts, support cuts,
// the shrinkwrap threshold, detwin and the centre-origin <-> FFT-order rolls.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "line_pass.cuh"

namespace qpb {

struct Dims3 {
  int d0, d1, d2;  // slowest first; 2D is {1, ny, nx}
  QPB_HD long long n() const { return static_cast<long long>(d0) * d1 * d2; }
};

// w[b][i] = A[i] / sqrt(n) * exp(i kTwoPi uniform(seed, k, i)) for global start
// s = first_start + b of problem q = s / starts_per_problem, k = s mod
// starts_per_problem, A = amplitude + q * amp_stride (kernels.cpp:104-117).
void random_wave(float2* w, const float* amplitude, long long amp_stride, int starts_per_problem,
                 long long n, int batch, std::uint64_t seed, std::uint64_t first_start,
                 cudaStream_t stream);

// x[b][i] = 0 outside support[b][i].
void support_project(float2* x, const std::uint8_t* support, long long n, int batch,
                     cudaStream_t stream);

// support[b][i] = Re(blurred[b][i]) > threshold * level(b).
void shrinkwrap_threshold(const float2* blurred, const LevelAcc* acc, long long n, int batch,
                          int method, float threshold, std::uint8_t* support, cudaStream_t stream);

// Detwin: support[b] &= centre-origin coordinate along `axis3` (a Dims3 axis)
// < the support's centre of mass along that axis. `moments` holds 2 u64 per start.
void detwin(std::uint8_t* support, unsigned long long* moments, Dims3 d, int axis3, int batch,
            cudaStream_t stream);

// out[b] = roll(in[b]) with out[i] = in[(i + off(n)) mod n] on every axis:
// to_fft_order uses off = n / 2, to_centered off = n - n / 2.
template <class T>
void roll(const T* in, T* out, Dims3 d, int batch, bool to_fft_order, cudaStream_t stream);

// Writes the control block fields of a stage.
void set_coefficients(Ctrl* ctrl, float a, float b, cudaStream_t stream);

// Writes a whole control block on `stream` (kernel arguments, so no host
// buffer has to outlive the call).
void set_ctrl(Ctrl* ctrl, const Ctrl& value, cudaStream_t stream);

// x[i] = x[i] * scale (complex), used for results of scaled storage.
void scale_complex(float2* x, long long count, float scale, cudaStream_t stream);

// Complex64 <-> fp16 pairs (round to nearest; widening is exact), `count`
// elements, for the fp16 iterate of the half variant.
void to_half(const float2* in, void* out, long long count, cudaStream_t stream);
void from_half(const void* in, float2* out, long long count, cudaStream_t stream);

}  // namespace qpb
