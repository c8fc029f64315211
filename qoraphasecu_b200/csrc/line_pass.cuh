// Line passes: batched 1D FFTs along one axis of a stack of FFT-order arrays,
// each fused with the point-wise step that follows or precedes it in the
// phase-retrieval iteration.
//
// An n-D transform is a sequence of passes, one per axis. Per iteration the
// solver runs (2D) Mod along y then Upd along x, keeping the invariant that the
// wave buffer `w` holds the x-axis transform of the iterate between
// iterations; 3D adds Inv/Fwd passes along y.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "fft_plan.hpp"

namespace qpb {

enum class Mode : int {
  kFwd,      // w <- FFT(w)
  kFwdFromX, // w <- FFT(x)
  kInv,      // w <- IFFT(w)
  kMod,      // w <- IFFT(P_M FFT(w)) and the Fourier-error numerator per start
  kUpd,      // P <- IFFT(w); x <- S ? P : a x + b P; w <- FFT(x)
  kBlur,     // w <- IFFT(g FFT(w)), g = exp(k f^2) / L along this axis
  kBlurMag,  // as kBlur on (|x|, 0)
  kGrad,     // w <- IFFT(2 (1 - A / (|y| + eps)) y), y = FFT(w), and sum (|y| - A)^2:
             // the gradient of the amplitude loss, 2 (x - P_M x)
};


enum class AmpStorage : int { kF32 = 0, kF16 = 1, kBF16 = 2 };

// Device control block shared by the kernels of one solver. Captured graphs
// reference it by address, so per-stage values live here instead of in
// kernel arguments.
struct Ctrl {
  double* errs;    // [capacity][starts_total] Fourier-error numerators
  int capacity;    // rows of errs
  float a;         // update coefficients of the current stage
  float b;
  int* counters;   // iteration counter per start group
};

// Per-start shrinkwrap level accumulator.
struct LevelAcc {
  double sum;
  unsigned long long count;
  int max_bits;  // bits of a non-negative float: ordered like the float
  int pad;
};

struct PassParams {
  float2* w;
  float2* x;
  const void* amp;                // signed amplitude (-1 masked), FFT order, one per problem
  // Several problems of one shape: the amplitude of global start s is at
  // amp + (s / starts_per_problem) * amp_stride elements (amp_stride 0: one problem).
  long long amp_stride;
  int starts_per_problem;
  const std::uint8_t* support;    // [batch][n]
  Ctrl* ctrl;
  LevelAcc* level;                // [batch], kBlur with level != 0
  const float2* twiddle;          // W_L^k, k < L
  const float2* stage_twiddle;    // the register-resident passes' stage-major table
  long long n;                    // elements per start
  int L;                          // line length
  int S;                          // element stride of a line
  int lines;                      // lines in this launch
  int lines_per_start;
  int lpc;                        // lines per CTA (divides lines_per_start)
  int group;                      // counter index (kMod, kUpd)
  int start0;                     // first global start of the batch (error column)
  int starts_total;               // error row width
  int stages;
  int radix[kMaxStages];
  float scale;                    // 1/sqrt(n) (kMod)
  float blur_k;                   // -2 (pi sigma)^2 (kBlur)
  int level_method;               // 0 none, 1 max, 2 rms (kBlur)
  float coef_a;                   // immediate coefficients when !coef_from_ctrl
  float coef_b;
  int coef_from_ctrl;
  int bump_counter;               // kUpd increments ctrl->counters[group]
  AmpStorage amp_storage;
  // The amplitude is stored in the CTA order of the modulus pass (written so
  // by the problem set-up's signed_kernel) instead of FFT order: one
  // contiguous tile per CTA, element-major for the register-resident pass
  // (kAmpTiledElements) or line-major for the TMA column pass
  // (kAmpTiledLines); 0 = FFT order.
  int amp_tiled;
  // Bounded waits of the staged (bulk-copied) inputs: polls before a wait
  // gives up, and the device counter a CTA that gave up increments (owned by
  // whoever launches the pass and checked by it afterwards).
  int wait_tries;
  int* wait_failures;
  // Fault injection for the tests of the timeout path: the staged copies are
  // not issued, so every staged wait runs out (nothing is left in flight).
  int starve;
  // Storage of the wave (w) and of the iterate (x): 0 complex64, 1 fp16
  // pairs (__half2; x and w then point at half2 arrays). With an fp16 wave a
  // modulus pass leaves the inverse's 1/sqrt(n) to the update pass, which
  // applies it after its inverse transform (values stay in fp16 range).
  int wave_half;
  int iter_half;
};

inline constexpr int kAmpTiledElements = 1;
inline constexpr int kAmpTiledLines = 2;

// Line-major tiles (kAmpTiledLines) store line `line` of a tile rotated by
// this many elements (element j at (j + rotation) mod L), so that the lines
// one warp of a column tile reads (32 / T of them, T = the transform's
// threads per line: L / 8 up to 64 points, L / 16 above) fall on disjoint
// shared-memory banks.
QPB_HD int amp_line_rotation(int L, int line) {
  const int T = L <= 64 ? L / 8 : L / 16;
  return T * (line % (32 / T));
}

// Element offset of the amplitude that global start `start` reads.
QPB_HD long long amp_offset(const PassParams& p, int start) {
  return p.amp_stride ? static_cast<long long>(start / p.starts_per_problem) * p.amp_stride : 0;
}

// Launches one generic line pass on `stream`.
void launch_line_pass(Mode mode, const PassParams& p, cudaStream_t stream);

// Raises the shared-memory limit of every line-pass kernel on the current
// device; called once per device before the first launch (never during capture).
void configure_line_passes();

// Lines per CTA for a line of length L with `lines_per_start` lines per start.
int choose_lpc(int L, int S, int lines_per_start);

}  // namespace qpb
