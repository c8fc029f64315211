// Generic shared-memory line pass: any line length up to kMaxLine whose prime
// factors are at most kMaxPrimeRadix. A CTA loads `lpc` lines into shared
// memory, runs mixed-radix Stockham stages between two shared buffers, applies
// the fused point-wise step and stores the lines back.
//
// This is the path for every shape; power-of-two lengths additionally have the
// register-resident kernels of fast_pass.cu.

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <set>
#include <stdexcept>

#include "butterfly.cuh"
#include "column_pass.cuh"
#include "fast_pass.cuh"
#include "line_pass.cuh"
#include "projection.cuh"
#include "reduce.cuh"

namespace qpb {

namespace {

constexpr int kThreads = 256;

template <bool INV>
__device__ __forceinline__ float2 twiddle(float2 v, const float2* __restrict__ tw, int e) {
  const float2 w = __ldg(tw + e);
  return INV ? cmulc(v, w) : cmul(v, w);
}

// One Stockham stage of radix R over `lines` lines of length L (pitch ldl):
// butterfly j reads src[j + q M] (M = L / R), twiddles by W_{Ns R}^{q (j mod Ns)}
// and writes dst[(j / Ns) Ns R + (j mod Ns) + q Ns].
template <bool INV>
__device__ void stockham_stage(const float2* __restrict__ src, float2* __restrict__ dst, int L,
                               int R, int Ns, const float2* __restrict__ tw, int lines, int ldl) {
  const int M = L / R;
  const int step = L / (Ns * R);
  const int total = lines * M;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int l = t / M;
    const int j = t - l * M;
    const float2* s = src + l * ldl;
    float2* d = dst + l * ldl;
    const int k = j % Ns;
    const int out = (j - k) * R + k;
    const int e = k * step;  // twiddle exponent of input q is q * e
    switch (R) {
      case 2: {
        float2 v0 = s[j], v1 = twiddle<INV>(s[j + M], tw, e);
        bfly2<INV>(v0, v1);
        d[out] = v0;
        d[out + Ns] = v1;
        break;
      }
      case 3: {
        float2 v0 = s[j], v1 = twiddle<INV>(s[j + M], tw, e),
               v2 = twiddle<INV>(s[j + 2 * M], tw, 2 * e);
        bfly3<INV>(v0, v1, v2);
        d[out] = v0;
        d[out + Ns] = v1;
        d[out + 2 * Ns] = v2;
        break;
      }
      case 4: {
        float2 v0 = s[j], v1 = twiddle<INV>(s[j + M], tw, e),
               v2 = twiddle<INV>(s[j + 2 * M], tw, 2 * e),
               v3 = twiddle<INV>(s[j + 3 * M], tw, 3 * e);
        bfly4<INV>(v0, v1, v2, v3);
        d[out] = v0;
        d[out + Ns] = v1;
        d[out + 2 * Ns] = v2;
        d[out + 3 * Ns] = v3;
        break;
      }
      case 5: {
        float2 v0 = s[j], v1 = twiddle<INV>(s[j + M], tw, e),
               v2 = twiddle<INV>(s[j + 2 * M], tw, 2 * e),
               v3 = twiddle<INV>(s[j + 3 * M], tw, 3 * e),
               v4 = twiddle<INV>(s[j + 4 * M], tw, 4 * e);
        bfly5<INV>(v0, v1, v2, v3, v4);
        d[out] = v0;
        d[out + Ns] = v1;
        d[out + 2 * Ns] = v2;
        d[out + 3 * Ns] = v3;
        d[out + 4 * Ns] = v4;
        break;
      }
      case 8: {
        float2 v[8];
        v[0] = s[j];
#pragma unroll
        for (int q = 1; q < 8; ++q) v[q] = twiddle<INV>(s[j + q * M], tw, q * e);
        bfly8<INV>(v);
#pragma unroll
        for (int q = 0; q < 8; ++q) d[out + q * Ns] = v[q];
        break;
      }
      default: {
        // Direct DFT of a prime radix: X[m] = sum_q v_q W_R^{q m}, W_R = W_L^{L / R}.
        const int wr = L / R;
        for (int m = 0; m < R; ++m) {
          float2 acc = {0.0f, 0.0f};
          for (int q = 0; q < R; ++q) {
            const float2 vq = q == 0 ? s[j] : twiddle<INV>(s[j + q * M], tw, q * e);
            acc = cadd(acc, twiddle<INV>(vq, tw, ((q * m) % R) * wr));
          }
          d[out + m * Ns] = acc;
        }
        break;
      }
    }
  }
}

// Runs every stage; returns the buffer holding the result (a or b).
template <bool INV>
__device__ float2* run_stages(const PassParams& p, float2* a, float2* b, int ldl) {
  int Ns = 1;
  for (int s = 0; s < p.stages; ++s) {
    stockham_stage<INV>(a, b, p.L, p.radix[s], Ns, p.twiddle, p.lpc, ldl);
    __syncthreads();
    Ns *= p.radix[s];
    float2* t = a;
    a = b;
    b = t;
  }
  return a;
}

template <class AmpT>
__device__ __forceinline__ float load_amp(const void* amp, long long i) {
  if constexpr (std::is_same_v<AmpT, float>) {
    return __ldg(static_cast<const float*>(amp) + i);
  } else if constexpr (std::is_same_v<AmpT, __half>) {
    return __half2float(static_cast<const __half*>(amp)[i]);
  } else {
    return __bfloat162float(static_cast<const __nv_bfloat16*>(amp)[i]);
  }
}

// Global element of (line, j).
__device__ __forceinline__ long long element(const PassParams& p, long long line, int j) {
  const long long outer = line / p.S;
  const long long inner = line - outer * p.S;
  return outer * static_cast<long long>(p.L) * p.S + inner + static_cast<long long>(j) * p.S;
}

// Index (l, j) of the idx-th element a thread moves: rows walk along the line,
// strided lines walk across lines first so neighbouring threads touch
// neighbouring addresses.
__device__ __forceinline__ void tile_coords(const PassParams& p, int idx, int& l, int& j) {
  if (p.S == 1) {
    l = idx / p.L;
    j = idx - l * p.L;
  } else {
    j = idx / p.lpc;
    l = idx - j * p.lpc;
  }
}

template <Mode M, class AmpT>
__global__ void __launch_bounds__(kThreads) line_pass_kernel(const PassParams p) {
  extern __shared__ float2 smem[];
  const int ldl = p.L;
  float2* buf_a = smem;
  float2* buf_b = smem + p.lpc * ldl;
  const long long line0 = static_cast<long long>(blockIdx.x) * p.lpc;
  const int batch_start = static_cast<int>(line0 / p.lines_per_start);
  const long long start_off = static_cast<long long>(batch_start) * p.n;
  const int tile = p.lpc * p.L;

  // ---- load
  for (int idx = threadIdx.x; idx < tile; idx += blockDim.x) {
    int l, j;
    tile_coords(p, idx, l, j);
    const long long g = element(p, line0 + l, j);
    float2 v;
    if constexpr (M == Mode::kFwdFromX) {
      v = p.x[g];
    } else if constexpr (M == Mode::kBlurMag) {
      const float2 xv = p.x[g];
      v = {sqrtf(xv.x * xv.x + xv.y * xv.y), 0.0f};
    } else {
      v = p.w[g];
    }
    buf_a[l * ldl + j] = v;
  }
  __syncthreads();

  constexpr bool kStartsInverse = M == Mode::kInv || M == Mode::kUpd;
  float2* res = run_stages<kStartsInverse>(p, buf_a, buf_b, ldl);
  float2* other = res == buf_a ? buf_b : buf_a;

  if constexpr (M == Mode::kMod || M == Mode::kGrad) {
    // P_M (or the loss gradient) on the unnormalised transform: scaled by s in,
    // and by s out so that the unnormalised inverse lands on the unitary result.
    float acc = 0.0f;
    const float s = p.scale;
    for (int idx = threadIdx.x; idx < tile; idx += blockDim.x) {
      int l, j;
      tile_coords(p, idx, l, j);
      const long long e = element(p, line0 + l, j) - start_off + amp_offset(p, p.start0 + batch_start);
      const float a = load_amp<AmpT>(p.amp, e);
      res[l * ldl + j] = pointwise_projection<M>(res[l * ldl + j], a, s, acc);
    }
    const double total = block_sum_double(static_cast<double>(acc));
    if (threadIdx.x == 0) {
      Ctrl* c = p.ctrl;
      const int row = c->counters[p.group];
      if (row < c->capacity) {
        atomicAdd(&c->errs[static_cast<long long>(row) * p.starts_total + p.start0 + batch_start],
                  total);
      }
    }
    __syncthreads();
    res = run_stages<true>(p, res, other, ldl);
  } else if constexpr (M == Mode::kUpd) {
    float ca = p.coef_a, cb = p.coef_b;
    if (p.coef_from_ctrl) {
      ca = p.ctrl->a;
      cb = p.ctrl->b;
    }
    for (int idx = threadIdx.x; idx < tile; idx += blockDim.x) {
      int l, j;
      tile_coords(p, idx, l, j);
      const long long g = element(p, line0 + l, j);
      const float2 pv = res[l * ldl + j];
      float2 xn = pv;
      if (!p.support[g]) {
        const float2 xo = p.x[g];
        xn = {ca * xo.x + cb * pv.x, ca * xo.y + cb * pv.y};
      }
      p.x[g] = xn;
      res[l * ldl + j] = xn;
    }
    if (p.bump_counter && blockIdx.x == 0 && threadIdx.x == 0) ++p.ctrl->counters[p.group];
    __syncthreads();
    res = run_stages<false>(p, res, other, ldl);
  } else if constexpr (M == Mode::kBlur || M == Mode::kBlurMag) {
    const float inv_l = 1.0f / static_cast<float>(p.L);
    for (int idx = threadIdx.x; idx < tile; idx += blockDim.x) {
      int l, j;
      tile_coords(p, idx, l, j);
      const float f = fftfreq(static_cast<std::uint32_t>(j), static_cast<std::uint32_t>(p.L));
      const float g = expf(p.blur_k * f * f) * inv_l;
      res[l * ldl + j] = cscale(res[l * ldl + j], g);
    }
    __syncthreads();
    res = run_stages<true>(p, res, other, ldl);
  }

  // ---- store (and the shrinkwrap level of the last blur pass)
  float peak = 0.0f;
  float sq = 0.0f;
  unsigned cnt = 0;
  for (int idx = threadIdx.x; idx < tile; idx += blockDim.x) {
    int l, j;
    tile_coords(p, idx, l, j);
    const long long g = element(p, line0 + l, j);
    const float2 v = res[l * ldl + j];
    p.w[g] = v;
    if constexpr (M == Mode::kBlur || M == Mode::kBlurMag) {
      if (p.level_method == 1) {
        peak = fmaxf(peak, v.x);
      } else if (p.level_method == 2 && p.support[g]) {
        sq += v.x * v.x;
        ++cnt;
      }
    }
  }
  if constexpr (M == Mode::kBlur || M == Mode::kBlurMag) {
    if (p.level_method == 1) {
      peak = warp_max(peak);
      if ((threadIdx.x & 31) == 0) atomicMax(&p.level[batch_start].max_bits, __float_as_int(peak));
    } else if (p.level_method == 2) {
      const double s2 = block_sum_double(static_cast<double>(sq));
      __syncthreads();
      const double c2 = block_sum_double(static_cast<double>(cnt));
      if (threadIdx.x == 0) {
        atomicAdd(&p.level[batch_start].sum, s2);
        atomicAdd(&p.level[batch_start].count, static_cast<unsigned long long>(c2));
      }
    }
  }
}

// Largest dynamic shared memory a line pass asks for (choose_lpc keeps the two
// buffers at or below this).
constexpr int kMaxPassSmem = 2 * 16 * 512 * static_cast<int>(sizeof(float2));

template <class Kernel>
void allow_smem(Kernel kernel) {
  QPB_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxPassSmem));
}

template <Mode M>
void launch_mode(const PassParams& p, cudaStream_t stream) {
  const dim3 grid(static_cast<unsigned>(p.lines / p.lpc));
  const std::size_t smem = 2u * static_cast<std::size_t>(p.lpc) * p.L * sizeof(float2);
  if (smem > static_cast<std::size_t>(kMaxPassSmem)) {
    throw std::logic_error("line pass: shared memory request above the configured maximum");
  }
  auto launch = [&](auto kernel) {
    kernel<<<grid, kThreads, smem, stream>>>(p);
    QPB_CHECK(cudaGetLastError());
    count_launches(1);
  };
  if constexpr (M == Mode::kMod || M == Mode::kGrad) {
    switch (p.amp_storage) {
      case AmpStorage::kF32:
        launch(line_pass_kernel<M, float>);
        break;
      case AmpStorage::kF16:
        launch(line_pass_kernel<M, __half>);
        break;
      case AmpStorage::kBF16:
        launch(line_pass_kernel<M, __nv_bfloat16>);
        break;
    }
  } else {
    launch(line_pass_kernel<M, float>);
  }
}

}  // namespace

void configure_line_passes() {
  // Once per device, outside any stream capture.
  static std::mutex mutex;
  static std::set<int> done;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  if (!done.insert(device).second) return;
  allow_smem(line_pass_kernel<Mode::kFwd, float>);
  allow_smem(line_pass_kernel<Mode::kFwdFromX, float>);
  allow_smem(line_pass_kernel<Mode::kInv, float>);
  allow_smem(line_pass_kernel<Mode::kMod, float>);
  allow_smem(line_pass_kernel<Mode::kMod, __half>);
  allow_smem(line_pass_kernel<Mode::kMod, __nv_bfloat16>);
  allow_smem(line_pass_kernel<Mode::kUpd, float>);
  allow_smem(line_pass_kernel<Mode::kBlur, float>);
  allow_smem(line_pass_kernel<Mode::kBlurMag, float>);
  allow_smem(line_pass_kernel<Mode::kGrad, float>);
  allow_smem(line_pass_kernel<Mode::kGrad, __half>);
  allow_smem(line_pass_kernel<Mode::kGrad, __nv_bfloat16>);
  configure_fast_passes();
  configure_column_passes();
}

int choose_lpc(int L, int S, int lines_per_start) {
  // About 2048 elements per CTA (32 KiB for the two buffers), at least one line,
  // and a power of two dividing lines_per_start so a CTA never spans two starts.
  int target = std::max(1, 2048 / std::max(L, 1));
  if (S > 1) target = std::max(target, std::min(16, 8192 / std::max(L, 1)));
  int lpc = 1;
  while (lpc * 2 <= target && lines_per_start % (lpc * 2) == 0) lpc *= 2;
  return lpc;
}

void launch_line_pass(Mode mode, const PassParams& p, cudaStream_t stream) {
  // a modulus pass follows the amplitude's layout, which the solver chose
  // with column_pass_preferred (or for the persistent schedule's column tiles)
  if (mode == Mode::kMod ? column_pass_lines(p, mode) > 0 : column_pass_preferred(p, mode)) {
    return launch_column_pass(mode, p, stream);
  }
  if (p.amp_tiled == kAmpTiledLines) {
    throw std::logic_error("line pass: a line-major tiled amplitude needs the column pass");
  }
  if (fast_passes_enabled() && fast_pass_supports(p)) return launch_fast_pass(mode, p, stream);
  const bool touches_x = mode == Mode::kFwdFromX || mode == Mode::kUpd || mode == Mode::kBlurMag;
  if (p.wave_half || (touches_x && p.iter_half)) {
    throw std::logic_error("line pass: fp16 storage needs the register-resident or column pass");
  }
  if (p.amp_tiled) throw std::logic_error("line pass: tiled amplitude needs the register-resident pass");
  if (p.lines % p.lpc != 0 || p.lines_per_start % p.lpc != 0) {
    throw std::logic_error("line pass: lines per CTA must divide the lines of a start");
  }
  switch (mode) {
    case Mode::kFwd:
      return launch_mode<Mode::kFwd>(p, stream);
    case Mode::kFwdFromX:
      return launch_mode<Mode::kFwdFromX>(p, stream);
    case Mode::kInv:
      return launch_mode<Mode::kInv>(p, stream);
    case Mode::kMod:
      return launch_mode<Mode::kMod>(p, stream);
    case Mode::kUpd:
      return launch_mode<Mode::kUpd>(p, stream);
    case Mode::kBlur:
      return launch_mode<Mode::kBlur>(p, stream);
    case Mode::kBlurMag:
      return launch_mode<Mode::kBlurMag>(p, stream);
    case Mode::kGrad:
      return launch_mode<Mode::kGrad>(p, stream);
  }
}

}  // namespace qpb
