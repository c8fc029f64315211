// TEST INFRASTRUCTURE (oracle). The FFT that the compiled reference oracle
// links in place of src/cpu/fft.cpp.
//
// QoraPhaseCU's CPU FFT (src/cpu/fft.cpp:12-35) calls pocketfft
// (mreineck/pocketfft, branch `cpp`, commit 4d865cba24359b05b37da4e75aee24498c3b78e7,
// fetched by CMakeLists.txt:41-47 and not vendored), which is absent here. This
// file implements the same class, qpcu::cpu::Fft (src/cpu/fft.hpp:11-24): an
// unnormalised mixed-radix C2C transform over every axis of a row-major array,
// scaled by 1/sqrt(N) in both directions, in float arithmetic with twiddles
// computed in double (the precision class of pocketfft's float transforms),
// parallel over the lines of each axis.

#include "fft.hpp"

#include <sched.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace qpcu::cpu {

namespace {

using C = std::complex<float>;

struct Plan {
  std::size_t n = 1;
  std::vector<int> radices;
  std::vector<C> twiddle;  // exp(-2 pi i k / n)
};

const Plan& plan_for(std::size_t n) {
  static std::mutex mutex;
  static std::map<std::size_t, std::unique_ptr<Plan>> cache;
  std::lock_guard<std::mutex> lock(mutex);
  auto& slot = cache[n];
  if (slot) return *slot;
  auto p = std::make_unique<Plan>();
  p->n = n;
  std::size_t rest = n;
  while (rest % 4 == 0) {
    p->radices.push_back(4);
    rest /= 4;
  }
  if (rest % 2 == 0) {
    p->radices.push_back(2);
    rest /= 2;
  }
  for (std::size_t f = 3; rest > 1; f += 2) {
    while (rest % f == 0) {
      p->radices.push_back(static_cast<int>(f));
      rest /= f;
    }
  }
  p->twiddle.resize(n);
  for (std::size_t k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * static_cast<double>(k) / static_cast<double>(n);
    p->twiddle[k] = C(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  slot = std::move(p);
  return *slot;
}

// Stockham autosort: stage with radix R reads src[j + q m] (m = n / R),
// multiplies input q by W_{Ns R}^{q (j mod Ns)}, takes an R-point DFT and
// writes dst[(j / Ns) Ns R + (j mod Ns) + r Ns]. Result in `a` on return.
void transform(const Plan& p, C* a, C* b, bool forward) {
  const std::size_t n = p.n;
  std::size_t ns = 1;
  C* src = a;
  C* dst = b;
  C v[64];
  std::vector<C> big;
  for (int radix : p.radices) {
    const std::size_t r = static_cast<std::size_t>(radix);
    const std::size_t m = n / r;
    const std::size_t step = n / (ns * r);
    C* vals = v;
    if (r > 64) {
      big.resize(r);
      vals = big.data();
    }
    for (std::size_t j = 0; j < m; ++j) {
      const std::size_t k = j % ns;
      for (std::size_t q = 0; q < r; ++q) {
        C w = p.twiddle[(q * k * step) % n];
        if (!forward) w = std::conj(w);
        vals[q] = src[j + q * m] * w;
      }
      const std::size_t out = (j - k) * r + k;
      if (r == 2) {
        dst[out] = vals[0] + vals[1];
        dst[out + ns] = vals[0] - vals[1];
      } else if (r == 4) {
        const C t0 = vals[0] + vals[2], t1 = vals[0] - vals[2];
        const C t2 = vals[1] + vals[3];
        const C d = vals[1] - vals[3];
        const C t3 = forward ? C(d.imag(), -d.real()) : C(-d.imag(), d.real());
        dst[out] = t0 + t2;
        dst[out + ns] = t1 + t3;
        dst[out + 2 * ns] = t0 - t2;
        dst[out + 3 * ns] = t1 - t3;
      } else {
        const std::size_t wr = n / r;
        for (std::size_t s = 0; s < r; ++s) {
          C acc(0.0f, 0.0f);
          for (std::size_t q = 0; q < r; ++q) {
            C w = p.twiddle[((q * s) % r) * wr];
            if (!forward) w = std::conj(w);
            acc += vals[q] * w;
          }
          dst[out + s * ns] = acc;
        }
      }
    }
    ns *= r;
    std::swap(src, dst);
  }
  if (src != a) std::copy(src, src + n, a);
}

std::size_t usable_threads(std::size_t requested) {
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) {
    requested = std::min<std::size_t>(requested, static_cast<std::size_t>(CPU_COUNT(&set)));
  }
  return std::max<std::size_t>(requested, 1);
}

}  // namespace

Fft::Fft(const Shape& shape)
    : shape_(shape),
      scale_(1.0f / std::sqrt(static_cast<float>(numel(shape)))),
      threads_(usable_threads(std::max(1u, std::thread::hardware_concurrency()))) {}

void Fft::forward(std::span<const Complex> in, std::span<Complex> out) const {
  exec(in, out, true);
}

void Fft::inverse(std::span<const Complex> in, std::span<Complex> out) const {
  exec(in, out, false);
}

void Fft::exec(std::span<const Complex> in, std::span<Complex> out, bool forward) const {
  const std::size_t total = in.size();
  if (out.data() != in.data()) std::copy(in.begin(), in.end(), out.begin());
  const std::size_t nd = shape_.size();
  for (std::size_t axis = 0; axis < nd; ++axis) {
    const std::size_t len = shape_[axis];
    std::size_t stride = 1;
    for (std::size_t a = axis + 1; a < nd; ++a) stride *= shape_[a];
    const std::size_t lines = total / len;
    const bool last = axis + 1 == nd;
    const Plan& plan = plan_for(len);
    const float scale = scale_;
    C* data = out.data();
#pragma omp parallel num_threads(static_cast<int>(threads_))
    {
      std::vector<C> line(len), work(len);
#pragma omp for schedule(static)
      for (std::ptrdiff_t l = 0; l < static_cast<std::ptrdiff_t>(lines); ++l) {
        const std::size_t outer = static_cast<std::size_t>(l) / stride;
        const std::size_t inner = static_cast<std::size_t>(l) % stride;
        C* base = data + outer * len * stride + inner;
        for (std::size_t j = 0; j < len; ++j) line[j] = base[j * stride];
        transform(plan, line.data(), work.data(), forward);
        if (last) {
          for (std::size_t j = 0; j < len; ++j) base[j * stride] = line[j] * scale;
        } else {
          for (std::size_t j = 0; j < len; ++j) base[j * stride] = line[j];
        }
      }
    }
  }
}

}  // namespace qpcu::cpu
