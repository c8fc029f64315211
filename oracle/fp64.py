"""FP64 oracle: a numpy restatement of QoraPhaseCU's CPU reconstruction path.

TEST INFRASTRUCTURE. Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline. The product
(``qoraphasecu_b200``) never calls it.

Every function restates the reference file and line it cites (paths are
relative to the QoraPhaseCU project root). Arithmetic is complex128/float64
except where the reference itself rounds to float32 in a way that changes
results bit for bit (the random phase, the update coefficients, the amplitude
and the shrinkwrap cut), which is reproduced in float32.

Arrays are FFT order inside the solver and centre-origin outside, as in the
reference (``src/core/layout.hpp:90-100``). Recipes are lists of the 7-tuples
``(kind, n, beta, threshold, sigma, method, axis)`` that the reference's Python
layer hands its FFI (``python/qoraphasecu/recipe.py:11-12``,
``python/bindings.cpp:22-23``).

``dtype=np.complex64`` with ``fft="scipy"`` turns the solver into the timed CPU
port: the same loop in float32 with scipy.fft (pocketfft C++) on all host cores,
the closest available stand-in for the reference's pocketfft + OpenMP path.
"""

from __future__ import annotations

import math
import os

import numpy as np

# src/core/pointwise.hpp:16-17
K_EPS = float(np.float32(1e-12))
K_TWO_PI = np.float32(6.28318530717958647692)

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


# ----------------------------------------------------------------------------- RNG
def mix64(z):
    """splitmix64 finaliser, src/core/pointwise.hpp:19-24 (uint64 wrap-around)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, start: int, index) -> np.ndarray:
    """Counter-based uniform in [0, 1) as float32, src/core/pointwise.hpp:29-32."""
    seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
    key = mix64(seed ^ mix64(np.uint64(start + 1)))
    idx = np.asarray(index, dtype=np.uint64)
    with np.errstate(over="ignore"):
        bits = mix64(key + idx) >> np.uint64(40)
    return bits.astype(np.float32) * np.float32(2.0**-24)


# ----------------------------------------------------------------- coefficients
def er_coefficients():
    """src/core/pointwise.hpp:41."""
    return np.float32(0.0), np.float32(0.0)


def hio_coefficients(beta):
    """src/core/pointwise.hpp:42."""
    return np.float32(1.0), -np.float32(beta)


def raar_coefficients(beta):
    """src/core/pointwise.hpp:45: (beta, 1 - 2 beta) evaluated in float32."""
    b = np.float32(beta)
    return b, np.float32(np.float32(1.0) - np.float32(2.0) * b)


def fftfreq(n: int) -> np.ndarray:
    """Signed frequency of every FFT-order index, float32, src/core/pointwise.hpp:48-51."""
    k = np.arange(n)
    s = np.where(k < (n + 1) // 2, k, k - n)
    return (s.astype(np.float32) / np.float32(n)).astype(np.float32)


# ----------------------------------------------------------------------- layout
def to_fft_order(a: np.ndarray) -> np.ndarray:
    """numpy ifftshift over every axis, src/core/layout.hpp:71-94."""
    return np.fft.ifftshift(a)


def to_centered(a: np.ndarray) -> np.ndarray:
    """numpy fftshift over every axis, src/core/layout.hpp:96-100."""
    return np.fft.fftshift(a)


# ----------------------------------------------------------------------- FFT
class Fft:
    """Unitary n-D C2C on FFT-order data, src/cpu/fft.hpp:11-24 and fft.cpp:12-35.

    The reference calls pocketfft (mreineck/pocketfft, branch ``cpp``, commit
    4d865cba24359b05b37da4e75aee24498c3b78e7, fetched by CMakeLists.txt:41-47
    and not vendored) with scale 1/sqrt(N) in both directions. Here the same
    transform is numpy.fft (complex128) or scipy.fft with ``workers``.
    """

    def __init__(self, ndim: int, backend: str = "numpy", workers: int | None = None):
        self.axes = tuple(range(-ndim, 0))
        self.backend = backend
        self.workers = workers or len(os.sched_getaffinity(0))
        if backend == "scipy":
            import scipy.fft as sfft

            self._sfft = sfft

    def forward(self, a):
        if self.backend == "scipy":
            return self._sfft.fftn(a, axes=self.axes, norm="ortho", workers=self.workers)
        return np.fft.fftn(a, axes=self.axes, norm="ortho")

    def inverse(self, a):
        if self.backend == "scipy":
            return self._sfft.ifftn(a, axes=self.axes, norm="ortho", workers=self.workers)
        return np.fft.ifftn(a, axes=self.axes, norm="ortho")


# --------------------------------------------------------------------- problem
class Problem:
    """src/core/problem.hpp:26-31: centre-origin amplitude (float32), mask, support."""

    def __init__(self, shape, amplitude, mask, support):
        self.shape = tuple(shape)
        self.amplitude = amplitude
        self.mask = mask
        self.support = support


def _check_shape(shape):
    """src/core/problem.cpp:21-28."""
    if len(shape) not in (2, 3):
        raise ValueError(f"shape must be 2D or 3D, got ndim={len(shape)}")
    if any(n == 0 for n in shape):
        raise ValueError("shape has a zero-length axis")


def make_problem(intensity, support=None, mask=None, support_threshold=0.1) -> Problem:
    """src/core/problem.cpp:40-70."""
    intensity = np.ascontiguousarray(intensity, dtype=np.float32)
    shape = intensity.shape
    _check_shape(shape)
    if not np.all(np.isfinite(intensity)):
        raise ValueError("intensity contains NaN or Inf")
    if mask is not None:
        mask = np.asarray(mask).reshape(shape)
        if np.all(mask != 0):
            raise ValueError("mask marks every pixel as bad; nothing left to fit")
    amplitude = np.sqrt(np.maximum(intensity, np.float32(0.0))).astype(np.float32)
    mask = np.zeros(shape, np.uint8) if mask is None else (mask != 0).astype(np.uint8)
    if support is None:
        support = autocorrelation_support(intensity, support_threshold)
    support = (np.asarray(support).reshape(shape) != 0).astype(np.uint8)
    return Problem(shape, amplitude, mask, support)


def autocorrelation_support(intensity, threshold=0.1) -> np.ndarray:
    """|IFFT(intensity)| > threshold * max, centre-origin, src/core/problem.cpp:72-88."""
    intensity = np.asarray(intensity, dtype=np.float32)
    _check_shape(intensity.shape)
    buf = to_fft_order(intensity).astype(np.complex128)
    ac = np.abs(Fft(intensity.ndim).inverse(buf))
    centered = to_centered(ac)
    level = float(np.float32(threshold) * np.float32(centered.max()))
    return (centered > level).astype(np.uint8)


def simulate_intensity(obj) -> np.ndarray:
    """|centred unitary FFT(obj)|^2 as float32, src/core/problem.cpp:90-99."""
    obj = np.asarray(obj, dtype=np.complex128)
    _check_shape(obj.shape)
    wave = Fft(obj.ndim).forward(to_fft_order(obj))
    return (np.abs(to_centered(wave)) ** 2).astype(np.float32)


def half_support(support, axis=0) -> np.ndarray:
    """Keep the support below its centre of mass along ``axis``, src/core/problem.cpp:101-127.

    ``support`` is centre-origin; the coordinate is the array index along the axis.
    """
    support = np.asarray(support) != 0
    if axis < 0 or axis >= support.ndim:
        raise ValueError("detwin axis out of range")
    n = support.shape[axis]
    shape = [1] * support.ndim
    shape[axis] = n
    coord = np.arange(n, dtype=np.float64).reshape(shape)
    weight = float(support.sum())
    moment = float((support * coord).sum())
    centre = moment / max(weight, 1.0)
    return (support & (coord < centre)).astype(np.uint8)


# ------------------------------------------------------------------- CPU kernels
def usable_energy(amplitude_fft, mask_fft) -> float:
    """src/cpu/kernels.cpp:16-23."""
    a = amplitude_fft.astype(np.float64)
    return float(np.sum(np.where(mask_fft != 0, 0.0, a * a)))


def modulus(wave, amplitude_fft, mask_fft, energy):
    """In place on the unitary forward transform; returns the Fourier error.

    src/cpu/kernels.cpp:25-42. ``wave`` may carry a leading start axis.
    Masked pixels are scaled by mag / (mag + eps), not left exactly alone.
    """
    mag = np.abs(wave)
    usable = mask_fft == 0
    amp = amplitude_fft.astype(mag.dtype)
    d = np.where(usable, mag - amp, 0.0)
    axes = tuple(range(-amplitude_fft.ndim, 0))
    num = np.sum(d.astype(np.float64) ** 2, axis=axes)
    target = np.where(usable, amp, mag)
    wave *= (target / (mag + mag.dtype.type(K_EPS))).astype(mag.dtype)
    err = np.sqrt(num / (energy + K_EPS))
    return err.astype(np.float32)


def update(x, projected, support, coefficients):
    """x <- S ? P : a x + b P, src/cpu/kernels.cpp:44-50."""
    a, b = coefficients
    real = x.real.dtype.type
    outside = real(a) * x + real(b) * projected
    x[...] = np.where(support != 0, projected, outside)


def blur(image, sigma, fft: Fft | None = None):
    """Gaussian blur by the FFT, transfer exp(k f^2), src/cpu/kernels.cpp:52-75.

    ``image`` may carry a leading start axis; the blur acts on the trailing
    ``fft`` axes. k = -2 (pi sigma)^2 is formed in float32 as in the reference.
    """
    ndim = len(fft.axes) if fft else image.ndim
    fft = fft or Fft(ndim)
    half = np.float32(K_TWO_PI / np.float32(2))
    k = np.float32(np.float32(-2.0) * half * half * np.float32(sigma) * np.float32(sigma))
    shape = image.shape[-ndim:]
    f2 = np.zeros(shape, np.float64)
    for ax, n in enumerate(shape):
        f = fftfreq(n).astype(np.float64)
        view = [1] * ndim
        view[ax] = n
        f2 = f2 + (f * f).reshape(view)
    transfer = np.exp(float(k) * f2)
    buf = fft.forward(image.astype(np.complex128 if fft.backend == "numpy" else np.complex64))
    buf = buf * transfer.astype(buf.real.dtype)
    return fft.inverse(buf).real


def shrinkwrap_level(blurred, support, method):
    """max of the blurred magnitude, or its rms inside the support, src/cpu/kernels.cpp:84-95."""
    if method == "max":
        return np.float32(blurred.max())
    inside = support != 0
    total = float(np.sum(np.where(inside, blurred.astype(np.float64) ** 2, 0.0)))
    count = float(inside.sum())
    return np.float32(math.sqrt(total / max(count, 1.0)))


def shrinkwrap(x, threshold, sigma, method, support, fft: Fft | None = None):
    """New support = blur(|x|) > threshold * level, src/cpu/kernels.cpp:77-102."""
    fft = fft or Fft(x.ndim)
    blurred = blur(np.abs(x), sigma, fft)
    level = shrinkwrap_level(blurred, support, method)
    cut = np.float32(np.float32(threshold) * level)
    return (blurred > float(cut)).astype(np.uint8), blurred, cut


def random_phases(shape_fft, seed, start):
    """kTwoPi * uniform(seed, start, i) in float32 for every FFT-order index."""
    n = int(np.prod(shape_fft))
    u = uniform(seed, start, np.arange(n, dtype=np.uint64))
    return (K_TWO_PI * u).astype(np.float32).reshape(shape_fft)


def random_start(amplitude_fft, support_fft, seed, start, fft: Fft, dtype=np.complex128):
    """A e^{i 2 pi u}, unitary inverse FFT, cut to the support; src/cpu/kernels.cpp:104-117."""
    phase = random_phases(amplitude_fft.shape, seed, start).astype(np.float64)
    x = amplitude_fft.astype(np.float64) * (np.cos(phase) + 1j * np.sin(phase))
    x = fft.inverse(x.astype(dtype))
    x[support_fft == 0] = 0
    return x.astype(dtype)


# ---------------------------------------------------------------------- recipe
def op(kind, n=0, beta=0.0, threshold=0.0, sigma=0.0, method="max", axis=0):
    """One recipe operation tuple, python/qoraphasecu/recipe.py:11-12."""
    return (kind, n, beta, threshold, sigma, method, axis)


def default_recipe():
    """RAAR(50), detwin(HIO(20)), RAAR(50), repeat(8, RAAR(50), Shrinkwrap()), ER(200).

    src/core/recipe.cpp:26-28.
    """
    ops = [op("raar", 50, 0.9), op("detwin_begin"), op("hio", 20, 0.9), op("detwin_end"),
           op("raar", 50, 0.9)]
    for _ in range(8):
        ops += [op("raar", 50, 0.9), op("shrinkwrap", threshold=0.3, sigma=1.0, method="max")]
    ops.append(op("er", 200))
    return ops


def iterations(ops) -> int:
    """src/core/recipe.cpp:16-24."""
    return sum(o[1] for o in ops if o[0] in ("er", "hio", "raar"))


def validate(ops):
    """src/core/recipe.cpp:30-61 (ValueError for std::invalid_argument)."""
    if not ops:
        raise ValueError("recipe is empty")
    in_detwin = False
    for kind, n, _beta, threshold, sigma, _method, _axis in ops:
        if kind in ("er", "hio", "raar"):
            if n < 1:
                raise ValueError(f"{kind.upper()} needs n >= 1")
        elif kind == "shrinkwrap":
            if not (threshold > 0.0) or not (sigma >= 0.0):
                raise ValueError("Shrinkwrap needs threshold > 0, sigma >= 0")
        elif kind == "detwin_begin":
            if in_detwin:
                raise ValueError("nested detwin")
            in_detwin = True
        elif kind == "detwin_end":
            if not in_detwin:
                raise ValueError("DetwinEnd without DetwinBegin")
            in_detwin = False
        else:
            raise ValueError(f"unknown recipe operation '{kind}'")
    if in_detwin:
        raise ValueError("DetwinBegin without DetwinEnd")


# ---------------------------------------------------------------------- solver
class Solver:
    """CpuSolver, src/cpu/cpu_solver.cpp:18-110, with every start held in one array.

    ``start`` (centre-origin objects, one per start) replaces the random phases
    and is cut to the support (:32-41). ``run`` continues from the current
    state and appends errors; ``results`` returns centre-origin objects.
    """

    def __init__(self, problem: Problem, starts=1, seed=0, start=None, sync_every=10,
                 progress=None, dtype=np.complex128, fft="numpy", workers=None):
        if starts < 1:
            raise ValueError("starts must be >= 1")
        if sync_every < 1:
            raise ValueError("sync_every must be >= 1")
        self.shape = problem.shape
        self.dtype = np.dtype(dtype)
        self.fft = Fft(len(self.shape), fft, workers)
        self.amplitude = to_fft_order(problem.amplitude)
        self.mask = to_fft_order(problem.mask)
        self.energy = usable_energy(self.amplitude, self.mask)
        support = to_fft_order(problem.support)
        self.support = np.stack([support] * starts)
        self.saved = None
        self.errors = [[] for _ in range(starts)]
        self.sync_every = sync_every
        self.progress = progress
        self.iteration = 0
        if start is None:
            self.x = np.stack([random_start(self.amplitude, support, seed, s, self.fft, self.dtype)
                               for s in range(starts)])
        else:
            start = np.asarray(start, dtype=np.complex64).reshape((starts, *self.shape))
            axes = tuple(range(1, 1 + len(self.shape)))
            self.x = np.fft.ifftshift(start, axes=axes).astype(self.dtype)
            self.x[self.support == 0] = 0

    def run(self, ops):
        validate(ops)
        for kind, n, beta, threshold, sigma, method, axis in ops:
            if kind == "er":
                self.iterate(n, er_coefficients())
            elif kind == "hio":
                self.iterate(n, hio_coefficients(beta))
            elif kind == "raar":
                self.iterate(n, raar_coefficients(beta))
            elif kind == "shrinkwrap":
                for s in range(len(self.x)):
                    self.support[s] = shrinkwrap(self.x[s], threshold, sigma, method,
                                                 self.support[s], self.fft)[0]
            elif kind == "detwin_begin":
                self.saved = self.support.copy()
                for s in range(len(self.x)):
                    half = half_support(to_centered(self.support[s]), axis)
                    self.support[s] = to_fft_order(half)
            elif kind == "detwin_end":
                self.support = self.saved

    def iterate(self, n, coefficients):
        """src/cpu/cpu_solver.cpp:82-93, all starts at once."""
        for _ in range(n):
            wave = self.fft.forward(self.x)
            errs = modulus(wave, self.amplitude, self.mask, self.energy)
            wave = self.fft.inverse(wave)
            update(self.x, wave.astype(self.dtype), self.support, coefficients)
            for s, e in enumerate(np.atleast_1d(errs)):
                self.errors[s].append(float(e))
            self.iteration += 1
            if self.progress and self.iteration % self.sync_every == 0:
                self.progress(self.iteration, [e[-1] for e in self.errors])

    def results(self):
        axes = tuple(range(1, 1 + len(self.shape)))
        obj = np.fft.fftshift(self.x, axes=axes).astype(np.complex64)
        sup = np.fft.fftshift(self.support, axes=axes).astype(bool)
        return [(obj[s], sup[s], np.asarray(self.errors[s], np.float32)) for s in range(len(obj))]


def reconstruct(problem: Problem, ops=None, **options):
    """src/core/solver.cpp:88-93."""
    solver = Solver(problem, **options)
    solver.run(default_recipe() if ops is None else ops)
    return solver.results()


# ---------------------------------------------------------------- operators
def modulus_project(problem: Problem, obj):
    """P_M of a centre-origin object and the Fourier error of the input, src/cpu/operators.cpp:11-24."""
    fft = Fft(len(problem.shape))
    amp = to_fft_order(problem.amplitude)
    mask = to_fft_order(problem.mask)
    x = fft.forward(to_fft_order(np.asarray(obj, np.complex128)))
    err = modulus(x, amp, mask, usable_energy(amp, mask))
    return to_centered(fft.inverse(x)), float(err)


def support_project(support, obj):
    """src/cpu/operators.cpp:26-31."""
    out = np.array(obj, copy=True)
    out[np.asarray(support) == 0] = 0
    return out


def gaussian_blur(image, sigma):
    """src/cpu/operators.cpp:33-39 (a circular blur commutes with the fftshift roll)."""
    image = np.asarray(image, np.float64)
    return blur(image, sigma, Fft(image.ndim))


# ----------------------------------------------------------------- metrics
def _translated_error(b, ref, fft):
    """src/core/metrics.cpp:17-59."""
    fr = fft.forward(ref)
    fb = fft.forward(b)
    cc = fft.inverse(fr * np.conj(fb))
    peak = int(np.argmax(np.abs(cc) ** 2))
    shift = np.unravel_index(peak, b.shape)
    shifted = np.roll(b, shift, axis=tuple(range(b.ndim)))
    overlap = np.sum(ref * np.conj(shifted))
    ref_norm = float(np.sum(np.abs(ref) ** 2))
    rotation = overlap / abs(overlap) if abs(overlap) > 0 else 1.0
    diff = float(np.sum(np.abs(rotation * shifted - ref) ** 2))
    return math.sqrt(diff / max(ref_norm, np.finfo(np.float64).tiny))


def aligned_error(a, reference) -> float:
    """||a - ref|| / ||ref|| after shift, conjugate flip and global phase; src/core/metrics.cpp:63-86."""
    a = np.asarray(a, np.complex128)
    reference = np.asarray(reference, np.complex128)
    if a.shape != reference.shape:
        raise ValueError("arrays do not match shape")
    fft = Fft(a.ndim)
    twin = np.conj(np.flip(a, axis=tuple(range(a.ndim))))
    twin = np.roll(twin, 1, axis=tuple(range(a.ndim)))
    return min(_translated_error(a, reference, fft), _translated_error(twin, reference, fft))


def relative_diff(a, b) -> float:
    """||a - b|| / ||b||, tests/test_cuda.cpp:15-23."""
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))
