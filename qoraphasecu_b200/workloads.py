"""Seeded synthetic inputs with the shapes and statistics of the benchmark configs.

No public dataset is involved: every object is generated here from
``numpy.random.default_rng(seed)`` and its intensity is ``|centred unitary
FFT|^2`` (QoraPhaseCU's ``simulate_intensity``, src/core/problem.cpp:90-99),
optionally with Poisson counts. Input generation runs on the host with numpy;
it is not part of the reconstruction path.

* ``square``: amplitude U[0,1] and phase U[-pi,pi) inside a centred square of
  side 24/64 of the field (the small CPU case, and the per-problem generator
  of the uneven batch).
* ``gaussians``: amplitude a sum of 5 Gaussians (sigma U[3,10] px) clipped to
  a disk of radius 60/256 of the field; phase a random linear ramp plus a
  Gaussian-filtered (sigma 6 px) normal field with std 1 rad; Poisson counts
  at a peak of 1e6 photons and a centred beamstop of radius 8 px.
* ``crystal``: 3D faceted convex crystal (12 random half-spaces inside a
  sphere of radius 40/128 of the field), displacement-field phase.
"""

from __future__ import annotations

import numpy as np

from .recipe import ER, RAAR, HIO, Recipe, Shrinkwrap, repeat


def centred_coords(shape):
    """Coordinates with index n // 2 at 0 along every axis."""
    return np.meshgrid(*[np.arange(n) - n // 2 for n in shape], indexing="ij")


def simulate_intensity(obj) -> np.ndarray:
    """|centred unitary FFT(obj)|^2 as float32."""
    wave = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(obj), norm="ortho"))
    return (np.abs(wave) ** 2).astype(np.float32)


def gaussian_filter(field, sigma):
    """Periodic Gaussian filter by the FFT."""
    f2 = sum(np.fft.fftfreq(n)[tuple(slice(None) if a == i else None for a in range(field.ndim))] ** 2
             for i, n in enumerate(field.shape))
    return np.fft.ifftn(np.fft.fftn(field) * np.exp(-2 * (np.pi * sigma) ** 2 * f2)).real


def poisson(intensity, peak, rng):
    scaled = intensity / max(float(intensity.max()), 1e-30) * peak
    return rng.poisson(scaled).astype(np.float32)


def beamstop(shape, radius):
    coords = centred_coords(shape)
    return sum(c.astype(np.float64) ** 2 for c in coords) <= radius**2


def square(n=64, seed=0, ndim=2):
    """Square object: uniform amplitude and phase inside a centred square."""
    rng = np.random.default_rng(seed)
    m = max(1, round(24 * n / 64))
    shape = (n,) * ndim
    obj = np.zeros(shape, np.complex64)
    lo = n // 2 - m // 2
    box = tuple(slice(lo, lo + m) for _ in range(ndim))
    amp = rng.random((m,) * ndim)
    phase = rng.uniform(-np.pi, np.pi, (m,) * ndim)
    obj[box] = (amp * np.exp(1j * phase)).astype(np.complex64)
    return obj


def gaussians(n=256, seed=1000, peak=1e6, stop=8.0):
    """Five Gaussian blobs with a smooth phase, Poisson counts, beamstop: returns (object, intensity, mask)."""
    rng = np.random.default_rng(seed)
    y, x = centred_coords((n, n))
    scale = n / 256
    amp = np.zeros((n, n))
    for _ in range(5):
        r = 40 * scale * np.sqrt(rng.random())
        t = 2 * np.pi * rng.random()
        cy, cx = r * np.sin(t), r * np.cos(t)
        sigma = rng.uniform(3, 10) * scale
        amp += rng.uniform(0.5, 1.0) * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * sigma**2))
    disk = y.astype(float) ** 2 + x.astype(float) ** 2 <= (60 * scale) ** 2
    amp *= disk
    ramp = rng.uniform(-1, 1, 2) * np.pi / (16 * scale)
    noise = gaussian_filter(rng.standard_normal((n, n)), 6 * scale)
    noise /= noise.std()
    phase = ramp[0] * y + ramp[1] * x + noise
    obj = (amp * np.exp(1j * phase)).astype(np.complex64)
    intensity = poisson(simulate_intensity(obj), peak, rng)
    return obj, intensity, beamstop((n, n), stop * scale)


def gaussians_recipe() -> Recipe:
    """repeat(10, RAAR(50, 0.9), Shrinkwrap(threshold 0.3, sigma 1.0)), ER(200): 700 iterations."""
    return Recipe(repeat(10, RAAR(50, 0.9), Shrinkwrap(0.3, 1.0)), ER(200))


def uneven_batch(count=64, seed=2000, sizes=(64, 128, 256, 512), peak=1e6):
    """Uneven batch: sides uniform over ``sizes``, square objects, beamstop n/32."""
    rng = np.random.default_rng(seed)
    problems = []
    for k in range(count):
        n = int(rng.choice(sizes))
        obj = square(n, seed + 1 + k)
        intensity = poisson(simulate_intensity(obj), peak, rng)
        problems.append((obj, intensity, beamstop((n, n), n / 32)))
    return problems


def uneven_recipe() -> Recipe:
    """repeat(4, HIO(50), Shrinkwrap(rms, threshold 0.3)), ER(100): 300 iterations."""
    return Recipe(repeat(4, HIO(50), Shrinkwrap(0.3, 1.0, "rms")), ER(100))


def crystal(n=128, seed=3000, peak=1e7):
    """3D Bragg-like crystal object: returns (object, intensity)."""
    rng = np.random.default_rng(seed)
    z, y, x = centred_coords((n, n, n))
    scale = n / 128
    r = np.stack([z, y, x]).astype(np.float64)
    inside = (r**2).sum(0) <= (40 * scale) ** 2
    for _ in range(12):
        normal = rng.standard_normal(3)
        normal /= np.linalg.norm(normal)
        offset = rng.uniform(20, 36) * scale
        inside &= np.tensordot(normal, r, axes=1) <= offset
    u = np.zeros((3, n, n, n))
    for _ in range(3):
        c = rng.uniform(-20, 20, 3) * scale
        sigma = rng.uniform(5, 15) * scale
        blob = np.exp(-((r - c[:, None, None, None]) ** 2).sum(0) / (2 * sigma**2))
        u += rng.standard_normal(3)[:, None, None, None] * blob
    q = rng.standard_normal(3)
    q /= np.linalg.norm(q)
    phase = 2.0 * np.tensordot(q, u, axes=1)
    obj = (inside * np.exp(1j * phase)).astype(np.complex64)
    intensity = poisson(simulate_intensity(obj), peak, rng)
    return obj, intensity


def hio_recipe(n=50) -> Recipe:
    return Recipe(HIO(n))
