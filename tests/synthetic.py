"""Synthetic objects of the reference's test suite (tests/synthetic.hpp) and
the README-figure triangle (python/tests/conftest.py:7-18)."""

from __future__ import annotations

import numpy as np

from oracle import fp64


def triangle(shape, m):
    """Right triangle of side m with an amplitude dip and a phase bump, in a box
    centred at n/2 - m/2 on every axis; 3D stacks it over m slices with a z
    phase (tests/synthetic.hpp:18-50). Returns (object, support, intensity)."""
    shape = tuple(shape)
    is3d = len(shape) == 3
    d = (1, *shape) if not is3d else shape
    z, y, x = np.meshgrid(np.arange(d[0]), np.arange(d[1]), np.arange(d[2]), indexing="ij")
    lz = z - (d[0] // 2 - m // 2)
    ly = y - (d[1] // 2 - m // 2)
    lx = x - (d[2] // 2 - m // 2)
    c = (m - 1) / 2.0
    in_box = (ly >= 0) & (ly < m) & (lx >= 0) & (lx < m)
    if is3d:
        in_box &= (lz >= 0) & (lz < m)
    inside = in_box & (ly + lx < m)
    ry, rx = ly - c, lx - c
    amp = 1.0 - 0.5 * np.exp(-(rx * rx + ry * ry) / 20.0)
    phase = 1.2 * np.exp(-((rx + 4) ** 2 + (ry + 4) ** 2) / 30.0)
    if is3d:
        phase = phase + 0.3 * (lz - c) / m
    amp32 = amp.astype(np.float32)
    ph32 = phase.astype(np.float32)
    obj = np.where(inside, amp32 * (np.cos(ph32) + 1j * np.sin(ph32)), 0).astype(np.complex64)
    obj = obj.reshape(shape)
    support = inside.reshape(shape).astype(np.uint8)
    return obj, support, fp64.simulate_intensity(obj)


def corner(n, m):
    """The 3D triangle with the corner x + y + z >= 1.5 m (box-relative) cut off
    (tests/synthetic.hpp:52-72)."""
    obj, support, _ = triangle((n, n, n), m)
    lo = n // 2 - m // 2
    z, y, x = np.indices((n, n, n))
    cut = (z + y + x) - 3 * lo >= 1.5 * m
    obj = np.where(cut, 0, obj).astype(np.complex64)
    support = np.where(cut, 0, support).astype(np.uint8)
    return obj, support, fp64.simulate_intensity(obj)


def random_field(n, seed):
    """LCG complex field in [-0.5, 0.5) (tests/synthetic.hpp:74-83)."""
    state = (seed * 2654435761 + 1) & 0xFFFFFFFF
    out = np.empty(2 * n, np.float32)
    for i in range(2 * n):
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = np.float32(state >> 8) / np.float32(16777216.0) - np.float32(0.5)
    return out.view(np.complex64)


def readme_triangle(n=64, m=24):
    """The QoraPhase README object (python/tests/conftest.py:7-18)."""
    y, x = np.indices((m, m)) - (m - 1) / 2
    inside = np.indices((m, m)).sum(0) < m
    block = (1 - 0.5 * np.exp(-(x**2 + y**2) / 20)) * np.exp(
        1j * 1.2 * np.exp(-((x + 4) ** 2 + (y + 4) ** 2) / 30)
    )
    obj = np.zeros((n, n), np.complex64)
    obj[n // 2 - m // 2 : n // 2 + m // 2, n // 2 - m // 2 : n // 2 + m // 2] = block * inside
    intensity = np.abs(np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(obj), norm="ortho"))) ** 2
    return obj, np.abs(obj) > 0, intensity.astype(np.float32)
