"""Single projections on centre-origin arrays (the reference's qpcu::cuda::
operators, include/qoraphasecu/operators.hpp:25-33), on the device."""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .api import Problem


def modulus_project(problem: Problem, obj, amp_storage: str = "f32"):
    """Returns ``(P_M obj, Fourier error of obj)``."""
    out = np.array(obj, dtype=np.complex64, order="C", copy=True)
    if out.shape != problem.shape:
        raise ValueError("obj does not match the problem shape")
    err = ctypes.c_float()
    lib = _lib.load()
    _lib.check(lib.qpb_modulus_project(ctypes.byref(problem._c()), _lib.ptr(out),
                                       _lib.AMP_STORAGE[amp_storage], ctypes.byref(err)))
    return out, float(err.value)


def support_project(support, obj):
    """Zero outside the support."""
    out = np.array(obj, dtype=np.complex64, order="C", copy=True)
    support = np.ascontiguousarray(support, dtype=bool).view(np.uint8)
    if support.shape != out.shape:
        raise ValueError("support does not match obj")
    lib = _lib.load()
    _lib.check(lib.qpb_support_project(_lib.ptr(support), _lib.ptr(out), out.size))
    return out


def gaussian_blur(image, sigma: float):
    """Periodic Gaussian blur with transfer function exp(-2 (pi sigma f)^2)."""
    image = np.ascontiguousarray(image, dtype=np.float32)
    out = np.empty_like(image)
    lib = _lib.load()
    _lib.check(lib.qpb_gaussian_blur(_lib.ptr(image), image.ndim, _lib.shape_arg(image.shape),
                                     sigma, _lib.ptr(out)))
    return out
