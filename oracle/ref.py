"""ctypes access to the compiled reference oracle (oracle/_ref/libqpcu_ref.so).

TEST INFRASTRUCTURE. The library is QoraPhaseCU's own CPU path compiled from
its sources by ``oracle/Makefile`` with ``oracle/fft_shim.cpp`` standing in for
the absent pocketfft. Only tests and bench.py's CPU-baseline legs use it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import time
from ctypes import POINTER, c_char_p, c_float, c_int, c_int64, c_size_t, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_ref" / "libqpcu_ref.so"
CUDA_LIBRARY = HERE / "_ref" / "libqpcu_ref_cuda.so"
DROPIN_LIBRARY = HERE / "_ref" / "libqpcu_dropin.so"

_lib = None
_libs = {}

OP_KINDS = {"er": 0, "hio": 1, "raar": 2, "shrinkwrap": 3, "detwin_begin": 4, "detwin_end": 5}


class _Op(ctypes.Structure):
    _fields_ = [("kind", c_int), ("n", c_int), ("beta", c_float), ("threshold", c_float),
                ("sigma", c_float), ("method", c_int), ("axis", c_int)]


def build(reference=None) -> bool:
    """Compiles the reference oracle libraries (oracle/Makefile) when the
    reference sources are present at `reference` (default: the QPCU_REFERENCE
    environment variable); without them, the libraries built before are kept."""
    root = reference or os.environ.get("QPCU_REFERENCE")
    if not root or not (Path(root) / "src" / "cpu" / "cpu_solver.cpp").exists():
        return LIBRARY.exists()
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={root}", "all"], check=True)
    return LIBRARY.exists()


def available() -> bool:
    return LIBRARY.exists()


def _configure(lib):
    lib.qref_last_error.restype = c_char_p
    lib.qref_set_threads.argtypes = [c_int]
    lib.qref_set_threads.restype = None
    lib.qref_create.argtypes = [c_void_p, c_void_p, c_void_p, c_int, POINTER(c_int64), c_int,
                                c_uint64, c_void_p, c_int, POINTER(c_void_p)]
    lib.qref_create_backend.argtypes = [c_void_p, c_void_p, c_void_p, c_int, POINTER(c_int64),
                                        c_int, c_uint64, c_void_p, c_int, c_int, c_int, c_int,
                                        POINTER(c_void_p)]
    lib.qref_reconstruct.argtypes = [c_void_p, c_void_p, c_void_p, c_int, POINTER(c_int64),
                                     c_void_p, c_size_t, c_int, c_uint64, c_int, c_void_p,
                                     c_void_p, c_void_p, POINTER(c_int)]
    lib.qref_cuda_available.restype = c_int
    lib.qref_run.argtypes = [c_void_p, c_void_p, c_size_t]
    lib.qref_results.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_size_t)]
    lib.qref_error_count.argtypes = [c_void_p]
    lib.qref_error_count.restype = c_size_t
    lib.qref_destroy.argtypes = [c_void_p]
    lib.qref_destroy.restype = None
    for name in ("qref_fft", "qref_make_problem", "qref_modulus_project", "qref_gaussian_blur",
                 "qref_half_support", "qref_autocorrelation_support",
                 "qref_simulate_intensity", "qref_aligned_error"):
        getattr(lib, name).restype = c_int
    return lib


def load_variant(which: str):
    """One of the oracle libraries: "cpu" (the reference's CPU path), "cuda"
    (plus the reference's own CUDA backend) or "dropin" (the reference's core
    with its Backend::cuda slot bound to the B200 adapter)."""
    path = {"cpu": LIBRARY, "cuda": CUDA_LIBRARY, "dropin": DROPIN_LIBRARY}[which]
    if which not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing: build it with oracle/Makefile")
        _libs[which] = _configure(ctypes.CDLL(str(path)))
    return _libs[which]


def load():
    """The reference's CPU path (oracle/_ref/libqpcu_ref.so)."""
    global _lib
    if _lib is None:
        _lib = load_variant("cpu")
    return _lib


def _check(status):
    if status == 0:
        return
    msg = load().qref_last_error().decode()
    raise (ValueError if status == 1 else RuntimeError)(msg)


def _p(a):
    return None if a is None else c_void_p(a.ctypes.data)


def _shape(shape):
    return (c_int64 * 3)(*(list(shape) + [0] * (3 - len(shape))))


def fft(a, forward=True):
    a = np.ascontiguousarray(a, np.complex64)
    out = np.empty_like(a)
    _check(load().qref_fft(_p(a), _p(out), a.ndim, _shape(a.shape), int(forward)))
    return out


def make_problem(intensity, support=None, mask=None, threshold=0.1):
    intensity = np.ascontiguousarray(intensity, np.float32)
    sup = None if support is None else np.ascontiguousarray(support, np.uint8)
    msk = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    amp = np.empty(intensity.shape, np.float32)
    m = np.empty(intensity.shape, np.uint8)
    s = np.empty(intensity.shape, np.uint8)
    _check(load().qref_make_problem(_p(intensity), intensity.ndim, _shape(intensity.shape), _p(sup),
                                    _p(msk), c_float(threshold), _p(amp), _p(m), _p(s)))
    return amp, m, s


def modulus_project(problem, obj):
    amp, mask, support = problem
    out = np.array(obj, np.complex64, order="C", copy=True)
    err = c_float()
    _check(load().qref_modulus_project(_p(amp), _p(mask), _p(support), amp.ndim, _shape(amp.shape),
                                       _p(out), ctypes.byref(err)))
    return out, float(err.value)


def gaussian_blur(image, sigma):
    image = np.ascontiguousarray(image, np.float32)
    out = np.empty_like(image)
    _check(load().qref_gaussian_blur(_p(image), image.ndim, _shape(image.shape), c_float(sigma),
                                     _p(out)))
    return out


def half_support(support, axis=0):
    support = np.ascontiguousarray(support, np.uint8)
    out = np.empty_like(support)
    _check(load().qref_half_support(_p(support), support.ndim, _shape(support.shape), axis, _p(out)))
    return out


def autocorrelation_support(intensity, threshold=0.1):
    intensity = np.ascontiguousarray(intensity, np.float32)
    out = np.empty(intensity.shape, np.uint8)
    _check(load().qref_autocorrelation_support(_p(intensity), intensity.ndim,
                                               _shape(intensity.shape), c_float(threshold), _p(out)))
    return out


def simulate_intensity(obj):
    obj = np.ascontiguousarray(obj, np.complex64)
    out = np.empty(obj.shape, np.float32)
    _check(load().qref_simulate_intensity(_p(obj), obj.ndim, _shape(obj.shape), _p(out)))
    return out


def aligned_error(a, ref):
    a = np.ascontiguousarray(a, np.complex64)
    ref = np.ascontiguousarray(ref, np.complex64)
    out = c_float()
    _check(load().qref_aligned_error(_p(a), _p(ref), a.ndim, _shape(a.shape), ctypes.byref(out)))
    return float(out.value)


def _ops(ops):
    arr = (_Op * max(len(ops), 1))()
    for i, (kind, n, beta, threshold, sigma, method, axis) in enumerate(ops):
        arr[i] = _Op(OP_KINDS[kind], int(n), beta, threshold, sigma, 1 if method == "rms" else 0,
                     int(axis))
    return arr


class Solver:
    """The reference CpuSolver (Backend::cpu) behind qpcu::make_solver."""

    def __init__(self, problem, starts=1, seed=0, start=None, sync_every=10):
        amp, mask, support = problem
        self.shape = amp.shape
        self.starts = starts
        st = None if start is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(start, np.complex64), (starts, *amp.shape)))
        self._keep = (amp, mask, support, st)
        h = c_void_p()
        _check(load().qref_create(_p(amp), _p(mask), _p(support), amp.ndim, _shape(amp.shape),
                                  starts, c_uint64(seed), _p(st), sync_every, ctypes.byref(h)))
        self._h = h

    def run(self, ops):
        arr = _ops(ops)
        _check(load().qref_run(self._h, arr, len(ops)))

    def results(self):
        count = load().qref_error_count(self._h)
        objs = np.empty((self.starts, *self.shape), np.complex64)
        sups = np.empty((self.starts, *self.shape), np.uint8)
        errs = np.empty((self.starts, count), np.float32)
        n = c_size_t()
        _check(load().qref_results(self._h, _p(objs), _p(sups), _p(errs), ctypes.byref(n)))
        return [(objs[s], sups[s].astype(bool), errs[s]) for s in range(self.starts)]

    def __del__(self):
        if getattr(self, "_h", None):
            load().qref_destroy(self._h)
            self._h = None


def reconstruct(problem, ops, starts=1, seed=0, start=None):
    s = Solver(problem, starts=starts, seed=seed, start=start)
    s.run(ops)
    return s.results()


def time_iterations(intensity, mask, starts, iterations, threads):
    """Seconds for `iterations` RAAR(0.9) iterations of `starts` starts with the
    reference CpuSolver on `threads` OpenMP threads (construction not timed)."""
    load().qref_set_threads(threads)
    problem = make_problem(intensity, None, mask)
    solver = Solver(problem, starts=starts, seed=0)
    t0 = time.perf_counter()
    solver.run([("raar", iterations, 0.9, 0.0, 0.0, "max", 0)])
    return time.perf_counter() - t0
