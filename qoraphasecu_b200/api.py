"""``reconstruct``: array in, reconstruction out, on the B200 backend.

Mirrors the reference's ``python/qoraphasecu/api.py`` (``reconstruct`` at
:120-185, ``Reconstruction``/``Ensemble`` at :16-66) and the C++
``make_problem``/``make_solver``/``Solver::run``/``results`` chain underneath
(``include/qoraphasecu/solver.hpp:67-80``), all through ``libqpb.so``.
"""

from __future__ import annotations

import ctypes
import sys
import threading
import warnings
from dataclasses import dataclass
from typing import Literal

import numpy as np

from . import _lib
from .recipe import Recipe, default_recipe

NEGATIVE_WARN_FRACTION = 0.01


@dataclass(frozen=True)
class Reconstruction:
    """One reconstructed object, defined up to a global phase, a translation and a twin."""

    object: np.ndarray
    support: np.ndarray
    errors: np.ndarray

    @property
    def amplitude(self):
        return abs(self.object)

    @property
    def phase(self):
        return self.object.angle() if _is_cuda_tensor(self.object) else np.angle(self.object)

    @property
    def error(self) -> float:
        """Final Fourier error (NaN before any iteration); the ranking key."""
        return float(self.errors[-1]) if self.errors.size else float("nan")


@dataclass(frozen=True)
class Ensemble:
    """The runs of a multi-start reconstruction, not mutually aligned."""

    runs: tuple

    def __len__(self) -> int:
        return len(self.runs)

    def __iter__(self):
        return iter(self.runs)

    def __getitem__(self, index):
        return self.runs[index]

    @property
    def ranking(self) -> tuple:
        """Run indices, lowest final error first."""
        return tuple(sorted(range(len(self.runs)), key=lambda i: self.runs[i].error))

    @property
    def best(self) -> Reconstruction:
        return self.runs[best_index(self.runs)]

    def average(self, runs: int | None = None):
        """The mean of the ``runs`` best runs (all by default), each translated,
        twin-flipped if that fits better and phase-rotated onto the best run
        (device alignment, :func:`align`). Returns ``(mean, aligned errors)``."""
        order = self.ranking[: runs or len(self.runs)]
        host = (lambda o: o.detach().cpu().numpy() if _is_cuda_tensor(o) else np.asarray(o))
        stack = np.stack([host(self.runs[i].object) for i in order])
        _, mean, errors = align(stack, stack[0])
        return mean, errors


def best_index(runs) -> int:
    """Index of the run with the lowest final error; a NaN run never displaces a
    finite one (src/core/solver.cpp:95-103)."""
    runs = list(runs)
    if not runs:
        raise ValueError("no runs")
    best = 0
    for i in range(1, len(runs)):
        e, b = runs[i].error, runs[best].error
        if e < b or np.isnan(b):
            best = i
    return best


def cuda_available() -> bool:
    return bool(_lib.load().qpb_cuda_available())


def set_device(device: int) -> None:
    """Device used on this thread by calls without a solver (make_problem,
    operators) and by reconstruct()."""
    _lib.check(_lib.load().qpb_set_device(device))
    _cache.device = device


def tuning_report() -> str:
    """The autotuner's choices so far: starts per launch per shape and start count."""
    buf = ctypes.create_string_buffer(8192)
    _lib.check(_lib.load().qpb_tuning_report(buf, len(buf)))
    return buf.value.decode()


def kernel_launches() -> int:
    """Kernels libqpb.so has launched in this process (graph replays count each node)."""
    return int(_lib.load().qpb_kernel_launches())


def _is_cuda_tensor(x) -> bool:
    """A torch tensor in device memory (the zero-copy path); torch is imported
    only by callers that pass one."""
    return type(x).__module__.startswith("torch") and bool(getattr(x, "is_cuda", False))


def _torch_stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


def _shape(array: np.ndarray):
    if array.ndim not in (2, 3):
        raise ValueError(f"intensity must be 2D or 3D, got ndim={array.ndim}")
    return _lib.shape_arg(array.shape)


def autocorrelation_support(intensity, threshold: float = 0.1) -> np.ndarray:
    """Loose support from the thresholded autocorrelation (device FFT); shrinkwrap tightens it."""
    intensity = np.ascontiguousarray(intensity, dtype=np.float32)
    out = np.empty(intensity.shape, np.uint8)
    lib = _lib.load()
    _lib.check(lib.qpb_autocorrelation_support(_lib.ptr(intensity), intensity.ndim,
                                               _shape(intensity), threshold, _lib.ptr(out)))
    return out.astype(bool)


def half_support(support, axis: int = 0) -> np.ndarray:
    """The support below its centre of mass along ``axis`` (the detwin cut)."""
    support = np.ascontiguousarray(support, dtype=bool).view(np.uint8)
    out = np.empty(support.shape, np.uint8)
    lib = _lib.load()
    _lib.check(lib.qpb_half_support(_lib.ptr(support), support.ndim, _shape(support), axis,
                                    _lib.ptr(out)))
    return out.astype(bool)


def aligned_error(a, reference):
    """``||a - reference|| / ||reference||`` after removing shift, global phase
    and twin (python/qoraphasecu/api.py:89-95 of the reference), on the device.
    ``a`` may also be a stack ``(batch, *reference.shape)``: then one error per
    object comes back, computed in one batch."""
    a = np.ascontiguousarray(a, dtype=np.complex64)
    reference = np.ascontiguousarray(reference, dtype=np.complex64)
    stacked = a.ndim == reference.ndim + 1 and a.shape[1:] == reference.shape
    if a.shape != reference.shape and not stacked:
        raise ValueError(f"shapes differ: {a.shape} vs {reference.shape}")
    batch = a.shape[0] if stacked else 1
    out = np.empty(batch, np.float32)
    _lib.check(_lib.load().qpb_aligned_error(_lib.ptr(a), _lib.ptr(reference), reference.ndim,
                                             _shape(reference), batch, _lib.ptr(out)))
    return out if stacked else float(out[0])


def align(objects, reference):
    """Moves every object of a stack ``(batch, *shape)`` onto ``reference``: the
    translation (cross-correlation peak), twin and global phase that
    ``aligned_error`` finds, applied on the device. Returns ``(aligned,
    mean, errors)``: the aligned stack, its average and the aligned errors."""
    objects = np.ascontiguousarray(objects, dtype=np.complex64)
    reference = np.ascontiguousarray(reference, dtype=np.complex64)
    if objects.ndim != reference.ndim + 1 or objects.shape[1:] != reference.shape:
        raise ValueError(f"objects.shape {objects.shape} is not a stack of {reference.shape}")
    aligned = np.empty_like(objects)
    mean = np.empty_like(reference)
    errors = np.empty(objects.shape[0], np.float32)
    _lib.check(_lib.load().qpb_align(_lib.ptr(objects), _lib.ptr(reference), reference.ndim,
                                     _shape(reference), objects.shape[0], _lib.ptr(errors),
                                     _lib.ptr(aligned), _lib.ptr(mean)))
    return aligned, mean, errors


def simulate_intensity(obj) -> np.ndarray:
    """|centred unitary FFT(obj)|^2 as float32 (src/core/problem.cpp:90-99), the
    transform on the device."""
    obj = np.ascontiguousarray(obj, dtype=np.complex64)
    out = np.empty(obj.shape, np.float32)
    _lib.check(_lib.load().qpb_simulate_intensity(_lib.ptr(obj), obj.ndim, _shape(obj),
                                                  _lib.ptr(out)))
    return out


@dataclass
class Problem:
    """Centre-origin amplitude, mask and support (the reference's qpcu::Problem)."""

    amplitude: np.ndarray
    mask: np.ndarray
    support: np.ndarray

    @property
    def shape(self):
        return tuple(self.amplitude.shape)

    @property
    def on_device(self) -> bool:
        """True when the arrays are CUDA torch tensors (make_problem of one)."""
        return _is_cuda_tensor(self.amplitude)

    def _c(self):
        p = _lib.Problem()
        p.ndim = self.amplitude.ndim
        p.shape = _lib.shape_arg(self.amplitude.shape)
        if self.on_device:
            p.amplitude = ctypes.cast(self.amplitude.data_ptr(), ctypes.POINTER(ctypes.c_float))
            p.mask = ctypes.cast(self.mask.data_ptr(), ctypes.POINTER(ctypes.c_uint8))
            p.support = ctypes.cast(self.support.data_ptr(), ctypes.POINTER(ctypes.c_uint8))
            return p
        p.amplitude = self.amplitude.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        p.mask = self.mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        p.support = self.support.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        return p


def _make_problem_device(intensity, support, mask, support_threshold):
    """make_problem on CUDA torch tensors: every array stays on the device."""
    import torch

    intensity = intensity.detach().to(torch.float32).contiguous()
    if intensity.dim() not in (2, 3):
        raise ValueError(f"intensity must be 2D or 3D, got ndim={intensity.dim()}")

    def flag(name, array):
        if array is None:
            return None
        array = torch.as_tensor(array, device=intensity.device)
        if tuple(array.shape) != tuple(intensity.shape):
            raise ValueError(f"{name}.shape {tuple(array.shape)} != intensity.shape "
                             f"{tuple(intensity.shape)}")
        return (array != 0).to(torch.uint8).contiguous()

    support = flag("support", support)
    mask = flag("mask", mask)
    amp = torch.empty_like(intensity)
    m = torch.empty(intensity.shape, dtype=torch.uint8, device=intensity.device)
    sup = torch.empty_like(m)
    ptr = (lambda t: None if t is None else ctypes.c_void_p(t.data_ptr()))
    _lib.check(_lib.load().qpb_make_problem_device(
        ptr(intensity), intensity.dim(), _lib.shape_arg(intensity.shape), ptr(support), ptr(mask),
        support_threshold, ptr(amp), ptr(m), ptr(sup), ctypes.c_void_p(_torch_stream())))
    return Problem(amp, m, sup)


def make_problem(intensity, support=None, mask=None, support_threshold: float = 0.1) -> Problem:
    """Validates the inputs and derives the amplitude; a missing support is the
    autocorrelation support (src/core/problem.cpp:40-70). A CUDA torch tensor
    gives a problem whose arrays stay on the device (no host copy)."""
    if _is_cuda_tensor(intensity):
        return _make_problem_device(intensity, support, mask, support_threshold)
    intensity = np.ascontiguousarray(intensity, dtype=np.float32)
    shape = _shape(intensity)
    support = _flag("support", support, intensity.shape)
    mask = _flag("mask", mask, intensity.shape)
    amp = np.empty(intensity.shape, np.float32)
    m = np.empty(intensity.shape, np.uint8)
    s = np.empty(intensity.shape, np.uint8)
    lib = _lib.load()
    _lib.check(lib.qpb_make_problem(_lib.ptr(intensity), intensity.ndim, shape, _lib.ptr(support),
                                    _lib.ptr(mask), support_threshold, _lib.ptr(amp),
                                    _lib.ptr(m), _lib.ptr(s)))
    return Problem(amp, m, s)


def _host_empty(shape, dtype):
    """A host array for results the device writes: page-locked memory from
    torch's caching pinned-memory allocator when torch is already loaded (the
    copy runs at full link speed, and a block the caller has dropped is reused
    without a new page-locking call), else ordinary numpy memory."""
    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_available():
        count = int(np.prod(shape)) * np.dtype(dtype).itemsize
        block = torch.empty(count, dtype=torch.uint8, pin_memory=True)
        return block.numpy().view(dtype).reshape(shape)
    return np.empty(shape, dtype)


def _flag(name, array, shape):
    if array is None:
        return None
    array = np.ascontiguousarray(array, dtype=bool)
    if array.shape != shape:
        raise ValueError(f"{name}.shape {array.shape} != intensity.shape {shape}")
    return array.view(np.uint8)


def _start(init, shape, starts):
    if init is None:
        return None
    init = np.asarray(init, dtype=np.complex64)
    if init.shape == tuple(shape):
        init = np.broadcast_to(init, (starts, *shape))
    if init.shape != (starts, *shape):
        raise ValueError(
            f"init.shape {init.shape} must be the intensity's {tuple(shape)} or (starts, *shape)"
        )
    return np.ascontiguousarray(init)


def _start_device(init, shape, starts):
    if init is None:
        return None
    import torch

    if not _is_cuda_tensor(init):
        raise ValueError("a device problem takes its init as a CUDA tensor")
    init = init.to(torch.complex64)
    if tuple(init.shape) == tuple(shape):
        init = init.expand(starts, *shape)
    if tuple(init.shape) != (starts, *shape):
        raise ValueError(f"init.shape {tuple(init.shape)} must be the intensity's {tuple(shape)} "
                         "or (starts, *shape)")
    return init.contiguous()


def _ops(recipe):
    ops = recipe.ops() if hasattr(recipe, "ops") else list(recipe)
    array = (_lib.Op * max(len(ops), 1))()
    for i, (kind, n, beta, threshold, sigma, method, axis) in enumerate(ops):
        if kind not in _lib.OP_KINDS:
            raise ValueError(f"unknown recipe operation '{kind}'")
        if method not in _lib.METHODS:
            raise ValueError(f"method must be 'max' or 'rms', got {method!r}")
        array[i] = _lib.Op(_lib.OP_KINDS[kind], int(n), float(beta), float(threshold),
                           float(sigma), _lib.METHODS[method], int(axis))
    return array, len(ops)


def _options(starts, batch, seed, start, sync_every, variant, amp_storage, device, stream,
             schedule):
    if variant not in _lib.VARIANTS:
        raise ValueError(f"unknown variant '{variant}' (this backend has 'batched', 'plain', "
                         "'half' and 'mixed')")
    if schedule not in _lib.SCHEDULES:
        raise ValueError(f"unknown schedule '{schedule}' (auto, streamed or resident)")
    if amp_storage not in _lib.AMP_STORAGE:
        raise ValueError(f"unknown amp_storage '{amp_storage}'")
    options = _lib.Options()
    options.starts = starts
    options.batch = 0 if batch is None else batch
    options.seed = 0 if seed is None else seed
    options.start = (start.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
                     if start is not None else None)
    options.sync_every = sync_every
    options.variant = _lib.VARIANTS[variant]
    options.amp_storage = _lib.AMP_STORAGE[amp_storage]
    options.device = device
    options.stream = stream
    options.schedule = _lib.SCHEDULES[schedule]
    return options


class Solver:
    """A live reconstruction: starts drawn on construction; ``run`` continues
    from the current state and appends errors (include/qoraphasecu/solver.hpp:67-74)."""

    def __init__(self, problem: Problem, *, starts: int = 1, batch: int | None = None,
                 seed: int | None = None, init=None, sync_every: int = 10,
                 variant: Literal["batched", "plain", "half", "mixed"] = "batched",
                 amp_storage: Literal["f32", "f16", "bf16"] = "f32", progress=None,
                 device: int = -1, stream: int | None = None,
                 schedule: Literal["auto", "streamed", "resident", "persistent"] = "auto"):
        self.problem = problem
        self.shape = problem.shape
        self._on_device = problem.on_device
        if self._on_device:
            start = _start_device(init, problem.shape, starts)
            options = _options(starts, batch, seed, None, sync_every, variant, amp_storage,
                               device, stream, schedule)
            if start is not None:
                options.start = ctypes.cast(start.data_ptr(), ctypes.POINTER(ctypes.c_float))
        else:
            start = _start(init, problem.shape, starts)
            options = _options(starts, batch, seed, start, sync_every, variant, amp_storage,
                               device, stream, schedule)
        self._lib = _lib.load()
        handle = ctypes.c_void_p()
        create = self._lib.qpb_create_device if self._on_device else self._lib.qpb_create
        _lib.check(create(ctypes.byref(problem._c()), ctypes.byref(options), ctypes.byref(handle)))
        self._handle = handle
        self._progress = None
        if progress is not None:
            self.set_progress(progress)

    def set_progress(self, fn):
        """``fn(iteration, errors)`` every ``sync_every`` iterations, on this thread."""
        if fn is None:
            self._progress = None
            _lib.check(self._lib.qpb_set_progress(self._handle, _lib.PROGRESS(), None))
            return

        def trampoline(_user, iteration, errors, count):
            fn(iteration, np.ctypeslib.as_array(errors, shape=(count,)).copy())

        self._progress = _lib.PROGRESS(trampoline)
        _lib.check(self._lib.qpb_set_progress(self._handle, self._progress, None))

    def run(self, recipe=None):
        ops, count = _ops(default_recipe() if recipe is None else recipe)
        _lib.check(self._lib.qpb_run(self._handle, ops, count))

    def reset(self, problem: Problem, *, seed: int | None = None, init=None):
        """Loads a new problem of the same shape (host or device arrays, as at
        construction) and draws new starts (or takes ``init``), keeping the
        device buffers, schedule and captured graphs: the cheap way to run many
        same-shape reconstructions. Error histories start afresh."""
        if tuple(problem.shape) != tuple(self.shape):
            raise ValueError(f"problem.shape {tuple(problem.shape)} != solver shape "
                             f"{tuple(self.shape)}")
        if problem.on_device != self._on_device:
            raise ValueError("reset takes the same kind of arrays (host or device) as construction")
        starts = self.starts
        if self._on_device:
            start = _start_device(init, problem.shape, starts)
            ptr = None if start is None else ctypes.c_void_p(start.data_ptr())
        else:
            start = _start(init, problem.shape, starts)
            ptr = None if start is None else ctypes.c_void_p(start.ctypes.data)
        _lib.check(self._lib.qpb_reset(self._handle, ctypes.byref(problem._c()), 1,
                                       0 if seed is None else seed, ptr))
        self.problem = problem

    def set_wait_limit(self, polls: int, starve: bool = False):
        """Polls a line pass's wait for its staged inputs makes before it gives
        up (``run`` then raises TimeoutError); ``starve`` leaves the staged
        copies out so that every such wait runs out, the fault injection of the
        timeout tests (results are invalid until ``reset``)."""
        _lib.check(self._lib.qpb_set_wait_limit(self._handle, int(polls), int(bool(starve))))

    def profile_passes(self, iterations: int = 20):
        """Mean device time (ms) per launch of each line pass of an iteration:
        each pass launched ``iterations`` times back to back from one captured
        CUDA graph, whose replay two CUDA events time; with the resident
        schedule, one value: the mean time per iteration of one launch of
        ``iterations`` iterations. Leaves the solver as it was (iterate, wave,
        error history and iteration count); the call holds one more copy of
        the iterate and the wave on the device."""
        ms = (ctypes.c_double * 8)()
        n = ctypes.c_int()
        _lib.check(self._lib.qpb_profile_passes(self._handle, iterations, ms, ctypes.byref(n)))
        return [ms[i] for i in range(n.value)]

    @property
    def starts(self) -> int:
        n = ctypes.c_int()
        _lib.check(self._lib.qpb_starts(self._handle, ctypes.byref(n)))
        return n.value

    def error_count(self) -> int:
        n = ctypes.c_size_t()
        _lib.check(self._lib.qpb_error_count(self._handle, ctypes.byref(n)))
        return n.value

    def results(self):
        if self._on_device:
            return self._results_device()
        starts = self.starts
        count = self.error_count()
        objects = _host_empty((starts, *self.shape), np.complex64)
        supports = _host_empty((starts, *self.shape), np.uint8)
        errors = np.empty((starts, count), np.float32)
        _lib.check(self._lib.qpb_results(self._handle, _lib.ptr(objects), _lib.ptr(supports),
                                         _lib.ptr(errors)))
        supports = supports.view(np.bool_)  # the device writes 0 or 1
        return [Reconstruction(objects[s], supports[s], errors[s]) for s in range(starts)]

    def _results_device(self):
        """Objects and supports as CUDA torch tensors, written by the device."""
        import torch

        starts = self.starts
        count = self.error_count()
        dev = self.problem.amplitude.device
        objects = torch.empty((starts, *self.shape), dtype=torch.complex64, device=dev)
        supports = torch.empty((starts, *self.shape), dtype=torch.uint8, device=dev)
        errors = np.empty((starts, count), np.float32)
        _lib.check(self._lib.qpb_results_device(
            self._handle, ctypes.c_void_p(objects.data_ptr()),
            ctypes.c_void_p(supports.data_ptr()), _lib.ptr(errors)))
        return [Reconstruction(objects[s], supports[s].bool(), errors[s]) for s in range(starts)]

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.qpb_destroy(self._handle)
            self._handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class BatchSolver:
    """Many problems, any mix of shapes, reconstructed together.

    Problems of one shape share one batched solver (its schedule autotuned for
    that shape and start count); every chunk of ``sync_every`` iterations of
    every shape runs as one CUDA graph with the shapes as parallel branches.
    ``starts`` starts per problem; ``init``, when given, is one start array per
    problem (shape ``shape`` or ``(starts, *shape)``). ``results()`` returns
    one list of reconstructions per problem."""

    def __init__(self, problems, *, starts: int = 1, batch: int | None = None,
                 seed: int | None = None, init=None, sync_every: int = 10,
                 variant: Literal["batched", "plain", "half", "mixed"] = "batched",
                 amp_storage: Literal["f32", "f16", "bf16"] = "f32", progress=None,
                 device: int = -1, stream: int | None = None,
                 schedule: Literal["auto", "streamed", "resident", "persistent"] = "auto"):
        self.problems = list(problems)
        if not self.problems:
            raise ValueError("no problems")
        start = None
        if init is not None:
            if len(init) != len(self.problems):
                raise ValueError(f"init has {len(init)} entries for {len(self.problems)} problems")
            start = np.concatenate([_start(i, p.shape, starts).ravel()
                                    for i, p in zip(init, self.problems)])
        options = _options(starts, batch, seed, start, sync_every, variant, amp_storage, device,
                           stream, schedule)
        self._starts = starts
        self._views = (_lib.Problem * len(self.problems))(*[p._c() for p in self.problems])
        self._lib = _lib.load()
        handle = ctypes.c_void_p()
        _lib.check(self._lib.qpb_create_batch(self._views, len(self.problems),
                                              ctypes.byref(options), ctypes.byref(handle)))
        self._handle = handle
        self._progress = None
        if progress is not None:
            self.set_progress(progress)

    def reset(self, problems, *, seed: int | None = None, init=None):
        """Loads new problems, problem q in the shape problem q had at
        construction (host or device arrays as then), and draws new starts (or
        takes ``init``, one start array per problem), keeping the device
        buffers, schedules and captured graphs. Error histories start afresh."""
        problems = list(problems)
        if len(problems) != len(self.problems):
            raise ValueError(f"reset needs {len(self.problems)} problems, got {len(problems)}")
        for q, (new, old) in enumerate(zip(problems, self.problems)):
            if tuple(new.shape) != tuple(old.shape):
                raise ValueError(f"problem {q} has shape {tuple(new.shape)}, the batch was built "
                                 f"with {tuple(old.shape)}")
        start = None
        if init is not None:
            if len(init) != len(problems):
                raise ValueError(f"init has {len(init)} entries for {len(problems)} problems")
            start = np.concatenate([_start(i, p.shape, self._starts).ravel()
                                    for i, p in zip(init, problems)])
        views = (_lib.Problem * len(problems))(*[p._c() for p in problems])
        ptr = None if start is None else ctypes.c_void_p(start.ctypes.data)
        _lib.check(self._lib.qpb_reset(self._handle, views, len(problems),
                                       0 if seed is None else seed, ptr))
        self.problems = problems
        self._views = views

    def set_progress(self, fn):
        """``fn(iteration, errors)`` every ``sync_every`` iterations; ``errors``
        holds problems * starts values, problem by problem."""
        if fn is None:
            self._progress = None
            _lib.check(self._lib.qpb_set_progress(self._handle, _lib.PROGRESS(), None))
            return

        def trampoline(_user, iteration, errors, count):
            fn(iteration, np.ctypeslib.as_array(errors, shape=(count,)).copy())

        self._progress = _lib.PROGRESS(trampoline)
        _lib.check(self._lib.qpb_set_progress(self._handle, self._progress, None))

    def run(self, recipe=None):
        ops, count = _ops(default_recipe() if recipe is None else recipe)
        _lib.check(self._lib.qpb_run(self._handle, ops, count))

    def error_count(self) -> int:
        n = ctypes.c_size_t()
        _lib.check(self._lib.qpb_error_count(self._handle, ctypes.byref(n)))
        return n.value

    def profile_passes(self, iterations: int = 20):
        """As ``Solver.profile_passes``; the problems must share one shape."""
        ms = (ctypes.c_double * 8)()
        n = ctypes.c_int()
        _lib.check(self._lib.qpb_profile_passes(self._handle, iterations, ms, ctypes.byref(n)))
        return [ms[i] for i in range(n.value)]

    def results(self):
        count = self.error_count()
        sizes = [int(np.prod(p.shape)) for p in self.problems]
        total = self._starts * sum(sizes)
        objects = _host_empty(total, np.complex64)
        supports = _host_empty(total, np.uint8)
        errors = np.empty((len(self.problems), self._starts, count), np.float32)
        _lib.check(self._lib.qpb_results(self._handle, _lib.ptr(objects), _lib.ptr(supports),
                                         _lib.ptr(errors)))
        supports = supports.view(np.bool_)  # the device writes 0 or 1
        out, at = [], 0
        for q, p in enumerate(self.problems):
            block = self._starts * sizes[q]
            obj = objects[at:at + block].reshape(self._starts, *p.shape)
            sup = supports[at:at + block].reshape(self._starts, *p.shape)
            out.append([Reconstruction(obj[s], sup[s], errors[q, s]) for s in range(self._starts)])
            at += block
        return out

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.qpb_destroy(self._handle)
            self._handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def reconstruct_batch(intensities, *, supports=None, masks=None, recipe=None, starts: int = 1,
                      support_threshold: float = 0.1, **options):
    """``reconstruct`` over many intensities of any mix of shapes in one batch
    (:class:`BatchSolver`); returns one Reconstruction (starts == 1) or
    Ensemble per intensity, in order. ``supports`` / ``masks``: None or one
    entry (possibly None) per intensity. The batch solver is kept for the next
    call with the same shapes in the same order and options (one per thread;
    clear_cache() releases it)."""
    intensities = list(intensities)
    supports = [None] * len(intensities) if supports is None else list(supports)
    masks = [None] * len(intensities) if masks is None else list(masks)
    if not (len(supports) == len(masks) == len(intensities)):
        raise ValueError("supports and masks need one entry per intensity")
    problems = [make_problem(i, s, m, support_threshold)
                for i, s, m in zip(intensities, supports, masks)]
    seed = options.pop("seed", None)
    init = options.pop("init", None)
    progress = options.pop("progress", None)
    # like reconstruct(): the batch solver of the last call with the same
    # shapes and options is reloaded (BatchSolver.reset) instead of rebuilt
    try:
        key = ("batch", tuple(tuple(p.shape) for p in problems), problems[0].on_device, starts,
               tuple(sorted(options.items())), _current_device())
        hash(key)
    except TypeError:
        key = None
    solver = _cached_solvers().get(key) if key is not None else None
    if solver is not None and solver._handle:
        solver.reset(problems, seed=seed, init=init)
    else:
        solver = BatchSolver(problems, starts=starts, seed=seed, init=init, **options)
        if key is not None:
            cache = _cached_solvers()
            for old in [k for k in cache if k[0] == "batch"]:
                cache.pop(old).close()
            cache[key] = solver
    try:
        solver.set_progress(progress)
        solver.run(default_recipe() if recipe is None else recipe)
        runs = solver.results()
        solver.set_progress(None)
    finally:
        if key is None:
            solver.close()
    return [r[0] if starts == 1 else Ensemble(tuple(r)) for r in runs]


def reconstruct(
    intensity,
    *,
    support=None,
    mask=None,
    recipe=None,
    starts: int = 1,
    batch: int | None = None,
    seed: int | None = None,
    init=None,
    support_threshold: float = 0.1,
    backend: Literal["auto", "b200"] = "auto",
    variant: Literal["batched", "plain", "half", "mixed"] = "batched",
    sync_every: int = 10,
    amp_storage: Literal["f32", "f16", "bf16"] = "f32",
    progress=None,
    schedule: Literal["auto", "streamed", "resident", "persistent"] = "auto",
) -> Reconstruction | Ensemble:
    """Array in, reconstruction out.

    Args:
        intensity: measured intensity, centre-origin, 2D or 3D: a numpy array,
            or a CUDA torch tensor, in which case every array stays on the
            device and the results' objects and supports are CUDA tensors.
        support: boolean, True inside the object; None derives the
            autocorrelation support.
        mask: boolean, True marks unusable pixels.
        recipe: a :class:`Recipe` (None: :func:`default_recipe`).
        starts: random starts; more than one returns an :class:`Ensemble`.
        batch: starts per launch (``variant="batched"``); None puts all in one.
        seed: seed of the random starting phases; None means 0.
        init: starting object(s), centre-origin, shape ``shape`` or
            ``(starts, *shape)``, cut to the support.
        backend: ``"auto"`` or ``"b200"``; both run this backend, which needs
            a CUDA device.
        variant: ``"batched"`` (graph-captured, all starts per launch),
            ``"plain"`` (one start per launch), or the fp16-storage forms of
            batched: ``"half"`` (iterate and wave as fp16 pairs) and
            ``"mixed"`` (fp16 wave for HIO and RAAR, FP32 iterate and ER);
            both need power-of-two extents of 16..1024.
        amp_storage: ``"f32"``, ``"f16"`` or ``"bf16"`` storage of the amplitude.
        progress: ``fn(iteration, errors)`` every ``sync_every`` iterations.
        schedule: how batched iterations run: ``"streamed"`` line passes,
            ``"resident"`` (square 2D of side 64, 128 or 256: each start held in
            a thread-block cluster's shared memory), ``"persistent"`` (2D with
            sides of 64, 128 or 256: a chunk of iterations of every start as
            one launch walking a work list of tiles) or ``"auto"`` (timed once
            per shape and start count).
    """
    if _is_cuda_tensor(intensity):
        if intensity.dim() not in (2, 3):
            raise ValueError(f"intensity must be 2D or 3D, got ndim={intensity.dim()}")
        negative = float((intensity < 0).float().mean().item())
    else:
        intensity = np.ascontiguousarray(intensity, dtype=np.float32)
        if intensity.ndim not in (2, 3):
            raise ValueError(f"intensity must be 2D or 3D, got ndim={intensity.ndim}")
        negative = float(np.mean(intensity < 0))
    if negative > NEGATIVE_WARN_FRACTION:
        warnings.warn(
            f"{negative:.1%} of intensity pixels are negative and will be clipped to 0; "
            "consider masking them instead",
            stacklevel=2,
        )
    if backend not in ("auto", "b200"):
        raise ValueError(
            f"backend '{backend}' is not provided here; this package is the 'b200' backend"
        )
    if recipe is None:
        recipe = default_recipe()
    problem = make_problem(intensity, support, mask, support_threshold)
    key = (tuple(problem.shape), problem.on_device, starts, batch, sync_every, variant,
           amp_storage, schedule, _current_device())
    solver = _cached_solvers().get(key)
    if solver is not None and solver._handle:
        solver.reset(problem, seed=seed, init=init)
    else:
        solver = Solver(problem, starts=starts, batch=batch, seed=seed, init=init,
                        sync_every=sync_every, variant=variant, amp_storage=amp_storage,
                        schedule=schedule)
        _cached_solvers()[key] = solver
    solver.set_progress(progress)
    solver.run(recipe)
    runs = solver.results()
    solver.set_progress(None)
    return runs[0] if starts == 1 else Ensemble(tuple(runs))


_cache = threading.local()


def _cached_solvers() -> dict:
    """reconstruct() keeps the solver of its last call per configuration and
    thread, and loads the next same-shape problem into it (Solver.reset):
    allocation and graph capture are paid once. clear_cache() releases them."""
    if not hasattr(_cache, "solvers"):
        _cache.solvers = {}
    return _cache.solvers


def clear_cache() -> None:
    """Releases the solvers (and their device memory) that reconstruct() and
    reconstruct_batch() keep for reuse on this thread."""
    for solver in _cached_solvers().values():
        solver.close()
    _cached_solvers().clear()


def _current_device() -> int:
    """The device set by set_device() on this thread (-1: never set), part of
    the reconstruct cache key."""
    return getattr(_cache, "device", -1)


__all__ = [
    "BatchSolver",
    "Ensemble",
    "Problem",
    "Recipe",
    "Reconstruction",
    "Solver",
    "align",
    "aligned_error",
    "autocorrelation_support",
    "best_index",
    "cuda_available",
    "half_support",
    "make_problem",
    "reconstruct",
    "reconstruct_batch",
    "simulate_intensity",
    "clear_cache",
]
