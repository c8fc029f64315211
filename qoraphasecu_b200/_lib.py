"""ctypes binding of libqpb.so (include/qpb.h).

The library is loaded on first use. There is no fallback: if it is missing,
every call raises with the command that builds it.
"""

from __future__ import annotations

import ctypes
import threading
from ctypes import (
    CFUNCTYPE,
    POINTER,
    Structure,
    c_char_p,
    c_double,
    c_float,
    c_int,
    c_int64,
    c_size_t,
    c_uint8,
    c_uint64,
    c_void_p,
)
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libqpb.so"

OK, INVALID_ARGUMENT, RUNTIME_ERROR, TIMEOUT = 0, 1, 2, 3

AMP_STORAGE = {"f32": 0, "f16": 1, "bf16": 2}
VARIANTS = {"batched": 0, "plain": 1, "half": 2, "mixed": 3}
SCHEDULES = {"auto": 0, "streamed": 1, "resident": 2, "persistent": 3}
OP_KINDS = {"er": 0, "hio": 1, "raar": 2, "shrinkwrap": 3, "detwin_begin": 4, "detwin_end": 5}
METHODS = {"max": 0, "rms": 1}

# Every function include/qpb.h declares.
EXPORTS = (
    "qpb_last_error",
    "qpb_cuda_available",
    "qpb_set_device",
    "qpb_device_info",
    "qpb_make_problem",
    "qpb_autocorrelation_support",
    "qpb_half_support",
    "qpb_create",
    "qpb_create_batch",
    "qpb_make_problem_device",
    "qpb_create_device",
    "qpb_results_device",
    "qpb_reset",
    "qpb_run",
    "qpb_set_wait_limit",
    "qpb_set_progress",
    "qpb_error_count",
    "qpb_starts",
    "qpb_results",
    "qpb_destroy",
    "qpb_kernel_launches",
    "qpb_tuning_report",
    "qpb_profile_passes",
    "qpb_amplitude_loss_grad",
    "qpb_project_support_bound",
    "qpb_modulus_project_noalloc",
    "qpb_aligned_error",
    "qpb_align",
    "qpb_simulate_intensity",
    "qpb_modulus_project",
    "qpb_support_project",
    "qpb_gaussian_blur",
)


class Problem(Structure):
    _fields_ = [
        ("ndim", c_int),
        ("shape", c_int64 * 3),
        ("amplitude", POINTER(c_float)),
        ("mask", POINTER(c_uint8)),
        ("support", POINTER(c_uint8)),
    ]


class Options(Structure):
    _fields_ = [
        ("starts", c_int),
        ("batch", c_int),
        ("seed", c_uint64),
        ("start", POINTER(c_float)),
        ("sync_every", c_int),
        ("variant", c_int),
        ("amp_storage", c_int),
        ("device", c_int),
        ("stream", c_void_p),
        ("schedule", c_int),
    ]


class Op(Structure):
    _fields_ = [
        ("kind", c_int),
        ("n", c_int),
        ("beta", c_float),
        ("threshold", c_float),
        ("sigma", c_float),
        ("method", c_int),
        ("axis", c_int),
    ]


PROGRESS = CFUNCTYPE(None, c_void_p, c_int, POINTER(c_float), c_int)

_lock = threading.Lock()
_lib = None


class ExtensionMissing(RuntimeError):
    pass


def load():
    """The loaded library; raises ExtensionMissing when it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIBRARY.exists():
            raise ExtensionMissing(
                f"{LIBRARY} is missing: build it with `python -m qoraphasecu_b200.build`"
            )
        lib = ctypes.CDLL(str(LIBRARY))
        lib.qpb_last_error.restype = c_char_p
        lib.qpb_last_error.argtypes = []
        lib.qpb_cuda_available.restype = c_int
        lib.qpb_cuda_available.argtypes = []
        lib.qpb_set_device.argtypes = [c_int]
        lib.qpb_device_info.argtypes = [c_char_p, c_size_t, POINTER(c_int), POINTER(c_int),
                                        POINTER(c_size_t), POINTER(c_size_t), POINTER(c_double)]
        lib.qpb_make_problem.argtypes = [c_void_p, c_int, POINTER(c_int64), c_void_p, c_void_p,
                                         c_float, c_void_p, c_void_p, c_void_p]
        lib.qpb_autocorrelation_support.argtypes = [c_void_p, c_int, POINTER(c_int64), c_float,
                                                    c_void_p]
        lib.qpb_half_support.argtypes = [c_void_p, c_int, POINTER(c_int64), c_int, c_void_p]
        lib.qpb_create.argtypes = [POINTER(Problem), POINTER(Options), POINTER(c_void_p)]
        lib.qpb_create_batch.argtypes = [POINTER(Problem), c_size_t, POINTER(Options),
                                         POINTER(c_void_p)]
        lib.qpb_make_problem_device.argtypes = [c_void_p, c_int, POINTER(c_int64), c_void_p,
                                                c_void_p, c_float, c_void_p, c_void_p, c_void_p,
                                                c_void_p]
        lib.qpb_create_device.argtypes = [POINTER(Problem), POINTER(Options), POINTER(c_void_p)]
        lib.qpb_results_device.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        lib.qpb_run.argtypes = [c_void_p, POINTER(Op), c_size_t]
        lib.qpb_reset.argtypes = [c_void_p, POINTER(Problem), c_size_t, c_uint64, c_void_p]
        lib.qpb_set_progress.argtypes = [c_void_p, PROGRESS, c_void_p]
        lib.qpb_set_wait_limit.argtypes = [c_void_p, c_int, c_int]
        lib.qpb_error_count.argtypes = [c_void_p, POINTER(c_size_t)]
        lib.qpb_starts.argtypes = [c_void_p, POINTER(c_int)]
        lib.qpb_results.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        lib.qpb_destroy.argtypes = [c_void_p]
        lib.qpb_destroy.restype = None
        lib.qpb_kernel_launches.argtypes = []
        lib.qpb_kernel_launches.restype = c_uint64
        lib.qpb_profile_passes.argtypes = [c_void_p, c_int, POINTER(c_double), POINTER(c_int)]
        lib.qpb_tuning_report.argtypes = [c_char_p, c_size_t]
        lib.qpb_modulus_project.argtypes = [POINTER(Problem), c_void_p, c_int, POINTER(c_float)]
        lib.qpb_amplitude_loss_grad.argtypes = [c_int, POINTER(c_int64), c_int, c_void_p,
                                                c_void_p, c_void_p, c_void_p, c_void_p]
        lib.qpb_project_support_bound.argtypes = [c_int64, c_int, c_void_p, c_float, c_void_p,
                                                  c_void_p]
        lib.qpb_modulus_project_noalloc.argtypes = [c_int, POINTER(c_int64), c_void_p, c_void_p,
                                                    c_void_p, c_void_p, c_void_p, c_void_p]
        lib.qpb_support_project.argtypes = [c_void_p, c_void_p, c_size_t]
        lib.qpb_aligned_error.argtypes = [c_void_p, c_void_p, c_int, POINTER(c_int64), c_int,
                                          c_void_p]
        lib.qpb_align.argtypes = [c_void_p, c_void_p, c_int, POINTER(c_int64), c_int, c_void_p,
                                  c_void_p, c_void_p]
        lib.qpb_simulate_intensity.argtypes = [c_void_p, c_int, POINTER(c_int64), c_void_p]
        lib.qpb_gaussian_blur.argtypes = [c_void_p, c_int, POINTER(c_int64), c_float, c_void_p]
        _lib = lib
        return lib


def check(status: int) -> None:
    """Raises the Python form of a qpb_status: ValueError for an invalid argument
    (the reference's std::invalid_argument), RuntimeError otherwise."""
    if status == OK:
        return
    message = load().qpb_last_error().decode(errors="replace")
    if status == INVALID_ARGUMENT:
        raise ValueError(message)
    if status == TIMEOUT:
        raise TimeoutError(message)
    raise RuntimeError(message)


def ptr(array):
    """Address of a C-contiguous numpy array (None for None)."""
    if array is None:
        return None
    return ctypes.c_void_p(array.ctypes.data)


def shape_arg(shape):
    return (c_int64 * 3)(*(list(shape) + [0] * (3 - len(shape))))
