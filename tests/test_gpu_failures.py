"""Failure paths, made to happen without faulting the GPU.

The reference turns CUDA and cuFFT failures into std::runtime_error
(src/cuda/common.cuh:15-31) and bad inputs into std::invalid_argument; at the C
ABI those are QPB_RUNTIME_ERROR and QPB_INVALID_ARGUMENT. This backend adds
bounded device waits (QPB_TIMEOUT): a line pass that stages its inputs by bulk
copies gives up after a number of polls, writes nothing and counts itself in
its solver's counter.

* Timeout: a solver whose staged copies are left out (fault injection through
  qpb_set_wait_limit, on valid memory, with a short poll limit) reports
  QPB_TIMEOUT from qpb_run; the device stays usable, and after a reset the same
  solver reproduces a fresh solver's results bit for bit. The failure is
  charged to that solver only: another solver run in between reports nothing.
* Allocation failure: a solver far larger than any GPU's memory is refused
  with QPB_RUNTIME_ERROR (cudaMalloc fails; nothing is launched), and the next
  call works.
* Caller pointers that bulk copies would read must be 16-byte aligned: the
  amplitude-loss entry point refuses a misaligned view before launching.
"""

import ctypes

import numpy as np
import pytest

from synthetic import triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import _lib
from qoraphasecu_b200.recipe import ER, HIO, Recipe

pytestmark = pytest.mark.gpu


def _problem(n=64, m=20):
    _, support, intensity = triangle((n, n), m)
    return qpc.make_problem(intensity, support=support)


@pytest.mark.parametrize("variant", ["batched", "plain"])
def test_starved_waits_time_out_and_the_solver_recovers(gpu, variant):
    problem = _problem()
    recipe = Recipe(HIO(6), ER(4))
    with qpc.Solver(problem, starts=4, seed=3, sync_every=5, variant=variant,
                    schedule="streamed" if variant == "batched" else "auto") as s:
        s.set_wait_limit(64, starve=True)
        with pytest.raises(TimeoutError, match="gave up"):
            s.run(recipe)
        # another solver meanwhile sees no failure of this one
        with qpc.Solver(problem, starts=2, seed=1) as other:
            other.run(Recipe(ER(3)))
        s.set_wait_limit(1 << 22, starve=False)
        s.reset(problem, seed=3)
        s.run(recipe)
        recovered = s.results()
    with qpc.Solver(problem, starts=4, seed=3, sync_every=5, variant=variant) as fresh:
        fresh.run(recipe)
        expected = fresh.results()
    for a, b in zip(recovered, expected, strict=True):
        np.testing.assert_array_equal(a.object, b.object)
        np.testing.assert_array_equal(a.errors, b.errors)


def test_wait_limit_is_validated(gpu):
    with qpc.Solver(_problem(32, 8), starts=1) as s:
        with pytest.raises(ValueError):
            s.set_wait_limit(0)


def test_allocation_failure_is_a_runtime_error_and_the_library_recovers(gpu):
    lib = _lib.load()
    problem = _problem(1024, 200)
    options = _lib.Options(starts=2_000_000, batch=2_000_000, seed=0, start=None, sync_every=10,
                           variant=0, amp_storage=0, device=-1, stream=None,
                           schedule=_lib.SCHEDULES["streamed"])
    handle = ctypes.c_void_p()
    before = lib.qpb_kernel_launches()
    status = lib.qpb_create(ctypes.byref(problem._c()), ctypes.byref(options),
                            ctypes.byref(handle))
    assert status == _lib.RUNTIME_ERROR
    assert "memory" in lib.qpb_last_error().decode().lower()
    assert not handle.value
    assert lib.qpb_kernel_launches() == before
    # the failed allocation leaves no error behind for the next launch
    run = qpc.reconstruct(*_triangle_args(), recipe=Recipe(ER(3)))
    assert np.isfinite(run.error)


def _triangle_args():
    _, support, intensity = triangle((32, 32), 8)
    return (intensity,)


def test_misaligned_gradient_arrays_are_refused(gpu):
    import torch

    lib = _lib.load()
    shape = (32, 32)
    buf = torch.zeros(2 * (1024 + 1), dtype=torch.float32, device="cuda")
    odd = buf[2:2 + 2048]
    assert odd.data_ptr() % 16 == 8
    amp = torch.ones(1024, dtype=torch.float32, device="cuda")
    grad = torch.zeros(2048, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    before = lib.qpb_kernel_launches()
    status = lib.qpb_amplitude_loss_grad(2, _lib.shape_arg(shape), 1, ctypes.c_void_p(amp.data_ptr()),
                                         ctypes.c_void_p(odd.data_ptr()),
                                         ctypes.c_void_p(grad.data_ptr()),
                                         ctypes.c_void_p(loss.data_ptr()), None)
    assert status == _lib.INVALID_ARGUMENT
    assert "aligned" in lib.qpb_last_error().decode()
    assert lib.qpb_kernel_launches() == before
