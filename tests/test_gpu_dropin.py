"""The B200 backend behind the reference's own C++ API.

oracle/_ref/libqpcu_dropin.so is QoraPhaseCU's core and CPU path compiled
unchanged from its sources, with its Backend::cuda factory slot bound to the
C++ adapter qoraphasecu_b200/adapter/b200_solver.cpp (a qpcu::Solver over
libqpb.so). So qpcu::make_solver, qpcu::reconstruct and qpcu::best_index
(src/core/solver.cpp:61-103 in the reference) run the B200 backend with
Options::backend = cuda, and the reference's CpuSolver with backend = cpu, in
one process. The checks follow the reference's CUDA-vs-CPU tests
(tests/test_cuda.cpp:66-87: per-iteration errors within 1e-3 relative plus
1e-6, objects within 1e-3, supports exact; here 1e-4) and its recovery test
on the default recipe (test_recover.cpp:69-76).
"""

import ctypes

import numpy as np
import pytest

from oracle import fp64, ref
from synthetic import readme_triangle, triangle

from qoraphasecu_b200 import workloads
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe, Shrinkwrap, default_recipe, detwin

pytestmark = pytest.mark.gpu

CPU, B200 = 0, 1


@pytest.fixture(scope="module")
def lib(gpu):
    lib = ref.load_variant("dropin")
    assert lib.qref_cuda_available() == 1
    return lib


def _status(lib, status):
    if status:
        raise (ValueError if status == 1 else RuntimeError)(lib.qref_last_error().decode())


def _made(lib, intensity, support=None, mask=None):
    amp = np.empty(intensity.shape, np.float32)
    m = np.empty(intensity.shape, np.uint8)
    s = np.empty(intensity.shape, np.uint8)
    sup = None if support is None else np.ascontiguousarray(support, np.uint8)
    msk = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    _status(lib, lib.qref_make_problem(ref._p(np.ascontiguousarray(intensity, np.float32)),
                                       intensity.ndim, ref._shape(intensity.shape), ref._p(sup),
                                       ref._p(msk), ctypes.c_float(0.1), ref._p(amp), ref._p(m),
                                       ref._p(s)))
    return amp, m, s


def _reconstruct(lib, problem, recipe, starts, seed, backend):
    amp, mask, support = problem
    ops = recipe.ops()
    arr = ref._ops(ops)
    iters = recipe.iterations()
    n = amp.size
    objects = np.empty((starts, *amp.shape), np.complex64)
    supports = np.empty((starts, *amp.shape), np.uint8)
    errors = np.empty((starts, iters), np.float32)
    best = ctypes.c_int(-1)
    _status(lib, lib.qref_reconstruct(ref._p(amp), ref._p(mask), ref._p(support), amp.ndim,
                                      ref._shape(amp.shape), arr, len(ops), starts,
                                      ctypes.c_uint64(seed), backend, ref._p(objects),
                                      ref._p(supports), ref._p(errors), ctypes.byref(best)))
    assert objects.size == starts * n
    return objects, supports.astype(bool), errors, best.value


def test_short_recipe_through_make_solver_matches_the_cpu_backend(lib):
    _, support, intensity = triangle((64, 48), 16)
    problem = _made(lib, intensity, support)
    recipe = Recipe(HIO(15), Shrinkwrap(), RAAR(10), detwin(HIO(5)), ER(10))
    cpu = _reconstruct(lib, problem, recipe, 2, 3, CPU)
    gpu = _reconstruct(lib, problem, recipe, 2, 3, B200)
    for s in range(2):
        np.testing.assert_allclose(gpu[2][s], cpu[2][s], rtol=1e-4, atol=1e-6)
        assert fp64.relative_diff(gpu[0][s], cpu[0][s]) < 1e-4
        np.testing.assert_array_equal(gpu[1][s], cpu[1][s])


def test_default_recipe_and_best_index_on_the_readme_object(lib):
    """qpcu::reconstruct(problem, default_recipe(), {.backend, .starts = 8}) and
    qpcu::best_index on both backends: the best runs agree within 1e-4 in final
    Fourier error and in aligned object error, and recover the object."""
    obj, _, intensity = readme_triangle()
    problem = _made(lib, intensity)
    out = {}
    for backend in (CPU, B200):
        objects, _, errors, best = _reconstruct(lib, problem, default_recipe(), 8, 0, backend)
        assert errors.shape == (8, 720)
        assert best == int(np.argmin(errors[:, -1]))
        out[backend] = (errors[best, -1], fp64.aligned_error(objects[best], obj))
    assert out[B200][0] < 1e-3 and out[B200][1] < 1e-2
    assert abs(out[B200][0] - out[CPU][0]) < 1e-4
    assert abs(out[B200][1] - out[CPU][1]) < 1e-4


def test_default_recipe_on_the_square_object(lib):
    """The 64 x 64 random square (uniform amplitude and phase in a 24 x 24 box,
    autocorrelation support, 8 starts): 720 iterations from random starts are
    chaotic on this object (the FP32 and FP64 CPU ports land far apart), so the
    B200 best run is checked to fall inside the reference CPU backend's
    ensemble: no worse than its median final error."""
    square = workloads.square(64, seed=0)
    intensity = workloads.simulate_intensity(square)
    problem = _made(lib, intensity)
    cpu = _reconstruct(lib, problem, default_recipe(), 8, 0, CPU)
    gpu = _reconstruct(lib, problem, default_recipe(), 8, 0, B200)
    assert np.all(np.isfinite(gpu[2]))
    assert gpu[3] == int(np.argmin(gpu[2][:, -1]))
    assert gpu[2][gpu[3], -1] <= np.median(cpu[2][:, -1])


def test_reference_exceptions_come_through_the_adapter(lib):
    _, support, intensity = triangle((32, 32), 8)
    amp, mask, sup = _made(lib, intensity, support)
    handle = ctypes.c_void_p()
    # make_solver's own validation (solver.cpp:62-78)
    status = lib.qref_create_backend(ref._p(amp), ref._p(mask), ref._p(sup), 2,
                                     ref._shape(amp.shape), 4, ctypes.c_uint64(0), None, 10, B200,
                                     3, 3, ctypes.byref(handle))
    assert status == 1 and "batch" in lib.qref_last_error().decode()
    # a recipe the B200 backend refuses: detwin along an axis the problem lacks
    status = lib.qref_create_backend(ref._p(amp), ref._p(mask), ref._p(sup), 2,
                                     ref._shape(amp.shape), 2, ctypes.c_uint64(0), None, 10, B200,
                                     3, 0, ctypes.byref(handle))
    assert status == 0
    try:
        arr = ref._ops(Recipe(detwin(ER(1), axis=2)).ops())
        assert lib.qref_run(handle, arr, 3) == 1
    finally:
        lib.qref_destroy(handle)
