"""The reference's own CUDA backend, compiled from its sources by
oracle/Makefile (oracle/_ref/libqpcu_ref_cuda.so), is the GPU baseline the
benchmark times beside this backend. This checks that the build computes what
the reference's CPU backend computes on the benchmark problem, as the
reference's own tests/test_cuda.cpp:66-87 does (per-iteration errors within
1e-3 relative plus 1e-6; here 1e-4), for the variants the benchmark times."""

import ctypes

import numpy as np
import pytest

from oracle import ref

from qoraphasecu_b200 import workloads
from qoraphasecu_b200.recipe import RAAR, Recipe

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["graph", "batched"])
def test_reference_cuda_build_matches_its_cpu_backend(gpu, variant):
    lib = ref.load_variant("cuda")
    assert lib.qref_cuda_available() == 1
    _, intensity, mask = workloads.gaussians(256, seed=1000)
    amp, msk, sup = ref.make_problem(intensity, None, mask)
    ops = Recipe(RAAR(3, 0.9)).ops()
    arr = ref._ops(ops)
    errors = {}
    for backend, v in ((0, 3), (1, {"graph": 2, "batched": 3}[variant])):
        handle = ctypes.c_void_p()
        assert lib.qref_create_backend(ref._p(amp), ref._p(msk), ref._p(sup), 2,
                                       ref._shape(amp.shape), 4, ctypes.c_uint64(0), None, 10,
                                       backend, v, 0, ctypes.byref(handle)) == 0, \
            lib.qref_last_error().decode()
        try:
            assert lib.qref_run(handle, arr, len(ops)) == 0, lib.qref_last_error().decode()
            e = np.empty((4, 3), np.float32)
            assert lib.qref_results(handle, None, None, ref._p(e),
                                    ctypes.byref(ctypes.c_size_t())) == 0
            errors[backend] = e
        finally:
            lib.qref_destroy(handle)
    np.testing.assert_allclose(errors[1], errors[0], rtol=1e-4, atol=1e-6)
