"""QoraPhase B200 backend: iterative phase retrieval as hand-written sm_100a kernels.

Array in, reconstruction out, with the surface of the reference's
``qoraphasecu`` package::

    import qoraphasecu_b200 as qpc
    result = qpc.reconstruct(intensity, support=support)

All public arrays are centre-origin, ``mask=True`` marks an unusable pixel and
``intensity`` is a measured intensity. Every call runs on the GPU through
``libqpb.so`` (include/qpb.h); there is no CPU path.
"""

from .api import (
    BatchSolver,
    Ensemble,
    Problem,
    Reconstruction,
    Solver,
    align,
    aligned_error,
    autocorrelation_support,
    best_index,
    cuda_available,
    half_support,
    kernel_launches,
    make_problem,
    reconstruct,
    reconstruct_batch,
    set_device,
    simulate_intensity,
)
from .operators import gaussian_blur, modulus_project, support_project
from .recipe import ER, HIO, RAAR, Recipe, Shrinkwrap, default_recipe, detwin, repeat

__all__ = [
    "BatchSolver",
    "ER",
    "HIO",
    "RAAR",
    "Ensemble",
    "Problem",
    "Recipe",
    "Reconstruction",
    "Shrinkwrap",
    "Solver",
    "align",
    "aligned_error",
    "autocorrelation_support",
    "best_index",
    "cuda_available",
    "default_recipe",
    "detwin",
    "gaussian_blur",
    "half_support",
    "make_problem",
    "modulus_project",
    "reconstruct",
    "reconstruct_batch",
    "repeat",
    "simulate_intensity",
    "support_project",
]
