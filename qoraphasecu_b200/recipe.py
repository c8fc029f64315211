"""Recipe stages with QoraPhase's names and defaults.

The same surface as the reference's ``python/qoraphasecu/recipe.py``: stages
flatten to 7-tuples ``(kind, n, beta, threshold, sigma, method, axis)``
(recipe.py:11-12 there), and ``repeat``/``detwin`` expand in place, so the
engine only ever walks a flat list (include/qoraphasecu/recipe.hpp:146-147).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Literal


def _op(kind, n=0, beta=0.0, threshold=0.0, sigma=0.0, method="max", axis=0):
    return (kind, n, beta, threshold, sigma, method, axis)


@dataclass(frozen=True)
class ER:
    """Error reduction: ``x <- P_S P_M x``."""

    n: int

    def ops(self):
        return [_op("er", self.n)]


@dataclass(frozen=True)
class HIO:
    """Hybrid input-output: ``P_M x`` inside the support, ``x - beta P_M x`` outside."""

    n: int
    beta: float = 0.9

    def ops(self):
        return [_op("hio", self.n, self.beta)]


@dataclass(frozen=True)
class RAAR:
    """Relaxed averaged alternating reflections: ``(beta/2)(R_S R_M x + x) + (1 - beta) P_M x``."""

    n: int
    beta: float = 0.9

    def ops(self):
        return [_op("raar", self.n, self.beta)]


@dataclass(frozen=True)
class Shrinkwrap:
    """New support: blurred magnitude above ``threshold`` times its max (or rms inside S)."""

    threshold: float = 0.3
    sigma: float = 1.0
    method: Literal["max", "rms"] = "max"

    def __post_init__(self):
        if self.method not in ("max", "rms"):
            raise ValueError(f"method must be 'max' or 'rms', got {self.method!r}")

    def ops(self):
        return [_op("shrinkwrap", threshold=self.threshold, sigma=self.sigma, method=self.method)]


class Recipe:
    """Stages in execution order."""

    def __init__(self, *stages):
        self.stages = tuple(stages)

    def __len__(self):
        return len(self.stages)

    def ops(self):
        out = []
        for stage in self.stages:
            out.extend(stage.ops())
        return out

    def iterations(self) -> int:
        return sum(o[1] for o in self.ops() if o[0] in ("er", "hio", "raar"))


@dataclass(frozen=True)
class _Repeat:
    n: int
    body: Recipe

    def ops(self):
        return self.body.ops() * self.n


@dataclass(frozen=True)
class _Detwin:
    body: Recipe
    axis: int

    def ops(self):
        return [_op("detwin_begin", axis=self.axis), *self.body.ops(), _op("detwin_end")]


def repeat(n: int, *stages) -> _Repeat:
    """``repeat(10, RAAR(50), Shrinkwrap())`` runs the stages ten times over."""
    return _Repeat(n, Recipe(*stages))


def detwin(*stages, axis: int = 0) -> _Detwin:
    """Runs ``stages`` on the support cut at its centre of mass along ``axis``, then restores it."""
    return _Detwin(Recipe(*stages), axis)


def default_recipe() -> Recipe:
    """QoraPhase's default: RAAR, a detwin pass, then shrinkwrapped RAAR, then ER (720 iterations)."""
    return Recipe(
        RAAR(50),
        detwin(HIO(20)),
        RAAR(50),
        repeat(8, RAAR(50), Shrinkwrap()),
        ER(200),
    )
