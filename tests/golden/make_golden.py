"""Regenerates tests/golden/*.npz from the reference's own CPU path.

    make -C oracle && python tests/golden/make_golden.py

The outputs come from oracle/_ref/libqpcu_ref.so: QoraPhaseCU's src/core and
src/cpu sources compiled unchanged, with oracle/fft_shim.cpp in place of the
absent pocketfft. Inputs are the reference test suite's synthetic objects
(tests/synthetic.hpp) and fixed seeds, so the fixtures pin the reference's
behaviour for the parity tests wherever the reference sources are absent.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

from oracle import fp64, ref  # noqa: E402
from synthetic import random_field, readme_triangle, triangle  # noqa: E402

SHORT_RECIPE = [fp64.op("hio", 15, 0.9), fp64.op("shrinkwrap", threshold=0.3, sigma=1.0),
                fp64.op("raar", 10, 0.9), fp64.op("detwin_begin"), fp64.op("hio", 5, 0.9),
                fp64.op("detwin_end"), fp64.op("er", 10)]


def operators():
    out = {}
    _, support, intensity = triangle((48, 40), 12)
    mask = np.zeros((48, 40), np.uint8)
    mask.flat[5] = 1
    problem = ref.make_problem(intensity, support, mask)
    x = random_field(48 * 40, 5).reshape(48, 40)
    projected, err = ref.modulus_project(problem, x)
    out.update(mp_intensity=intensity, mp_support=support, mp_mask=mask, mp_x=x,
               mp_out=projected, mp_err=np.float32(err))
    rng = np.random.default_rng(3)
    image = rng.random((16, 20, 12)).astype(np.float32)
    out.update(blur_image=image, blur_sigma=np.float32(1.0),
               blur_out=ref.gaussian_blur(image, 1.0))
    _, sup2, inten2 = triangle((64, 48), 16)
    out.update(half_support=sup2, half_axis0=ref.half_support(sup2, 0),
               half_axis1=ref.half_support(sup2, 1))
    out.update(ac_intensity=inten2, ac_support=ref.autocorrelation_support(inten2, 0.1))
    return out


def short_recipe():
    _, support, intensity = triangle((64, 48), 16)
    runs = ref.reconstruct(ref.make_problem(intensity, support), SHORT_RECIPE, starts=2, seed=3)
    return dict(intensity=intensity, support=support,
                objects=np.stack([r[0] for r in runs]),
                supports=np.stack([r[1] for r in runs]).astype(np.uint8),
                errors=np.stack([r[2] for r in runs]))


def default_recipe():
    obj, _, intensity = readme_triangle()
    runs = ref.reconstruct(ref.make_problem(intensity), fp64.default_recipe(), starts=8)
    errors = np.array([r[2][-1] for r in runs], np.float32)
    best = int(np.argmin(errors))
    return dict(intensity=intensity, truth=obj, final_errors=errors, best=np.int64(best),
                best_object=runs[best][0],
                best_aligned=np.float32(ref.aligned_error(runs[best][0], obj)))


def main():
    if not ref.available():
        raise SystemExit("oracle/_ref/libqpcu_ref.so is missing: run `make -C oracle` first")
    np.savez_compressed(HERE / "operators.npz", **operators())
    np.savez_compressed(HERE / "short_recipe.npz", **short_recipe())
    np.savez_compressed(HERE / "default_recipe.npz", **default_recipe())
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
