"""Generate golden vectors by running the reference's own ``N4.py``.

Run in a container where the reference checkout is available::

    python tests/golden/make_golden.py [--reference /path/to/CUDA-N4] [--c1]

``N4.py`` imports ``nibabel`` and ``matplotlib`` (unused by its functions)
and ends in a script cell that reads a test image the repository does not
ship; the loader below stubs the two modules and executes only the function
definitions (``N4.py:1-334``).  Nothing from the reference is copied into
this repository: only its outputs on seeded phantoms are stored.

Outputs (``tests/golden/``):

* ``components.npz`` - ``sharpenImage``, ``FitBspline3D``,
  ``EvaluateBspline3D``, ``UpsampleLattice3D``, ``cubicBspline`` and
  ``CalculateConvergenceMeasurement`` on small seeded inputs;
* ``n4_small.npz`` - whole ``N4`` runs on small phantoms (fixed iteration
  counts and a thresholded run);
* ``n4_c1.npz`` (``--c1``, about 15 minutes) - ``N4`` on the 64x64x48
  phantom, 3 levels x 50 iterations: final lattice, per-level iteration
  counts and summary statistics of the corrected volume.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cuda-n4_b200"))
from n4b200.phantom import make_phantom  # noqa: E402


def load_reference(path: str) -> dict:
    for name in ("nibabel", "matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    src = open(os.path.join(path, "N4.py")).read()
    cut = src.index("#%% Test the N4 algorithm")
    ns: dict = {"__name__": "reference_N4"}
    exec(compile(src[:cut], os.path.join(path, "N4.py"), "exec"), ns)
    return ns


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def components(ref) -> dict:
    out = {}
    ph = make_phantom((24, 20, 16), seed=11, sigma=0.03, grid=4, coeff_std=0.2)
    mask = ph.mask.astype(np.float64)
    with np.errstate(divide="ignore"):
        logim = np.where(mask != 0, np.log(ph.im.astype(np.float64)), 0.0)
    out["sharp_in"], out["sharp_mask"] = logim, mask
    for fwhm, tag in ((0.15, "a"), (0.3, "b")):
        for bins in (200, 64):
            out[f"sharp_out_{tag}{bins}"] = ref["sharpenImage"](logim, mask, bins, 0.01, fwhm)
    rng = np.random.default_rng(12)
    # fit / evaluate on shapes that include exact span boundaries (44 / 8 = 5.5)
    for k, (shape, ncpt) in enumerate((((24, 20, 16), (4, 4, 4)),
                                       ((22, 12, 44), (5, 7, 11)),
                                       ((17, 9, 13), (6, 4, 5)))):
        field = rng.normal(0.0, 0.3, size=shape)
        fmask = (rng.uniform(size=shape) > 0.2).astype(np.float64)
        out[f"fit_field_{k}"], out[f"fit_mask_{k}"] = field, fmask
        out[f"fit_ncpt_{k}"] = np.array(ncpt)
        out[f"fit_out_{k}"] = ref["FitBspline3D"](field, fmask, ncpt)
        lat = rng.normal(0.0, 0.5, size=ncpt)
        out[f"eval_lat_{k}"] = lat
        out[f"eval_out_{k}"] = ref["EvaluateBspline3D"](lat, ncpt, np.array(shape))
    for n in (4, 5, 7):
        lat = rng.normal(0.0, 1.0, size=(n, n, n))
        out[f"up_in_{n}"] = lat
        out[f"up_out_{n}"] = ref["UpsampleLattice3D"](lat)
    t = np.linspace(0.0, 1.0, 11)
    out["bspline_t"] = t
    out["bspline_w"] = np.stack([ref["cubicBspline"](v) for v in t])
    f1 = rng.normal(0.0, 0.05, size=(12, 10, 8))
    f2 = rng.normal(0.0, 0.05, size=(12, 10, 8))
    cm = (rng.uniform(size=(12, 10, 8)) > 0.3).astype(np.float64)
    out["cv_f1"], out["cv_f2"], out["cv_mask"] = f1, f2, cm
    out["cv_out"] = np.array(ref["CalculateConvergenceMeasurement"](f1, f2, cm))
    return out


# threshold of the "thresh" case, chosen so that every level stops on it with
# a margin of >= 1% between the last two convergence values and the threshold
THRESH = 0.0027


def n4_small(ref) -> dict:
    out = {}
    cases = [
        ("fixed", (40, 36, 32), 21, 2, [3, 2], 0.0),
        ("thresh", (40, 40, 32), 22, 3, [6, 4, 3], THRESH),
    ]
    for tag, shape, seed, levels, iters, thr in cases:
        ph = make_phantom(shape, seed=seed, sigma=0.03, grid=4, coeff_std=0.2)
        with np.errstate(divide="ignore", invalid="ignore"):
            norm, lat = quiet(ref["N4"], ph.im.astype(np.float64), ph.mask.astype(np.float64),
                              low_value=0, maximumNumberOfLevels=levels,
                              maximumNumberOfIterations=iters, ConvergenceThreshold=thr)
        out[f"{tag}_im"], out[f"{tag}_mask"] = ph.im, ph.mask
        out[f"{tag}_levels"], out[f"{tag}_iters"] = np.array(levels), np.array(iters)
        out[f"{tag}_thr"] = np.array(thr)
        out[f"{tag}_norm"], out[f"{tag}_lattice"] = norm, lat
    return out


def n4_c1(ref) -> dict:
    ph = make_phantom((64, 64, 48), seed=1, sigma=0.03, grid=4, coeff_std=0.15)
    buf = io.StringIO()
    t0 = time.time()
    with contextlib.redirect_stdout(buf), np.errstate(divide="ignore", invalid="ignore"):
        norm, lat = ref["N4"](ph.im.astype(np.float64), ph.mask.astype(np.float64),
                              low_value=0, maximumNumberOfLevels=3,
                              maximumNumberOfIterations=[50, 50, 50],
                              ConvergenceThreshold=0.0)
    lines = [ln for ln in buf.getvalue().splitlines() if ln.startswith("Level")]
    iters = [sum(1 for ln in lines if ln.startswith(f"Level {lv},")) for lv in range(3)]
    m = ph.mask != 0
    return dict(seed=np.array(1), lattice=lat, iterations=np.array(iters),
                norm_sum_mask=np.array(norm[m].sum()), norm_sum=np.array(norm.sum()),
                norm_sample=norm.reshape(-1)[::97].copy(),
                seconds=np.array(time.time() - t0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("N4_REFERENCE_DIR"),
                    help="checkout of JiancongWang/CUDA-N4 holding N4.py (or set N4_REFERENCE_DIR)")
    ap.add_argument("--c1", action="store_true")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference <checkout of the reference> or set N4_REFERENCE_DIR")
    ref = load_reference(a.reference)
    if a.c1:
        np.savez_compressed(os.path.join(HERE, "n4_c1.npz"), **n4_c1(ref))
        return
    np.savez_compressed(os.path.join(HERE, "components.npz"), **components(ref))
    np.savez_compressed(os.path.join(HERE, "n4_small.npz"), **n4_small(ref))


if __name__ == "__main__":
    main()
