"""Seeded synthetic MR phantoms for the N4 workloads.

The reference ships no test volume (its ``N4.py`` test cell reads
``./testImage/shrink.nii.gz``, which is not in the repository), so every
workload here is generated from a seed:

* anatomy: three nested ellipsoids centred in the field of view with
  semi-axes 0.45 / 0.35 / 0.20 of the FOV along each axis, each semi-axis
  jittered by a factor U(0.9, 1.1); tissue intensities 0.35 / 0.70 / 1.00
  from the outer to the inner ellipsoid; background 0;
* bias: the clean image is multiplied by ``exp(b)`` where ``b`` is a cubic
  B-spline on a ``g x g x g`` control grid with N(0, s^2) coefficients,
  evaluated with the same span/weight convention as the fit;
* noise: Rician, ``|x + sigma (n1 + i n2)|`` with standard normal n1, n2;
* mask: the outer ellipsoid.

All draws come from ``numpy.random.default_rng(seed)`` (PCG64), in a fixed
order, so a phantom is identical on every machine.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Phantom", "make_phantom", "bspline_field", "CONFIGS", "batch_dims"]


def _axis_weights(size: int, ncpt: int) -> np.ndarray:
    """Dense (size x ncpt) cubic B-spline weight matrix along one axis."""
    nspans = ncpt - 3
    span = np.float64(size) / np.float64(nspans)
    i = np.arange(size, dtype=np.float64)
    s = np.floor((i + 0.5) / span).astype(np.int64)
    t = ((i + 0.5) - s * span) / span
    w = np.stack([(1 - t) ** 3 / 6, (3 * t ** 3 - 6 * t ** 2 + 4) / 6,
                  (-3 * t ** 3 + 3 * t ** 2 + 3 * t + 1) / 6, t ** 3 / 6], axis=1)
    M = np.zeros((size, ncpt))
    M[np.repeat(np.arange(size), 4), (s[:, None] + np.arange(4)).ravel()] = w.ravel()
    return M


def bspline_field(coeffs: np.ndarray, shape) -> np.ndarray:
    """Evaluate a cubic B-spline control lattice densely on ``shape``."""
    X, Y, Z = shape
    cx, cy, cz = coeffs.shape
    t = np.tensordot(coeffs, _axis_weights(Z, cz), axes=([2], [1]))
    t = np.tensordot(t, _axis_weights(Y, cy), axes=([1], [1]))
    t = np.tensordot(t, _axis_weights(X, cx), axes=([0], [1]))
    return np.ascontiguousarray(t.transpose(2, 1, 0))


@dataclass
class Phantom:
    im: np.ndarray        # float32 [X][Y][Z], z fastest
    mask: np.ndarray      # float32, 1 inside the outer ellipsoid
    log_bias: np.ndarray  # float64 true log bias field
    seed: int


def make_phantom(shape, seed: int, sigma: float = 0.03, grid: int = 4,
                 coeff_std: float = 0.15) -> Phantom:
    X, Y, Z = (int(d) for d in shape)
    rng = np.random.default_rng(seed)
    jitter = rng.uniform(0.9, 1.1, size=(3, 3))
    coeffs = rng.normal(0.0, coeff_std, size=(grid, grid, grid))
    u = [(np.arange(n, dtype=np.float64) + 0.5) / n - 0.5 for n in (X, Y, Z)]
    clean = np.zeros((X, Y, Z), dtype=np.float64)
    mask = None
    for k, (radius, value) in enumerate(((0.45, 0.35), (0.35, 0.70), (0.20, 1.00))):
        r = radius * jitter[k]
        d = ((u[0] / r[0]) ** 2)[:, None, None] + ((u[1] / r[1]) ** 2)[None, :, None] \
            + ((u[2] / r[2]) ** 2)[None, None, :]
        inside = d <= 1.0
        clean[inside] = value
        if k == 0:
            mask = inside
    log_bias = bspline_field(coeffs, (X, Y, Z))
    biased = (clean * np.exp(log_bias)).astype(np.float32)
    n1 = rng.standard_normal((X, Y, Z), dtype=np.float32)
    n2 = rng.standard_normal((X, Y, Z), dtype=np.float32)
    s = np.float32(sigma)
    im = np.sqrt((biased + s * n1) ** 2 + (s * n2) ** 2).astype(np.float32)
    return Phantom(im=im, mask=mask.astype(np.float32), log_bias=log_bias, seed=seed)


# The five workloads (shapes, generator settings and N4 parameters).
CONFIGS = {
    "c1": dict(shape=(64, 64, 48), sigma=0.03, grid=4, coeff_std=0.15, shrink=1,
               levels=3, iterations=50, threshold=0.0),
    "c2": dict(shape=(256, 256, 176), sigma=0.02, grid=6, coeff_std=0.25, shrink=4,
               levels=4, iterations=50, threshold=0.001),
    "c3": dict(shape=(512, 512, 320), sigma=0.02, grid=8, coeff_std=0.25, shrink=2,
               levels=4, iterations=50, threshold=0.001),
    "c4": dict(n=48, sigma=0.03, grid=4, coeff_std=0.15, shrink=4, levels=4,
               iterations=50, threshold=0.001),
}


def batch_dims(n: int, seed: int):
    """Per-volume shapes of the batched workload: every axis drawn uniformly
    from 96, 104, ..., 288."""
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.choice(np.arange(96, 289, 8), size=3)) for _ in range(n)]
