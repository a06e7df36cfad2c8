"""FP64 CPU oracle for the N4 bias-field correction path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it is imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the CPU-baseline legs of
``bench.py``.  The product (``libn4b200.so`` and the ``n4b200`` package) never
imports, links or calls it.

It restates the reference's numpy implementation ``N4.py`` function for
function, vectorised so that the full-size configurations finish in seconds
instead of the tens of minutes the per-voxel Python loops of ``N4.py`` need:

=============================  =====================================
oracle function                reference
=============================  =====================================
``sharpenImage``               ``N4.py:9-118``
``CalculateConvergenceMeasurement``  ``N4.py:121-126``
``UpsampleLattice3D``          ``N4.py:132-165`` (and ``cudaN4.cu:995-1084``)
``cubicBspline``               ``N4.py:174-181``
``FitBspline3D``               ``N4.py:186-237``
``EvaluateBspline3D``          ``N4.py:241-273``
``N4``                         ``N4.py:276-332``
=============================  =====================================

Arithmetic is IEEE FP64 except where ``N4.py`` itself drops to single
precision: its smoothing numerator is a ``complex64`` array
(``N4.py:75``) whose forward FFT numpy 2.x evaluates in single precision.
The oracle reproduces that quirk so that it agrees with ``N4.py`` to
round-off.

Parity pin: ``tests/golden/*.npz`` hold outputs of ``N4.py`` itself (imported
with its unused ``nibabel``/``matplotlib`` imports stubbed) on seeded
phantoms; ``tests/test_oracle_golden.py`` checks every function here against
them.  The generating script is ``tests/golden/make_golden.py``.

Extensions beyond ``N4.py`` (all default to ``N4.py`` behaviour):

* ``cv_ddof=1`` selects the ``N - 1`` standard deviation of the CUDA
  reference (``cudaN4.cu:979``); ``fit_zero_den=True`` selects its
  ``den != 0 ? num/den : 0`` fit division (``cudaN4.cu:123-127``).
* ``N4`` accepts per-level iteration counts, the histogram/filter parameters
  that ``N4.py`` hard-codes at ``N4.py:307-311``, an initial control-point
  grid other than 4x4x4 (``N4.py:292``) and a warm-start lattice.
* ``N4Shrink`` adds the shrink factor that the reference lacks: a block
  reduction of the thresholded volume before fitting and a final evaluation
  of the lattice at full resolution.
"""
from __future__ import annotations

import numpy as np
from numpy.fft import fft, ifft

__all__ = [
    "padded_histogram_size", "histogram", "sharpening_map", "sharpenImage",
    "CalculateConvergenceMeasurement", "UpsampleLattice3D", "cubicBspline",
    "axis_tables", "FitBspline3D", "FitBspline3D_literal", "EvaluateBspline3D",
    "EvaluateBspline3D_literal", "N4", "N4Shrink", "shrink_volume",
    "lattice_dims",
]


# --------------------------------------------------------------------------
# histogram sharpening (N4.py:9-118)
# --------------------------------------------------------------------------
def padded_histogram_size(bins: int) -> tuple[int, int]:
    """Padded FFT length and histogram offset, ``N4.py:32-37``."""
    exponent = np.ceil(np.log(bins) / np.log(2.0)) + 1
    padded = int(2.0 ** exponent + 0.5)
    offset = int(0.5 * (padded - bins))
    return padded, offset


def histogram(x: np.ndarray, bins: int):
    """Fractional (linearly split) histogram of the masked values ``x``.

    ``N4.py:14-29``.  Returns ``(H, binMin, binMax, slope)``.  Contributions
    are accumulated in voxel order, exactly as the reference loop does, so
    the result is bitwise the reference's.  A voxel whose bin index is the
    last bin with a non-zero offset is dropped, as in the reference.
    """
    binMin, binMax = x.min(), x.max()
    slope = (binMax - binMin) / (bins - 1)
    cidx = (x - binMin) / slope
    idx = np.floor(cidx).astype(np.int64)
    off = cidx - idx
    zero = off == 0.0
    split = (~zero) & (idx < bins - 1)
    w0 = np.where(zero, 1.0, np.where(split, 1.0 - off, 0.0))
    w1 = np.where(split, off, 0.0)
    b = np.stack([idx, idx + 1], axis=1).ravel()
    w = np.stack([w0, w1], axis=1).ravel()
    b = np.clip(b, 0, bins)  # a dropped or exact-top voxel has weight 0 at idx+1
    H = np.bincount(b, weights=w, minlength=bins + 1)[:bins]
    return H, binMin, binMax, slope


def sharpening_map(H: np.ndarray, binMin, slope, WienerFilterNoise=0.01,
                   BiasFieldFullWidthAtHalfMaximium=0.15):
    """Gaussian Wiener deconvolution of the histogram and the intensity map
    ``E`` (one value per bin), ``N4.py:32-101``."""
    bins = H.shape[0]
    padded, offset = padded_histogram_size(bins)
    V = np.zeros(padded)
    V[offset:offset + bins] = H
    Vf = fft(V)

    scaledFWHM = BiasFieldFullWidthAtHalfMaximium / slope
    expFactor = 4.0 * np.log(2.0) / (scaledFWHM * scaledFWHM)
    scaleFactor = 2.0 * np.sqrt(np.log(2.0) / np.pi) / scaledFWHM
    F = np.zeros(padded)
    F[0] = scaleFactor
    half = int(0.5 * padded)
    i = np.arange(1, half + 1, dtype=np.float64)
    g = scaleFactor * np.exp(-i * i * expFactor)
    F[1:half + 1] = g
    F[padded - np.arange(1, half + 1)] = g
    if padded % 2 == 0:
        F[half] = scaleFactor * np.exp(-0.25 * padded * padded * expFactor)
    Ff = fft(F)
    c = np.conj(Ff)
    Gf = c / (c * Ff + WienerFilterNoise)
    Uf = Vf * np.real(Gf)
    U = np.real(ifft(Uf))
    U[U < 0] = 0

    centers = binMin + (np.arange(padded) - offset) * slope
    numerator = (centers * U).astype(np.complex64)       # N4.py:75-78
    numerator = ifft(fft(numerator) * Ff)
    denominator = ifft(fft(U) * Ff)
    nu = numerator.real
    de = denominator.real
    E = np.zeros(padded)
    nz = de != 0
    E[nz] = nu[nz] / de[nz]
    return E[offset:offset + bins]


def remap(x: np.ndarray, E: np.ndarray, binMin, slope) -> np.ndarray:
    """Piecewise-linear intensity remap through ``E``, ``N4.py:105-113``."""
    bins = E.shape[0]
    cidx = (x - binMin) / slope
    idx = np.floor(cidx).astype(np.int64)
    lo = np.clip(idx, 0, bins - 2)
    lerp = E[lo] + (E[lo + 1] - E[lo]) * (cidx - idx)
    return np.where(idx < bins - 1, lerp, E[-1])


def sharpenImage(im_before_sharpen, mask, numberOfHistogramBins=200,
                 WienerFilterNoise=0.01, BiasFieldFullWidthAtHalfMaximium=1.5,
                 details=False):
    """``N4.py:9-118``.  Masked-out voxels of the result are 0."""
    m = mask != 0
    x = im_before_sharpen[m]
    H, binMin, binMax, slope = histogram(x, numberOfHistogramBins)
    E = sharpening_map(H, binMin, slope, WienerFilterNoise,
                       BiasFieldFullWidthAtHalfMaximium)
    out = np.zeros(im_before_sharpen.shape)
    out[m] = remap(x, E, binMin, slope)
    if details:
        return out, dict(H=H, E=E, binMin=binMin, binMax=binMax, slope=slope)
    return out


# --------------------------------------------------------------------------
# convergence (N4.py:121-126)
# --------------------------------------------------------------------------
def CalculateConvergenceMeasurement(field1, field2, mask, ddof=0):
    field_diff = field1 - field2
    pixel = np.exp(field_diff)[mask != 0]
    return np.std(pixel, ddof=ddof) / np.mean(pixel)


# --------------------------------------------------------------------------
# lattice refinement (N4.py:132-165, cudaN4.cu:995-1084)
# --------------------------------------------------------------------------
_BW = (np.array([1 / 8, 6 / 8, 1 / 8]), np.array([0.0, 1 / 2, 1 / 2]))


def _refine_axis(a: np.ndarray, axis: int) -> np.ndarray:
    """One axis of the (n+3) -> (2n+3) refinement with the reference's
    clamped ("constant") boundary."""
    a = np.moveaxis(a, axis, 0)
    n = a.shape[0] - 3
    out = np.zeros((2 * n + 3,) + a.shape[1:])
    for i in range(-1, n + 2):
        pieces = [a[min(max(k, -1), n + 1) + 1] for k in (i - 1, i, i + 1)]
        for par in (0, 1):
            o = 2 * i + par
            if -1 <= o <= 2 * n + 1:
                bw = _BW[par]
                out[o + 1] = bw[0] * pieces[0] + bw[1] * pieces[1] + bw[2] * pieces[2]
    return np.moveaxis(out, 0, axis)


def UpsampleLattice3D(lattice: np.ndarray) -> np.ndarray:
    """(n+3)^3 -> (2n+3)^3 refinement.

    The reference applies the 27-point tensor weights in one sum; because the
    weights are a tensor product and the clamp is per axis, that equals three
    separable 3-tap passes (exactly so in exact arithmetic; to round-off in
    FP64).  For anisotropic lattices ``N4.py`` clips every axis with the first
    axis' extent (``N4.py:152-161``); the per-axis extents of
    ``cudaN4.cu:1039-1041`` are used here, which agree with ``N4.py`` for the
    cubic lattices ``N4.py`` supports.
    """
    out = np.asarray(lattice, dtype=np.float64)
    for ax in range(3):
        out = _refine_axis(out, ax)
    return out


# --------------------------------------------------------------------------
# cubic B-spline fit / evaluate (N4.py:174-273)
# --------------------------------------------------------------------------
def cubicBspline(t):
    t2 = t ** 2
    t3 = t ** 3
    B0 = (1 - t) ** 3 / 6
    B1 = (3 * t3 - 6 * t2 + 4) / 6
    B2 = (-3 * t3 + 3 * t2 + 3 * t + 1) / 6
    B3 = t3 / 6
    return np.array([B0, B1, B2, B3])


def axis_tables(size: int, ncpt: int):
    """Span index and the 4 cubic weights of every voxel along one axis,
    exactly as ``N4.py:210-222`` computes them per voxel."""
    nspans = ncpt - 3
    span = np.float64(size) / np.float64(nspans)
    i = np.arange(size, dtype=np.float64)
    s = np.floor((i + 0.5) / span).astype(np.int64)
    t = ((i + 0.5) - s * span) / span
    w = cubicBspline(t).T  # (size, 4)
    return s, w


def _dense(size, ncpt, power=1, normalise=False):
    s, w = axis_tables(size, ncpt)
    wp = w ** power
    if normalise:
        wp = wp / (w ** 2).sum(axis=1, keepdims=True)
    M = np.zeros((size, ncpt))
    rows = np.repeat(np.arange(size), 4)
    cols = (s[:, None] + np.arange(4)[None, :]).ravel()
    M[rows, cols] = wp.ravel()
    return M


def _contract(field, Mx, My, Mz):
    t = np.tensordot(field, Mz, axes=([2], [0]))   # (X, Y, cz)
    t = np.tensordot(t, My, axes=([1], [0]))       # (X, cz, cy)
    t = np.tensordot(t, Mx, axes=([0], [0]))       # (cz, cy, cx)
    return np.ascontiguousarray(t.transpose(2, 1, 0))


def FitBspline3D(field, mask, numberOfControlPoints, eps=1e-3, zero_den=False):
    """Single-level scattered-data B-spline fit, ``N4.py:186-237``.

    Separable evaluation of the same sums: for a voxel with tensor weights
    ``wc = wx wy wz`` the reference accumulates ``wc^2 * (r wc / sum wc^2)``
    and ``wc^2``; ``sum wc^2 = (sum wx^2)(sum wy^2)(sum wz^2)``, so both sums
    are three successive per-axis contractions.  ``FitBspline3D_literal``
    is the per-voxel form; the tests check that both agree.
    """
    ncpt = tuple(int(c) for c in numberOfControlPoints)
    X, Y, Z = field.shape
    m = (mask != 0)
    r = np.where(m, field, 0.0)
    num = _contract(r, _dense(X, ncpt[0], 3, True), _dense(Y, ncpt[1], 3, True),
                    _dense(Z, ncpt[2], 3, True))
    den = _contract(m.astype(np.float64), _dense(X, ncpt[0], 2), _dense(Y, ncpt[1], 2),
                    _dense(Z, ncpt[2], 2))
    if zero_den:
        out = np.zeros_like(num)
        nz = den != 0
        out[nz] = num[nz] / den[nz]
        return out
    return num / (den + eps)


def FitBspline3D_literal(field, mask, numberOfControlPoints, eps=1e-3, chunk=1 << 16):
    """Per-voxel scatter form of ``N4.py:186-237`` (vectorised in chunks,
    accumulated in voxel order)."""
    ncpt = np.array(numberOfControlPoints)
    size = np.array(field.shape)
    sx, wx = axis_tables(size[0], ncpt[0])
    sy, wy = axis_tables(size[1], ncpt[1])
    sz, wz = axis_tables(size[2], ncpt[2])
    ii, jj, kk = np.nonzero(mask != 0)
    num = np.zeros(int(np.prod(ncpt)))
    den = np.zeros(int(np.prod(ncpt)))
    off = np.arange(4)
    for c0 in range(0, ii.size, chunk):
        i, j, k = ii[c0:c0 + chunk], jj[c0:c0 + chunk], kk[c0:c0 + chunk]
        wc = wx[i][:, :, None, None] * wy[j][:, None, :, None] * wz[k][:, None, None, :]
        wc2 = wc ** 2
        wsum = wc2.reshape(len(i), 64).sum(axis=1)
        phi = field[i, j, k][:, None, None, None] * wc / wsum[:, None, None, None]
        lin = ((sx[i][:, None, None, None] + off[None, :, None, None]) * ncpt[1]
               + (sy[j][:, None, None, None] + off[None, None, :, None])) * ncpt[2] \
            + (sz[k][:, None, None, None] + off[None, None, None, :])
        num += np.bincount(lin.ravel(), weights=(wc2 * phi).ravel(), minlength=num.size)
        den += np.bincount(lin.ravel(), weights=wc2.ravel(), minlength=den.size)
    return (num / (den + eps)).reshape(tuple(ncpt))


def EvaluateBspline3D(lattice, numberOfControlPoints, size):
    """Dense evaluation of the lattice on a grid of ``size`` voxels,
    ``N4.py:241-273`` (separable form)."""
    ncpt = tuple(int(c) for c in numberOfControlPoints)
    X, Y, Z = (int(s) for s in size)
    Wx, Wy, Wz = _dense(X, ncpt[0]), _dense(Y, ncpt[1]), _dense(Z, ncpt[2])
    t = np.tensordot(lattice, Wz, axes=([2], [1]))   # (cx, cy, Z)
    t = np.tensordot(t, Wy, axes=([1], [1]))         # (cx, Z, Y)
    t = np.tensordot(t, Wx, axes=([0], [1]))         # (Z, Y, X)
    return np.ascontiguousarray(t.transpose(2, 1, 0))


def EvaluateBspline3D_literal(lattice, numberOfControlPoints, size, chunk=1 << 16):
    """Per-voxel form of ``N4.py:241-273`` (vectorised in chunks)."""
    ncpt = np.array(numberOfControlPoints)
    X, Y, Z = (int(s) for s in size)
    sx, wx = axis_tables(X, ncpt[0])
    sy, wy = axis_tables(Y, ncpt[1])
    sz, wz = axis_tables(Z, ncpt[2])
    out = np.zeros(X * Y * Z)
    lat = np.asarray(lattice, dtype=np.float64)
    for c0 in range(0, out.size, chunk):
        lin = np.arange(c0, min(c0 + chunk, out.size))
        i, j, k = lin // (Y * Z), (lin // Z) % Y, lin % Z
        acc = np.zeros(lin.size)
        for a in range(4):
            for b in range(4):
                for c in range(4):
                    acc += (wx[i, a] * wy[j, b] * wz[k, c]) * lat[sx[i] + a, sy[j] + b, sz[k] + c]
        out[c0:c0 + lin.size] = acc
    return out.reshape(X, Y, Z)


# --------------------------------------------------------------------------
# the driver (N4.py:276-332)
# --------------------------------------------------------------------------
def lattice_dims(ncpt0, levels):
    """Control points per axis at the last level, ``main.cpp:87-91``."""
    return tuple(((int(c) - 3) << (levels - 1)) + 3 for c in ncpt0)


def _iterate(im_log, mask, lattice, logBiasField, maxIter, thr, p, report, level):
    ncpt = lattice.shape
    cv = 10000000000.0
    it = 0
    cvs = []
    logU = im_log - logBiasField
    while cv > thr and it < maxIter:
        it += 1
        sharp = sharpenImage(logU, mask, p["bins"], p["wiener"], p["fwhm"])
        resid = logU - sharp
        lattice = lattice + FitBspline3D(resid, mask, ncpt, p["eps"], p["zero_den"])
        newLog = EvaluateBspline3D(lattice, ncpt, im_log.shape)
        cv = CalculateConvergenceMeasurement(logBiasField, newLog, mask, p["ddof"])
        cvs.append(cv)
        logBiasField = newLog
        logU = im_log - logBiasField
    if report is not None:
        report.setdefault("iterations", []).append(it)
        report.setdefault("cv", []).append(cvs)
    return lattice, logBiasField


def N4(im, mask, low_value=10, maximumNumberOfLevels=1,
       maximumNumberOfIterations=(50,), ConvergenceThreshold=0.001,
       numberOfHistogramBins=200, WienerFilterNoise=0.01,
       BiasFieldFullWidthAtHalfMaximum=0.15, numberOfControlPoints=(4, 4, 4),
       fit_eps=1e-3, fit_zero_den=False, cv_ddof=0, initial_lattice=None,
       report=None, return_log_bias=False):
    """``N4.py:276-332`` with the extensions listed in the module docstring.

    ``maximumNumberOfIterations`` may be a scalar (the CUDA reference's
    single count, ``cudaN4.h:75``) or one count per level (``N4.py``).
    With ``initial_lattice`` (first-level control points) the first
    iteration is run from it and from the zero lattice; the warm start is
    kept only if its first-iteration convergence value is not larger than
    the zero-lattice one (``report['warm_start_used']``).
    """
    if np.isscalar(maximumNumberOfIterations):
        maximumNumberOfIterations = [int(maximumNumberOfIterations)] * maximumNumberOfLevels
    p = dict(bins=numberOfHistogramBins, wiener=WienerFilterNoise,
             fwhm=BiasFieldFullWidthAtHalfMaximum, eps=fit_eps,
             zero_den=fit_zero_den, ddof=cv_ddof)
    im, mask = np.array(im, dtype=np.float64), np.array(mask, dtype=np.float64)
    low = im <= low_value
    mask[low] = 0
    im[low] = 0
    with np.errstate(divide="ignore"):
        im_log = np.log(im)
    logBiasField = np.zeros_like(im)
    lattice = np.zeros(tuple(int(c) for c in numberOfControlPoints))
    if report is not None:
        report["warm_start_used"] = False

    for level in range(maximumNumberOfLevels):
        maxIter = int(maximumNumberOfIterations[level])
        if level == 0 and initial_lattice is not None and maxIter > 0:
            warm = np.array(initial_lattice, dtype=np.float64).reshape(lattice.shape)
            rw, rp = {}, {}
            lw, bw = _iterate(im_log, mask, warm,
                              EvaluateBspline3D(warm, warm.shape, im.shape),
                              1, -1.0, p, rw, level)
            lp, bp = _iterate(im_log, mask, lattice, logBiasField, 1, -1.0, p, rp, level)
            use_warm = rw["cv"][0][0] <= rp["cv"][0][0]
            first_cv = (rw if use_warm else rp)["cv"][0][0]
            lattice, logBiasField = (lw, bw) if use_warm else (lp, bp)
            rest = {}
            if first_cv > ConvergenceThreshold and maxIter > 1:
                lattice, logBiasField = _iterate(im_log, mask, lattice, logBiasField,
                                                 maxIter - 1, ConvergenceThreshold, p,
                                                 rest, level)
            if report is not None:
                report["warm_start_used"] = bool(use_warm)
                report["first_cv_warm"] = rw["cv"][0][0]
                report["first_cv_plain"] = rp["cv"][0][0]
                report.setdefault("iterations", []).append(1 + (rest["iterations"][0] if rest else 0))
                report.setdefault("cv", []).append([first_cv] + (rest["cv"][0] if rest else []))
        else:
            lattice, logBiasField = _iterate(im_log, mask, lattice, logBiasField, maxIter,
                                             ConvergenceThreshold, p, report, level)
        if level != maximumNumberOfLevels - 1:
            lattice = UpsampleLattice3D(lattice)

    logBiasField = EvaluateBspline3D(lattice, lattice.shape, im.shape)
    im_normalized = im / np.exp(logBiasField)
    if return_log_bias:
        return im_normalized, lattice, logBiasField
    return im_normalized, lattice


# --------------------------------------------------------------------------
# shrink factor (not in the reference; defined by this project)
# --------------------------------------------------------------------------
def shrink_volume(im, mask, shrink, low_value):
    """Block reduction of a thresholded volume by ``shrink`` per axis.

    The volume is first thresholded at full resolution (intensity and mask
    set to 0 where ``im <= low_value``, ``N4.py:284-285``).  A shrunk voxel
    is in the mask when a strict majority of its block is; its intensity is
    the mean over the masked voxels of the block, or over the whole block
    when none of it is masked.  Every axis must be a multiple of ``shrink``.
    """
    s = int(shrink)
    if any(d % s for d in np.shape(im)):
        raise ValueError("volume dimensions must be multiples of the shrink factor")
    im = np.array(im, dtype=np.float64)
    m = (np.asarray(mask) != 0) & (im > low_value)
    im = np.where(im > low_value, im, 0.0)
    X, Y, Z = (d // s for d in im.shape)
    im_c = im[:X * s, :Y * s, :Z * s].reshape(X, s, Y, s, Z, s)
    m_c = m[:X * s, :Y * s, :Z * s].reshape(X, s, Y, s, Z, s)
    cnt = m_c.sum(axis=(1, 3, 5))
    tot = (im_c * m_c).sum(axis=(1, 3, 5))
    allmean = im_c.mean(axis=(1, 3, 5))
    with np.errstate(invalid="ignore", divide="ignore"):
        mean = np.where(cnt > 0, tot / np.maximum(cnt, 1), allmean)
    mask_s = (2 * cnt > s ** 3).astype(np.float64)
    return mean, mask_s


def N4Shrink(im, mask, shrink=1, low_value=10, **kw):
    """N4 fitted on a shrunk volume and applied at full resolution.

    With ``shrink == 1`` this is exactly ``N4``.  Otherwise the lattice is
    fitted on ``shrink_volume(...)`` and the final log bias field is the
    lattice evaluated on the full-resolution grid (span = full size /
    number of spans); the corrected volume is the thresholded full-resolution
    volume divided by its exponential.
    """
    return_log_bias = kw.pop("return_log_bias", False)
    if int(shrink) == 1:
        return N4(im, mask, low_value=low_value, return_log_bias=return_log_bias, **kw)
    im_s, mask_s = shrink_volume(im, mask, shrink, low_value)
    _, lattice = N4(im_s, mask_s, low_value=low_value, **kw)
    im_full = np.array(im, dtype=np.float64)
    im_full[im_full <= low_value] = 0
    logb = EvaluateBspline3D(lattice, lattice.shape, im_full.shape)
    out = im_full / np.exp(logb)
    if return_log_bias:
        return out, lattice, logb
    return out, lattice
