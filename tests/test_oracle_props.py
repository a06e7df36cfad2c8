"""Size-independent properties of the oracle (known-answer tests)."""
import numpy as np
import pytest

import n4_oracle as O


def test_partition_of_unity():
    t = np.linspace(0, 1, 101)
    assert np.allclose(O.cubicBspline(t).sum(axis=0), 1.0, atol=1e-15)


@pytest.mark.parametrize("size,ncpt", [(44, 11), (48, 4), (17, 6), (176, 11)])
def test_axis_tables(size, ncpt):
    s, w = O.axis_tables(size, ncpt)
    assert s.min() >= 0 and s.max() <= ncpt - 4
    assert np.all(np.diff(s) >= 0)
    assert np.allclose(w.sum(axis=1), 1.0)


def test_constant_lattice_evaluates_to_constant():
    lat = np.full((7, 5, 6), 0.37)
    f = O.EvaluateBspline3D(lat, lat.shape, (20, 13, 9))
    assert np.allclose(f, 0.37, atol=1e-14)


@pytest.mark.parametrize("shape,nc", [((24, 20, 16), (4, 4, 4)), ((33, 18, 44), (5, 7, 11))])
def test_refinement_preserves_the_function(shape, nc):
    rng = np.random.default_rng(3)
    lat = rng.normal(size=nc)
    up = O.UpsampleLattice3D(lat)
    assert up.shape == tuple(2 * c - 3 for c in nc)
    a = O.EvaluateBspline3D(lat, lat.shape, shape)
    b = O.EvaluateBspline3D(up, up.shape, shape)
    assert np.abs(a - b).max() < 1e-12


def test_fit_is_linear_and_mirror_symmetric():
    """The single-level fit is linear in the field (the numerator is a
    weighted sum, the denominator depends on the mask only) and commutes
    with mirroring an axis (the span grid is symmetric)."""
    rng = np.random.default_rng(4)
    f1, f2 = rng.normal(size=(2, 21, 14, 18))
    m = (rng.uniform(size=(21, 14, 18)) > 0.3).astype(float)
    nc = (6, 5, 7)
    a = O.FitBspline3D(2.0 * f1 - 0.5 * f2, m, nc)
    b = 2.0 * O.FitBspline3D(f1, m, nc) - 0.5 * O.FitBspline3D(f2, m, nc)
    assert np.abs(a - b).max() < 1e-12
    c = O.FitBspline3D(f1[::-1], m[::-1], nc)
    assert np.abs(c[::-1] - O.FitBspline3D(f1, m, nc)).max() < 1e-12


def test_histogram_mass_and_top_bin_rule():
    rng = np.random.default_rng(0)
    x = rng.normal(size=5000)
    H, lo, hi, slope = O.histogram(x, 200)
    # every value adds weight 1 except one at the exact top whose offset is
    # non-zero after rounding (dropped by the reference rule)
    assert abs(H.sum() - x.size) <= 1.0 + 1e-9
    # a value exactly on a bin centre adds 1 to that bin
    H2, *_ = O.histogram(np.array([0.0, 1.0, 2.0, 4.0]), 5)
    assert np.allclose(H2, [1, 1, 1, 0, 1])


def test_sharpening_map_identity_and_contraction():
    centres = -1.0 + np.arange(200) * 0.01
    # a flat histogram maps the middle of its support to itself
    H = np.zeros(200)
    H[50:150] = 100.0
    E = O.sharpening_map(H, -1.0, 0.01, 0.01, 0.15)
    assert np.abs(E - centres)[90:110].max() < 1e-3
    # a narrow peak pulls the bins around it towards its centre
    H = np.zeros(200)
    H[95:106] = 100.0
    E = O.sharpening_map(H, -1.0, 0.01, 0.01, 0.15)
    near = np.r_[80:95, 106:120]
    assert np.all(np.abs(E[near] - centres[100]) < np.abs(centres[near] - centres[100]))


def test_shrink_volume():
    im = np.arange(64, dtype=np.float64).reshape(4, 4, 4) + 1.0
    mask = np.ones_like(im)
    mask[0, 0, 0] = 0
    s, m = O.shrink_volume(im, mask, 2, 0.0)
    assert s.shape == (2, 2, 2) and m.sum() == 8
    blk = im[:2, :2, :2]
    assert s[0, 0, 0] == pytest.approx((blk.sum() - im[0, 0, 0]) / 7)
    with pytest.raises(ValueError):
        O.shrink_volume(np.ones((5, 4, 4)), np.ones((5, 4, 4)), 2, 0.0)


def test_n4shrink_one_equals_n4():
    from n4b200.phantom import make_phantom
    ph = make_phantom((16, 12, 12), seed=5)
    a = O.N4Shrink(ph.im, ph.mask, 1, low_value=0, maximumNumberOfLevels=2,
                   maximumNumberOfIterations=[2, 2], ConvergenceThreshold=0.0)
    b = O.N4(ph.im, ph.mask, low_value=0, maximumNumberOfLevels=2,
             maximumNumberOfIterations=[2, 2], ConvergenceThreshold=0.0)
    assert np.array_equal(a[1], b[1])


def test_warm_start_rule():
    """A perfect warm start is kept; a bad one is discarded."""
    from n4b200.phantom import make_phantom
    ph = make_phantom((20, 16, 16), seed=7, coeff_std=0.2)
    kw = dict(low_value=0, maximumNumberOfLevels=1, maximumNumberOfIterations=[6],
              ConvergenceThreshold=0.0)
    rep0 = {}
    _, lat = O.N4(ph.im, ph.mask, report=rep0, **kw)
    rep1 = {}
    O.N4(ph.im, ph.mask, initial_lattice=lat, report=rep1, **kw)
    assert rep1["warm_start_used"] and rep1["first_cv_warm"] < rep1["first_cv_plain"]
    rep2 = {}
    O.N4(ph.im, ph.mask, initial_lattice=np.full((4, 4, 4), 3.0), report=rep2, **kw)
    assert not rep2["warm_start_used"]
