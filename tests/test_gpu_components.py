"""Component kernels (through the C ABI) against N4.py's golden vectors.

The sharpening map is computed in FP64 on the device (an FP32 map differs
from the FP64 oracle by ~2e-5 of its range in sparse bins, which N4's
residual accumulation amplifies ~200-fold); it is compared at 1e-6.

Tolerance: the kernels compute in FP32 against FP64 references, so results
are compared relative to the reference's largest magnitude
(``max|gpu - ref| / max|ref|``) with the bound stated per test.
"""
import numpy as np
import pytest

import n4_oracle as O

pytestmark = pytest.mark.gpu


def nrel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a.astype(np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("k", [0, 1, 2])
def test_fit(cuda, golden_components, k):
    import n4b200
    g = golden_components
    f, m, nc = g[f"fit_field_{k}"], g[f"fit_mask_{k}"], g[f"fit_ncpt_{k}"]
    lat = n4b200.FitBspline3D(cuda.tensor(f, dtype=cuda.float32, device="cuda"),
                              cuda.tensor(m, dtype=cuda.float32, device="cuda"), nc)
    assert nrel(lat, g[f"fit_out_{k}"]) < 1e-5


def test_fit_zero_den_semantics(cuda):
    """cudaN4.cu:123-127: control points without support get 0."""
    import n4b200
    rng = np.random.default_rng(1)
    f = rng.normal(size=(20, 16, 12))
    m = np.zeros_like(f)
    m[:10] = 1.0                      # the upper half of x has no voxels
    a = n4b200.FitBspline3D(f, m, (7, 5, 5), zero_den=True)
    ref = O.FitBspline3D(f, m, (7, 5, 5), zero_den=True)
    assert nrel(a, ref) < 1e-5
    assert np.all(np.asarray(a)[-1] == 0.0)


@pytest.mark.parametrize("shape,nc", [((64, 48, 160), (8, 7, 11)), ((40, 36, 320), (6, 9, 35)),
                                      ((20, 18, 400), (5, 5, 19)), ((33, 17, 36), (6, 5, 40)),
                                      ((16, 16, 8), (5, 4, 7)), ((10, 6, 800), (4, 5, 23)),
                                      ((8, 8, 1028), (4, 4, 12))])
def test_fit_row_kernels_agree_bitwise(cuda, shape, nc):
    """The z contraction has three kernels, chosen by Z and the alignment of
    the field and mask: rows read in 32-byte steps (Z % 8 == 0, 32-byte
    aligned), in 16-byte steps (Z % 4 == 0, 16-byte aligned), both for
    Z <= 1024, and the scalar kernel (otherwise).  All add the same terms in
    the same order, so the field at a 32-byte boundary, 16 bytes and 4 bytes
    further on give bitwise the same lattice; NaNs where the mask is 0 are
    ignored by all.  Covers more spans than voxels along z (empty spans), a
    target count that is not a multiple of 4 and a Z above the vectorised
    kernels' limit."""
    import n4b200
    rng = np.random.default_rng(7)
    n = int(np.prod(shape))
    f = rng.normal(0, 0.3, size=n).astype(np.float32)
    m = (rng.random(n) < 0.6).astype(np.float32)
    f[(m == 0) & (rng.random(n) < 0.05)] = np.nan
    lats = []
    for off in (0, 4, 1):                         # floats: 32-, 16- and 4-byte aligned starts
        fb = cuda.empty(n + 8, device="cuda")
        mb = cuda.empty(n + 8, device="cuda")
        assert fb.data_ptr() % 32 == 0 and mb.data_ptr() % 32 == 0
        fb[off:off + n] = cuda.tensor(f, device="cuda")
        mb[off:off + n] = cuda.tensor(m, device="cuda")
        lats.append(n4b200.FitBspline3D(fb[off:off + n].view(shape), mb[off:off + n].view(shape), nc))
    cuda.cuda.synchronize()
    assert cuda.isfinite(lats[0]).all()
    assert cuda.equal(lats[0], lats[1]) and cuda.equal(lats[0], lats[2])
    ref = O.FitBspline3D(np.where(m == 0, 0.0, f).reshape(shape).astype(np.float64), m.reshape(shape), nc)
    assert nrel(lats[0], ref) < 1e-5


@pytest.mark.parametrize("k", [0, 1, 2])
def test_evaluate(cuda, golden_components, k):
    import n4b200
    g = golden_components
    nc, shape = g[f"fit_ncpt_{k}"], g[f"fit_field_{k}"].shape
    out = n4b200.EvaluateBspline3D(cuda.tensor(g[f"eval_lat_{k}"], dtype=cuda.float32, device="cuda"), nc, shape)
    assert nrel(out, g[f"eval_out_{k}"]) < 1e-5


@pytest.mark.parametrize("shape", [(64, 64, 48), (37, 29, 23), (256, 256, 176)])
def test_evaluate_sizes(cuda, shape):
    """float4 (z % 4 == 0) and scalar paths, full-resolution size."""
    import n4b200
    rng = np.random.default_rng(2)
    lat = rng.normal(0, 0.3, size=(11, 11, 11))
    out = n4b200.EvaluateBspline3D(lat, lat.shape, shape)
    assert nrel(out, O.EvaluateBspline3D(lat, lat.shape, shape)) < 1e-5


@pytest.mark.parametrize("n", [4, 5, 7])
def test_upsample(cuda, golden_components, n):
    import n4b200
    g = golden_components
    out = n4b200.UpsampleLattice3D(g[f"up_in_{n}"])
    assert nrel(out, g[f"up_out_{n}"]) < 1e-6


def test_upsample_anisotropic(cuda):
    import n4b200
    lat = np.random.default_rng(5).normal(size=(4, 6, 5))
    assert nrel(n4b200.UpsampleLattice3D(lat), O.UpsampleLattice3D(lat)) < 1e-6


@pytest.mark.parametrize("tag,fwhm", [("a", 0.15), ("b", 0.3)])
@pytest.mark.parametrize("bins", [200, 64])
def test_sharpen(cuda, golden_components, tag, fwhm, bins):
    import n4b200
    g = golden_components
    x = g["sharp_in"].astype(np.float32)
    out, det = n4b200.sharpenImage(x, g["sharp_mask"], bins, 0.01, fwhm, details=True)
    # same FP32 input through the FP64 oracle, and the N4.py golden output
    ref = O.sharpenImage(x.astype(np.float64), g["sharp_mask"], bins, 0.01, fwhm)
    assert nrel(out, ref) < 1e-6
    assert nrel(out, g[f"sharp_out_{tag}{bins}"]) < 1e-5
    m = g["sharp_mask"] != 0
    assert det["binMin"] == x[m].min() and det["binMax"] == x[m].max()


def test_sharpen_map_matches_oracle(cuda, golden_components):
    import n4b200
    g = golden_components
    x = g["sharp_in"].astype(np.float32)
    m = g["sharp_mask"]
    _, det = n4b200.sharpenImage(x, m, 200, 0.01, 0.15, details=True)
    _, od = O.sharpenImage(x.astype(np.float64), m, 200, 0.01, 0.15, details=True)
    E = det["E"].astype(np.float64)
    live = od["H"] > 0          # bins that voxels actually map through
    assert np.abs(E - od["E"])[live].max() / np.abs(od["E"]).max() < 1e-6


def test_convergence(cuda, golden_components):
    import n4b200
    g = golden_components
    cv = n4b200.CalculateConvergenceMeasurement(g["cv_f1"], g["cv_f2"], g["cv_mask"])
    assert cv == pytest.approx(float(g["cv_out"]), rel=1e-4)
    cv1 = n4b200.CalculateConvergenceMeasurement(g["cv_f1"], g["cv_f2"], g["cv_mask"], ddof=1)
    ref1 = O.CalculateConvergenceMeasurement(g["cv_f1"], g["cv_f2"], g["cv_mask"], ddof=1)
    assert cv1 == pytest.approx(ref1, rel=1e-4)


def test_component_autotuner_records_and_reuses_tile_shapes(cuda):
    """n4_autotune_components times the fit's z-contraction shapes and the
    evaluation's tile shapes on one field and lattice size and records the
    fastest of each; later FitBspline3D / EvaluateBspline3D calls with that
    key run them (n4_last_timings reports the shape a call used), with
    bitwise the results of the default shapes, and another size keeps the
    defaults."""
    import n4b200
    rng = np.random.default_rng(41)
    shape, nc = (64, 72, 160), (8, 7, 11)
    f = cuda.tensor(rng.normal(0.0, 0.3, size=shape).astype(np.float32), device="cuda")
    m = cuda.tensor((rng.random(shape) < 0.6).astype(np.float32), device="cuda")
    ctx = n4b200.Context()
    lat0 = n4b200.FitBspline3D(f, m, nc, ctx=ctx)
    ev0 = n4b200.EvaluateBspline3D(lat0, nc, shape, ctx=ctx)
    t = n4b200.autotune_components(f, m, nc, ctx=ctx)
    assert len(t["fit"]) >= 8 and len(t["evaluate"]) >= 4
    assert all(ms > 0 for *_, ms in t["fit"]) and all(ms > 0 for *_, ms in t["evaluate"])
    assert t["fit_chosen"] == min(t["fit"], key=lambda c: c[3])[:3]
    assert t["evaluate_chosen"] == min(t["evaluate"], key=lambda c: c[2])[:2]
    ctx.set_profiling(True)
    lat1 = n4b200.FitBspline3D(f, m, nc, ctx=ctx)
    tf = ctx.last_timings()
    ev1 = n4b200.EvaluateBspline3D(lat1, nc, shape, ctx=ctx)
    te = ctx.last_timings()
    assert (tf["fit_step"], tf["fit_depth"], tf["fit_rows"]) == t["fit_chosen"]
    assert (te["correct_rows"], te["correct_threads"]) == t["evaluate_chosen"]
    assert cuda.equal(lat0, lat1) and cuda.equal(ev0, ev1)
    # a different field size: the default shapes
    f2, m2 = f[:, :, :80].contiguous(), m[:, :, :80].contiguous()
    n4b200.FitBspline3D(f2, m2, nc, ctx=ctx)
    assert (ctx.last_timings()["fit_step"], ctx.last_timings()["fit_rows"]) == (8, 64)
    n4b200.EvaluateBspline3D(lat1, nc, (64, 72, 80), ctx=ctx)
    assert (ctx.last_timings()["correct_rows"], ctx.last_timings()["correct_threads"]) == (128, 256)
    ctx.set_profiling(False)
    ctx.close()
