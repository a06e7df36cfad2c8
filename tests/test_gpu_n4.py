"""Whole-N4 parity through the C ABI against the FP64 oracle and N4.py.

Tolerance (from the target): corrected volume and log bias field within
1e-4 relative of the FP64 reference, measured as
``max|gpu - ref| / max|ref|``; the lattice to the same bound.  Iteration
counts must match exactly where the reference stops on the threshold.
"""
import numpy as np
import pytest

import n4_oracle as O
from n4b200.phantom import make_phantom

pytestmark = pytest.mark.gpu
TOL = 1e-4


def nrel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a.astype(np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def param(levels, iters, thr, **kw):
    import n4b200
    return n4b200.N4Param(NumberOfFittingLevels=levels, MaximumNumberOfIterations=list(iters),
                          ConvergenceThreshold=thr, low_value=0.0, **kw)


def log_bias(lat, shape):
    return O.EvaluateBspline3D(np.asarray(lat, dtype=np.float64), np.shape(lat), shape)


@pytest.mark.parametrize("tag", ["fixed", "thresh"])
@pytest.mark.parametrize("force", [0, 0x8])
def test_small_vs_reference_n4py(cuda, golden_small, tag, force):
    """Against N4.py itself (golden), cluster path and whole-GPU path."""
    import n4b200
    s = golden_small
    levels, iters, thr = int(s[f"{tag}_levels"]), list(s[f"{tag}_iters"]), float(s[f"{tag}_thr"])
    im = cuda.tensor(s[f"{tag}_im"], device="cuda")
    mk = cuda.tensor(s[f"{tag}_mask"], device="cuda")
    res = n4b200.N4(im, mk, param(levels, iters, thr, flags=force), return_bias=True)
    rep = {}
    O.N4(s[f"{tag}_im"], s[f"{tag}_mask"], low_value=0, maximumNumberOfLevels=levels,
         maximumNumberOfIterations=iters, ConvergenceThreshold=thr, report=rep)
    assert res.report["status"] == "N4_OK"
    assert res.report["iterations"] == rep["iterations"]
    assert res.report["path"] == ("grid" if force else "cluster")
    lat_ref = s[f"{tag}_lattice"]
    assert nrel(res.lattice, lat_ref) < TOL
    assert nrel(log_bias(res.lattice.cpu().numpy(), im.shape), log_bias(lat_ref, im.shape)) < TOL
    assert nrel(res.im_normalized, s[f"{tag}_norm"]) < TOL
    b = res.bias_field.cpu().numpy()
    assert nrel(np.log(b), log_bias(lat_ref, im.shape)) < TOL


def test_small_volume_few_iterations(cuda):
    """32x32x24 (a 24 k-voxel fitting grid), 2 levels x 4 iterations: a small
    lattice (max |L| ~0.04), where an error of the remap's bin coordinate shows
    most (an FP32 coordinate alone moves the oracle's lattice by 1.4e-4)."""
    import n4b200
    for seed in (3, 4, 5):
        ph = make_phantom((32, 32, 24), seed=seed, sigma=0.03, grid=4, coeff_std=0.15)
        res = n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"),
                        param(2, [4, 4], 0.0))
        out, lat = O.N4(ph.im, ph.mask, low_value=0, maximumNumberOfLevels=2, maximumNumberOfIterations=[4, 4],
                        ConvergenceThreshold=0.0)
        assert nrel(res.lattice, lat) < TOL
        assert nrel(res.im_normalized, out) < TOL


def test_c1_fixed_iterations(cuda, golden_c1):
    """64x64x48 phantom, 3 levels x 50 iterations, against N4.py's run."""
    import n4b200
    g = golden_c1
    ph = make_phantom((64, 64, 48), seed=int(g["seed"]), sigma=0.03, grid=4, coeff_std=0.15)
    res = n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"),
                    param(3, [50, 50, 50], 0.0))
    assert res.report["iterations"] == [50, 50, 50]
    assert nrel(res.lattice, g["lattice"]) < TOL
    assert nrel(res.im_normalized.cpu().numpy().reshape(-1)[::97], g["norm_sample"]) < TOL


@pytest.mark.parametrize("force", [0, 0x8])
def test_c1_against_oracle(cuda, force):
    ph = make_phantom((64, 64, 48), seed=1, sigma=0.03, grid=4, coeff_std=0.15)
    import n4b200
    res = n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"),
                    param(3, [12, 12, 12], 0.0, flags=force))
    out, lat, lb = O.N4(ph.im, ph.mask, low_value=0, maximumNumberOfLevels=3,
                        maximumNumberOfIterations=[12, 12, 12], ConvergenceThreshold=0.0,
                        return_log_bias=True)
    assert nrel(res.lattice, lat) < TOL
    assert nrel(log_bias(res.lattice.cpu().numpy(), ph.im.shape), lb) < TOL
    assert nrel(res.im_normalized, out) < TOL


def test_c2_shape_shrink4(cuda):
    """256x256x176 at shrink 4, 4 levels; fixed iterations for exact parity,
    then to convergence 0.001."""
    import n4b200
    ph = make_phantom((256, 256, 176), seed=2, sigma=0.02, grid=6, coeff_std=0.25)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    res = n4b200.N4(im, mk, param(4, [8] * 4, 0.0, ShrinkFactor=4), return_bias=True)
    assert res.report["path"] == "cluster" and res.report["cluster_size"] == 16
    out, lat, lb = O.N4Shrink(ph.im, ph.mask, 4, low_value=0, maximumNumberOfLevels=4,
                              maximumNumberOfIterations=[8] * 4, ConvergenceThreshold=0.0,
                              return_log_bias=True)
    assert nrel(res.lattice, lat) < TOL
    assert nrel(np.log(res.bias_field.cpu().numpy()), lb) < TOL
    assert nrel(res.im_normalized, out) < TOL
    conv = n4b200.N4(im, mk, param(4, [50] * 4, 0.001, ShrinkFactor=4))
    rep = {}
    _, lat2 = O.N4Shrink(ph.im, ph.mask, 4, low_value=0, maximumNumberOfLevels=4,
                         maximumNumberOfIterations=[50] * 4, ConvergenceThreshold=0.001, report=rep)
    got = conv.report["iterations"]
    assert all(abs(a - b) <= 1 for a, b in zip(got, rep["iterations"])), (got, rep["iterations"])
    if got == rep["iterations"]:
        assert nrel(conv.lattice, lat2) < TOL
    # the oracle's own stopping points, run as fixed counts: the converged
    # lattice is pinned even where a CV within rounding of the threshold
    # stops the two runs one iteration apart
    pinned = n4b200.N4(im, mk, param(4, rep["iterations"], 0.0, ShrinkFactor=4))
    assert pinned.report["iterations"][:4] == rep["iterations"]
    assert nrel(pinned.lattice, lat2) < TOL


def test_cluster_and_grid_paths_agree(cuda):
    import n4b200
    ph = make_phantom((64, 64, 48), seed=9, sigma=0.03, grid=4, coeff_std=0.2)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    a = n4b200.N4(im, mk, param(3, [10] * 3, 0.0))
    b = n4b200.N4(im, mk, param(3, [10] * 3, 0.0, flags=0x8))
    assert a.report["path"] == "cluster" and b.report["path"] == "grid"
    # different partitions sum in different orders; N4 amplifies the FP32
    # difference (~2e-5 here), so the paths are compared at the parity bound
    assert nrel(a.lattice, b.lattice.cpu().numpy().astype(np.float64)) < TOL
    c = n4b200.N4(im, mk, param(3, [10] * 3, 0.0, flags=0x8 | n4b200._lib.FLAG_CTA_512))
    assert c.report["path"] == "grid"
    assert nrel(c.lattice, b.lattice.cpu().numpy().astype(np.float64)) < TOL


def test_deterministic(cuda):
    import n4b200
    ph = make_phantom((48, 40, 36), seed=4)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    p = param(2, [6, 6], 0.0)
    a = n4b200.N4(im, mk, p)
    b = n4b200.N4(im, mk, p)
    assert cuda.equal(a.lattice, b.lattice) and cuda.equal(a.im_normalized, b.im_normalized)


def test_batched_matches_single(cuda):
    """A volume's result does not depend on the other volumes of its batch:
    with the same cluster size and threads per CTA, the batched run and the
    single run do the same arithmetic (the histogram's fixed-point scale is
    chosen per volume), so they agree bitwise."""
    import n4b200
    shapes = [(40, 48, 32), (64, 56, 40), (24, 32, 48), (56, 56, 56), (32, 24, 40)]
    vols = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=100 + i, sigma=0.03, grid=4, coeff_std=0.15)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    p = param(3, [20] * 3, 0.001)
    batch = n4b200.N4Batch(vols, p)
    for (im, mk), r in zip(vols, batch):
        s = n4b200.N4(im, mk, p)
        assert r.report["status"] == "N4_OK"
        assert r.report["cluster_size"] == s.report["cluster_size"]
        assert r.report["iterations"] == s.report["iterations"]
        assert cuda.equal(r.lattice, s.lattice) and cuda.equal(r.im_normalized, s.im_normalized)


def test_host_path_matches_device_path(cuda):
    import n4b200
    ph = make_phantom((32, 28, 24), seed=6)
    p = param(2, [5, 5], 0.0)
    h = n4b200.N4(ph.im, ph.mask, p, return_bias=True)
    d = n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"), p, return_bias=True)
    assert np.array_equal(h.lattice, d.lattice.cpu().numpy())
    assert np.array_equal(h.im_normalized, d.im_normalized.cpu().numpy())
    assert np.array_equal(h.bias_field, d.bias_field.cpu().numpy())


def test_warm_start(cuda):
    """A good warm lattice is kept and converges in fewer iterations; a bad
    one is discarded (first-iteration CV rule), as the oracle decides."""
    import n4b200
    ph = make_phantom((64, 64, 48), seed=11, sigma=0.03, grid=4, coeff_std=0.2)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    p1 = param(1, [50], 0.001)
    plain = n4b200.N4(im, mk, p1)
    good = n4b200.N4(im, mk, p1, warm_lattice=plain.lattice)
    assert good.report["warm_start_used"]
    assert good.report["iterations"][0] < plain.report["iterations"][0]
    # a constant lattice only rescales the intensities (invisible to N4); a
    # spatially varying wrong one is what the first-iteration rule rejects
    wrong = cuda.tensor(np.random.default_rng(0).normal(0.0, 1.0, (4, 4, 4)), dtype=cuda.float32, device="cuda")
    bad = n4b200.N4(im, mk, p1, warm_lattice=wrong)
    assert not bad.report["warm_start_used"]
    assert bad.report["iterations"] == plain.report["iterations"]
    assert nrel(bad.lattice, plain.lattice.cpu().numpy().astype(np.float64)) < 1e-6
    rep = {}
    _, lat = O.N4(ph.im, ph.mask, low_value=0, maximumNumberOfLevels=1, maximumNumberOfIterations=[4],
                  ConvergenceThreshold=0.0, initial_lattice=plain.lattice.cpu().numpy(), report=rep)
    g4 = n4b200.N4(im, mk, param(1, [4], 0.0), warm_lattice=plain.lattice)
    assert g4.report["warm_start_used"] == rep["warm_start_used"]
    assert nrel(g4.lattice, lat) < TOL


# ------------------------------------------------------------------ edge cases
def test_empty_mask(cuda):
    import n4b200
    ph = make_phantom((16, 16, 16), seed=1)
    with pytest.raises(n4b200.N4Error, match="EMPTY_MASK"):
        n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.zeros((16, 16, 16), device="cuda"), param(1, [3], 0.0))


def test_constant_image(cuda):
    """A constant masked image has no histogram range: nothing to fit."""
    import n4b200
    im = np.full((20, 20, 20), 0.7, dtype=np.float32)
    res = n4b200.N4(cuda.tensor(im, device="cuda"), None, param(2, [5, 5], 0.0))
    assert float(res.lattice.abs().max()) == 0.0
    assert nrel(res.im_normalized, im.astype(np.float64)) < 1e-7


@pytest.mark.parametrize("shape,nc", [((17, 13, 11), (4, 4, 4)), ((23, 19, 30), (5, 4, 6))])
def test_ragged_shapes_and_anisotropic_lattice(cuda, shape, nc):
    import n4b200
    ph = make_phantom(shape, seed=8)
    p = param(2, [4, 4], 0.0, NumberOfControlPoints_x=nc[0], NumberOfControlPoints_y=nc[1],
              NumberOfControlPoints_z=nc[2])
    for force in (0, 0x8):
        p.flags = force
        res = n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"), p)
        out, lat = O.N4(ph.im, ph.mask, low_value=0, maximumNumberOfLevels=2, maximumNumberOfIterations=[4, 4],
                        ConvergenceThreshold=0.0, numberOfControlPoints=nc)
        assert nrel(res.lattice, lat) < TOL
        assert nrel(res.im_normalized, out) < TOL


def test_low_value_threshold_and_inplace(cuda):
    """Voxels at or below low_value leave the mask and are zero in the
    output; N4_FLAG_INPLACE_THRESH writes that back like cudaN4.cu:1459."""
    import n4b200
    ph = make_phantom((32, 32, 24), seed=12)
    low = 0.5
    p = param(2, [4, 4], 0.0)
    p.low_value = low
    out, lat = O.N4(ph.im, ph.mask, low_value=low, maximumNumberOfLevels=2, maximumNumberOfIterations=[4, 4],
                    ConvergenceThreshold=0.0)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    res = n4b200.N4(im, mk, p)
    assert nrel(res.lattice, lat) < TOL and nrel(res.im_normalized, out) < TOL
    assert float(res.im_normalized[im <= low].abs().max()) == 0.0
    assert float((im <= low).sum()) > 0 and float(im[im <= low].abs().max()) > 0.0
    p.flags = 0x4
    n4b200.N4(im, mk, p)
    assert float(im[cuda.tensor(ph.im, device="cuda") <= low].abs().max()) == 0.0
    assert float(mk[cuda.tensor(ph.im, device="cuda") <= low].abs().max()) == 0.0


def test_invalid_arguments(cuda):
    import n4b200
    im = cuda.ones((16, 16, 18), device="cuda")
    with pytest.raises(n4b200.N4Error, match="INVALID_ARG"):
        n4b200.N4(im, None, param(1, [2], 0.0, ShrinkFactor=4))   # 18 % 4 != 0
    with pytest.raises(n4b200.N4Error, match="UNSUPPORTED_SPLINE_ORDER"):
        n4b200.N4(im, None, param(1, [2], 0.0, SplineOrder=2))


def test_nonfinite_input_is_reported(cuda):
    import n4b200
    ph = make_phantom((16, 16, 16), seed=3)
    im = ph.im.copy()
    im[8, 8, 8] = np.inf
    with pytest.raises(n4b200.N4Error, match="NONFINITE"):
        n4b200.N4(cuda.tensor(im, device="cuda"), cuda.tensor(ph.mask, device="cuda"), param(1, [2], 0.0))


@pytest.mark.parametrize("shrink", [2, 4])
@pytest.mark.parametrize("u8", [False, True])
def test_vector_prologue_matches_scalar(cuda, shrink, u8):
    """Shrink 2 and 4 read each block's rows with one vector load per row when
    the image and mask are aligned for it, else with scalar loads; the same
    volume at an aligned address and 4 bytes (1 byte for a byte mask) further
    on corrects bitwise alike, and a non-finite voxel inside the mask is
    reported by both."""
    import n4b200
    ph = make_phantom((64, 64, 48), seed=21)
    n = ph.im.size
    mask = (ph.mask.ravel() != 0).astype(np.uint8) if u8 else ph.mask.ravel().astype(np.float32)
    res = []
    for bad in (False, True):
        for off in (0, 1):
            ib = cuda.zeros(n + 8, device="cuda")
            ib[off:off + n] = cuda.tensor(ph.im.ravel(), device="cuda")
            mb = cuda.zeros(n + 8, dtype=cuda.uint8 if u8 else cuda.float32, device="cuda")
            mb[off:off + n] = cuda.tensor(mask, device="cuda")
            im, mk = ib[off:off + n].view(ph.im.shape), mb[off:off + n].view(ph.im.shape)
            p = param(2, [6, 6], 0.0, ShrinkFactor=shrink)
            if bad:
                idx = tuple(int(i) for i in np.argwhere(ph.mask != 0)[len(np.argwhere(ph.mask != 0)) // 2])
                im[idx] = float("inf")
                with pytest.raises(n4b200.N4Error, match="NONFINITE"):
                    n4b200.N4(im, mk, p)
            else:
                res.append(n4b200.N4(im, mk, p))
    assert res[0].report["status"] == "N4_OK"
    assert cuda.equal(res[0].lattice, res[1].lattice)
    assert cuda.equal(res[0].im_normalized, res[1].im_normalized)


def test_shrink2_batch_prologue_matches_scalar(cuda):
    """A shrink-2 batch with more fitting voxels than prologue threads
    (4 x 64x64x48 = 786k against 148 SMs x 16 CTAs x 256) makes threads take
    further voxels, some of them in another volume, on their grid-stride loop;
    the batch corrects bitwise alike when one volume sits 4 bytes off
    alignment, which sends the whole batch through the scalar prologue."""
    import n4b200
    shape = (128, 128, 96)
    phs = [make_phantom(shape, seed=300 + i) for i in range(4)]
    n = phs[0].im.size
    p = param(2, [4, 4], 0.0, ShrinkFactor=2)
    res = []
    for off in (0, 1):
        vols = []
        for i, ph in enumerate(phs):
            o = off if i == 2 else 0
            ib = cuda.zeros(n + 8, device="cuda")
            ib[o:o + n] = cuda.tensor(ph.im.ravel(), device="cuda")
            mb = cuda.zeros(n + 8, device="cuda")
            mb[o:o + n] = cuda.tensor(ph.mask.ravel().astype(np.float32), device="cuda")
            vols.append((ib[o:o + n].view(shape), mb[o:o + n].view(shape)))
        res.append(n4b200.N4Batch(vols, p))
    for a, b in zip(res[0], res[1]):
        assert a.report["status"] == "N4_OK"
        assert cuda.equal(a.lattice, b.lattice)
        assert cuda.equal(a.im_normalized, b.im_normalized)


def test_batch_graph_replays(cuda):
    """The graph-recorded batch equals N4Batch, and a launch after refilling
    an input in place corrects the new data."""
    import n4b200
    shapes = [(40, 48, 32), (64, 56, 40), (24, 32, 48)]
    vols = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=200 + i)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    p = param(3, [20] * 3, 0.001)
    g = n4b200.N4BatchGraph(vols, p)
    for _ in range(2):
        g.launch()
    res = g.sync()
    ref = n4b200.N4Batch(vols, p)
    for r, q in zip(res, ref):
        assert r.report["status"] == "N4_OK" and r.report["iterations"] == q.report["iterations"]
        assert cuda.equal(r.lattice, q.lattice) and cuda.equal(r.im_normalized, q.im_normalized)
    ph = make_phantom(shapes[0], seed=999)
    g.inputs[0][0].copy_(cuda.tensor(ph.im, device="cuda"))
    g.inputs[0][1].copy_(cuda.tensor(ph.mask, device="cuda"))
    g.launch()
    res = g.sync()
    single = n4b200.N4(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"), p)
    # a volume's arithmetic depends on its cluster size, not on its batch
    assert res[0].report["cluster_size"] == single.report["cluster_size"]
    assert cuda.equal(res[0].lattice, single.lattice)
    g.close()


def test_autotune_records_the_fastest_configuration(cuda):
    """n4_autotune times every cluster size that fits; later runs of volumes
    of the same sizes use the recorded one."""
    import n4b200
    shapes = [(96, 96, 64), (112, 96, 72), (96, 104, 64), (120, 96, 80)]
    vols = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=300 + i)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    p = param(3, [10] * 3, 0.001, ShrinkFactor=4)
    ctx = n4b200.Context()
    ref = n4b200.N4Batch(vols, p, ctx=ctx)
    assert all(q.report["cluster_size"] == 16 for q in ref)       # untuned: the largest cluster
    t = n4b200.autotune(vols, p, ctx=ctx)
    sizes = [k for k, _, _ in t["candidates"]]
    assert len(sizes) >= 4 and 16 in sizes
    assert {nt for _, nt, _ in t["candidates"]} == {512, 768, 1024}
    assert all(ms > 0 for _, _, ms in t["candidates"])
    best = min(t["candidates"], key=lambda c: c[2])
    assert (t["chosen"], t["chosen_threads"]) == (best[0], best[1])
    res = n4b200.N4Batch(vols, p, ctx=ctx)
    for r in res:
        assert r.report["status"] == "N4_OK"
        assert r.report["cluster_size"] == t["chosen"]
    # correction tile shapes: every shape timed on the chosen path, the
    # fastest recorded and used by later runs of the same key, all bitwise alike
    corr = t["correction"]
    assert len(corr) >= 4 and all(ms > 0 for _, _, ms in corr)
    assert t["correction_chosen"] == min(corr, key=lambda c: c[2])[:2]
    subs = t["sub_batches_ms"]
    uniform = [(s, tp) for s, tp, ad, _ in subs if ad == 0]
    assert uniform == [(1, False), (2, False), (3, False), (4, False), (3, True), (4, True)]
    assert all(ms > 0 for *_, ms in subs)
    assert t["sub_batches_chosen"] == min(subs, key=lambda c: c[3])[:3]
    ctx.set_profiling(True)
    again = n4b200.N4Batch(vols, p, ctx=ctx)
    tm = ctx.last_timings()
    ctx.set_profiling(False)
    assert (tm["correct_rows"], tm["correct_threads"]) == t["correction_chosen"]
    for a, b in zip(res, again):
        assert cuda.equal(a.im_normalized, b.im_normalized)
    # another batch shape is not affected by the record
    other = n4b200.N4Batch(vols[:2], p, ctx=ctx)
    assert all(r.report["cluster_size"] == 16 for r in other)
    ctx.close()


def test_every_cluster_size_matches_the_oracle(cuda):
    """Cluster sizes 16 .. 2 (every size whose per-CTA share fits), with 1024
    and 512 threads per CTA, on a 128x128x96 phantom at shrink 4 against the
    FP64 oracle, fixed iterations."""
    import n4b200
    ph = make_phantom((128, 128, 96), seed=4, sigma=0.02, grid=6, coeff_std=0.25)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    out, lat, _ = O.N4Shrink(ph.im, ph.mask, 4, low_value=0, maximumNumberOfLevels=4,
                             maximumNumberOfIterations=[8] * 4, ConvergenceThreshold=0.0, return_log_bias=True)
    ran = []
    for K in (16, 12, 8, 6, 4, 2):
        for threads_flag in (0, n4b200._lib.FLAG_CTA_512):
            pk = param(4, [8] * 4, 0.0, ShrinkFactor=4, flags=n4b200.cluster_size_flag(K) | threads_flag)
            try:
                res = n4b200.N4(im, mk, pk)
            except n4b200.N4Error as e:
                assert "N4_ERR_TOO_LARGE" in str(e)
                continue
            assert res.report["cluster_size"] == K
            assert nrel(res.lattice, lat) < TOL, (K, threads_flag)
            assert nrel(res.im_normalized, out) < TOL, (K, threads_flag)
            ran.append((K, threads_flag))
    assert len(ran) >= 8, ran


def test_batch_mixing_cluster_and_whole_gpu_volumes(cuda):
    """A batch whose largest volume does not fit a cluster: the others run
    on the cluster path, it on the whole-GPU path, each as in a single run;
    the autotuner's record keeps that split."""
    import n4b200
    # fitting grids 32x32x24, 112x112x64 (more than a 16-CTA cluster holds), 48x40x32
    shapes = [(64, 64, 48), (224, 224, 128), (96, 80, 64)]
    vols = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=400 + i)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    p = param(3, [10] * 3, 0.001, ShrinkFactor=2)
    ctx = n4b200.Context()
    res = n4b200.N4Batch(vols, p, ctx=ctx)
    assert [r.report["path"] for r in res] == ["cluster", "grid", "cluster"]
    for (im, mk), r in zip(vols, res):
        single = n4b200.N4(im, mk, p, ctx=ctx)
        assert r.report["status"] == "N4_OK" and r.report["iterations"] == single.report["iterations"]
        assert nrel(r.lattice, single.lattice.cpu().numpy().astype(np.float64)) < 1e-6
        assert nrel(r.im_normalized, single.im_normalized.cpu().numpy().astype(np.float64)) < 1e-6
    t = n4b200.autotune(vols, p, ctx=ctx)
    tuned = n4b200.N4Batch(vols, p, ctx=ctx)
    assert tuned[1].report["path"] == "grid"
    assert all(r.report["cluster_size"] == t["chosen"] for r in (tuned[0], tuned[2]))
    ctx.close()


def test_byte_masks_match_float_masks(cuda):
    """N4_FLAG_MASK_U8: a uint8 mask gives bitwise the float mask's result on
    every entry point that takes a run's masks (single, host, batched, graph,
    warm inputs), and the in-place threshold clears its bytes."""
    import n4b200
    ph = make_phantom((64, 64, 48), seed=21)
    im = cuda.tensor(ph.im, device="cuda")
    mf = cuda.tensor(ph.mask, device="cuda")
    mb = (mf != 0).to(cuda.uint8)
    p = param(2, [6, 6], 0.001, ShrinkFactor=2)
    a, b = n4b200.N4(im, mf, p), n4b200.N4(im, mb, p)
    assert cuda.equal(a.lattice, b.lattice) and cuda.equal(a.im_normalized, b.im_normalized)
    h = n4b200.N4(ph.im, (ph.mask != 0).astype(np.uint8), p)
    assert np.array_equal(h.lattice, a.lattice.cpu().numpy())
    ra = n4b200.N4Batch([(im, mf), (im * 1.5, mf)], p)
    rb = n4b200.N4Batch([(im, mb), (im * 1.5, mb)], p)
    for x, y in zip(ra, rb):
        assert cuda.equal(x.lattice, y.lattice) and cuda.equal(x.im_normalized, y.im_normalized)
    g = n4b200.N4BatchGraph([(im, mb)], p)
    g.launch()
    assert cuda.equal(g.sync()[0].lattice, a.lattice)
    g.close()
    assert cuda.equal(n4b200.warm_inputs([(im, mf)], p), n4b200.warm_inputs([(im, mb)], p))
    with pytest.raises(ValueError):
        n4b200.N4Batch([(im, mf), (im, mb)], p)
    # in-place threshold on a byte mask (shrink 1)
    low = 0.5
    p1 = param(1, [2], 0.0, flags=0x4)
    p1.low_value = low
    im2, mb2 = im.clone(), mb.clone()
    n4b200.N4(im2, mb2, p1)
    below = im <= low
    assert int(mb2[below].max()) == 0 and float(im2[below].abs().max()) == 0.0
    assert cuda.equal(mb2[~below], mb[~below])
