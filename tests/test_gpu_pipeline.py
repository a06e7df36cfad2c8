"""Sub-batch pipelining of cluster-path batches and per-volume reports.

A batch on the cluster path may run as k sub-batches (N4_FLAG_SUB_BATCHES):
each sub-batch's prologue, warm start and correction overlap the other
sub-batches' iterations.  Every volume goes through the same kernels with the
same shared-memory plan either way, so the results must be bitwise those of
the single pass, eagerly, recorded as a graph and with the learned warm start.
"""
import numpy as np
import pytest

from n4b200.phantom import make_phantom

pytestmark = pytest.mark.gpu

SHAPES = [(40, 48, 32), (64, 56, 40), (48, 48, 48), (32, 40, 56), (56, 64, 32)]


def _param(sub, **kw):
    import n4b200
    p = n4b200.N4Param(NumberOfFittingLevels=2, MaximumNumberOfIterations=[8, 8], ConvergenceThreshold=0.0,
                       low_value=0.0, **kw)
    p.flags |= n4b200._lib.FLAG_SUB_BATCHES(sub)
    return p


def _volumes(cuda, n, seed):
    vols = []
    for i in range(n):
        ph = make_phantom(SHAPES[i % len(SHAPES)], seed=seed + i)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    return vols


def _same(cuda, a, b):
    for r, q in zip(a, b):
        assert r.report["status"] == q.report["status"] == "N4_OK"
        assert r.report["iterations"] == q.report["iterations"]
        assert cuda.equal(r.lattice, q.lattice)
        assert cuda.equal(r.im_normalized, q.im_normalized)


@pytest.mark.parametrize("sub", [2, 3, 4])
def test_sub_batches_match_one_pass(cuda, sub):
    """Ten volumes of five shapes: 2, 3 and 4 sub-batches (uneven ranges for
    3 and 4) against one pass, every volume bitwise."""
    import n4b200
    vols = _volumes(cuda, 10, 700)
    one = n4b200.N4Batch(vols, _param(1), return_bias=True)
    many = n4b200.N4Batch(vols, _param(sub), return_bias=True)
    _same(cuda, one, many)
    for r, q in zip(one, many):
        assert cuda.equal(r.bias_field, q.bias_field)


def test_sub_batches_in_a_graph_with_warm_start(cuda):
    """The graph-recorded warm-started batch (the bench path), 3 sub-batches
    against one pass, over two replays."""
    import n4b200
    from n4b200.warmstart import load_encoder
    vols = _volumes(cuda, 9, 800)
    enc = load_encoder(max_batch=16)
    ref = n4b200.N4Batch(vols, _param(1), encoder=enc)
    g = n4b200.N4BatchGraph(vols, _param(3), encoder=enc)
    for _ in range(2):
        g.launch()
        _same(cuda, ref, g.sync())
    g.close()


def test_nonfinite_voxel_is_reported_on_its_own_volume(cuda):
    """A non-finite voxel inside the mask of the third volume of a batch
    fails that volume only (its sub-batch's prologue flags it by index)."""
    import n4b200
    from n4b200 import _lib
    for sub in (1, 3):
        vols = _volumes(cuda, 6, 900)
        im, mk = vols[2]
        idx = tuple(int(i) for i in np.argwhere(mk.cpu().numpy() != 0)[0])
        im[idx] = float("inf")
        ctx = n4b200.Context()
        n4b200.N4Batch(vols, _param(sub), ctx=ctx, synchronous=False)
        reps = (_lib.n4_report_t * len(vols))()
        st = _lib.load().n4_sync(ctx.handle, reps, len(vols))
        assert _lib.STATUS[st] == "N4_ERR_NONFINITE"
        got = [_lib.STATUS[r.status] for r in reps]
        assert got == ["N4_OK", "N4_OK", "N4_ERR_NONFINITE", "N4_OK", "N4_OK", "N4_OK"], (sub, got)


def test_reports_follow_the_callers_order(cuda):
    """A run holds its volumes largest first (sub-batches end with the small
    ones); outputs and reports still belong to the caller's volumes: given
    smallest first, every volume's foreground count and iterations equal
    those of its own single run, and its lattice is bitwise that run's
    (same cluster size)."""
    import n4b200
    shapes = [(24, 24, 24), (32, 32, 24), (40, 32, 32), (48, 40, 40), (56, 48, 48), (64, 56, 56)]
    vols = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=950 + i)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    p = _param(3)
    p.flags |= n4b200.cluster_size_flag(8)
    batch = n4b200.N4Batch(vols, p)
    p1 = _param(1)
    p1.flags |= n4b200.cluster_size_flag(8)
    for (im, mk), r in zip(vols, batch):
        s = n4b200.N4(im, mk, p1)
        assert r.report["foreground"] == s.report["foreground"] == int((mk != 0).sum())
        assert r.report["iterations"] == s.report["iterations"]
        assert cuda.equal(r.lattice, s.lattice)


def test_sub_batches_on_their_own_cluster_sizes(cuda):
    """N4_FLAG_SUB_CLUSTER_FLOOR: the largest volumes' sub-batch runs on a
    large cluster, the small volumes' on the smallest size that holds them;
    every volume's result is bitwise its single run on the same size."""
    import n4b200
    from n4b200 import _lib
    shapes = [(192, 192, 128), (64, 64, 48), (176, 192, 128), (56, 64, 48)]
    vols = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=700 + i, sigma=0.03, grid=4, coeff_std=0.15)
        vols.append((cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")))
    flags = _lib.FLAG_CTA_512 | _lib.FLAG_SUB_BATCHES(2) | _lib.FLAG_SUB_CLUSTER_FLOOR(2)
    p = n4b200.N4Param(NumberOfFittingLevels=3, MaximumNumberOfIterations=[6] * 3, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=2, flags=flags)
    res = n4b200.N4Batch(vols, p)
    sizes = [r.report["cluster_size"] for r in res]
    print("cluster sizes", sizes)
    assert all(r.report["status"] == "N4_OK" and r.report["path"] == "cluster" for r in res)
    # planned largest first: the two large volumes form the first sub-batch,
    # on a larger cluster than the two small ones
    assert sizes[0] == sizes[2] and sizes[1] == sizes[3] and sizes[0] > sizes[1]
    for (im, mk), r in zip(vols, res):
        q = n4b200.N4Param(NumberOfFittingLevels=3, MaximumNumberOfIterations=[6] * 3, ConvergenceThreshold=0.001,
                           low_value=0.0, ShrinkFactor=2,
                           flags=_lib.FLAG_CTA_512 | n4b200.cluster_size_flag(r.report["cluster_size"]))
        s = n4b200.N4(im, mk, q)
        assert s.report["cluster_size"] == r.report["cluster_size"]
        assert r.report["iterations"] == s.report["iterations"]
        assert cuda.equal(r.lattice, s.lattice) and cuda.equal(r.im_normalized, s.im_normalized)
    # the same in a recorded graph
    g = n4b200.N4BatchGraph(vols, p)
    g.launch()
    for r, gr in zip(res, g.sync()):
        assert gr.report["cluster_size"] == r.report["cluster_size"]
        assert cuda.equal(r.lattice, gr.lattice)
    g.close()
