"""n4_run_batched_host: host-resident volumes corrected through the pipelined
upload / batched run / download path.

Each sub-batch of ``per`` volumes is one batched run, so every volume must
come back bitwise equal to N4Batch over the same sub-batch on device copies
(same plan, same kernels), with float and byte masks, the bias output and
the learned warm start; sub-batches of different sizes and more sub-batches
than staging slots are covered.
"""
import numpy as np
import pytest

from n4b200.phantom import make_phantom

pytestmark = pytest.mark.gpu


def _vols(cuda, shapes, seed0, u8=False):
    out = []
    for i, sh in enumerate(shapes):
        ph = make_phantom(sh, seed=seed0 + i, sigma=0.03, grid=4, coeff_std=0.15)
        m = (ph.mask != 0).astype(np.uint8) if u8 else ph.mask
        out.append((cuda.from_numpy(ph.im).pin_memory(), cuda.from_numpy(m).pin_memory()))
    return out


@pytest.mark.parametrize("u8", [False, True])
def test_host_batch_matches_device_batches(cuda, u8):
    import n4b200
    shapes = [(64, 64, 48), (48, 56, 40), (64, 48, 64), (40, 40, 32), (56, 64, 48), (48, 48, 48), (64, 56, 40)]
    vols = _vols(cuda, shapes, 700, u8)
    p = n4b200.N4Param(NumberOfFittingLevels=3, MaximumNumberOfIterations=20, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=4)
    per = 1   # 7 sub-batches over the 4 lanes: every lane's staging slot is reused
    res, ms = n4b200.N4BatchHost(vols, p, per=per, return_bias=True, ctx=n4b200.Context())
    assert ms > 0
    ctx = n4b200.Context()
    for lo in range(0, len(vols), per):
        dev = [(a.cuda(), b.cuda()) for a, b in vols[lo:lo + per]]
        ref = n4b200.N4Batch(dev, p, return_bias=True, ctx=ctx)
        for r, q in zip(res[lo:lo + per], ref):
            assert r.report["status"] == "N4_OK"
            assert r.report["iterations"] == q.report["iterations"]
            assert cuda.equal(r.lattice, q.lattice.cpu())
            assert cuda.equal(r.im_normalized, q.im_normalized.cpu())
            assert cuda.equal(r.bias_field, q.bias_field.cpu())


def test_host_batch_with_warm_start(cuda):
    import n4b200
    from n4b200.warmstart import load_encoder
    vols = _vols(cuda, [(96, 96, 64)] * 5, 800)
    p = n4b200.N4Param(NumberOfFittingLevels=4, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=4)
    enc = load_encoder(max_batch=8)
    res, _ = n4b200.N4BatchHost(vols, p, per=3, encoder=enc, ctx=n4b200.Context())
    ctx = n4b200.Context()
    for lo in (0, 3):
        dev = [(a.cuda(), b.cuda()) for a, b in vols[lo:lo + 3]]
        ref = n4b200.N4Batch(dev, p, encoder=enc, ctx=ctx)
        for r, q in zip(res[lo:lo + 3], ref):
            assert r.report["warm_start_used"] == q.report["warm_start_used"]
            assert cuda.equal(r.lattice, q.lattice.cpu())
            assert cuda.equal(r.im_normalized, q.im_normalized.cpu())
