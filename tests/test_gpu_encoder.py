"""The warm-start encoder's BF16 tensor-core kernels against the FP64 CPU
reference (``oracle/encoder_ref.py``), which rounds to BF16 exactly where the
kernels store BF16.  Tolerance: max|gpu - ref| / max|ref| < 2e-2 per tensor
(a BF16 value carries 8 significant bits; accumulation is FP32 on the GPU and
FP64 on the CPU, so isolated elements can round to neighbouring BF16 values).
"""
import numpy as np
import pytest

import encoder_ref as R

pytestmark = pytest.mark.gpu


def nrel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def _inputs(B, seed):
    rng = np.random.default_rng(seed)
    x = R.bf16(rng.normal(-0.3, 0.4, size=(B, 32, 32, 24)))
    t = rng.normal(0.0, 0.1, size=(B, 64))
    return x, t


def test_forward_and_gradients(cuda):
    from n4b200.encoder import Encoder, init_params
    B = 6
    p = init_params(seed=3)
    x, t = _inputs(B, 4)
    enc = Encoder(max_batch=8, params=p)
    xd = cuda.tensor(x, dtype=cuda.bfloat16, device="cuda")
    td = cuda.tensor(t, dtype=cuda.float32, device="cuda")
    out = enc.predict(xd).reshape(B, 64).cpu().numpy()
    ref_out, _ = R.forward(p, x)
    assert nrel(out, ref_out) < 2e-2
    loss = enc.train_step(xd, td, lr=0.0)
    assert loss == pytest.approx(float(np.mean((ref_out - t) ** 2)), rel=2e-2)
    g = enc.grads()
    gref, _ = R.backward(p, x, t)
    o = 0
    from n4b200.encoder import layer_shapes
    for name, shape in layer_shapes():
        n = int(np.prod(shape))
        assert nrel(g[o:o + n], gref[o:o + n]) < 2e-2, name
        o += n


def test_adam_step_matches_reference(cuda):
    """One Adam step (lr 1e-3, b1 0.9, b2 0.999, eps 1e-8) from the GPU grads."""
    from n4b200.encoder import Encoder, init_params
    p = init_params(seed=5)
    x, t = _inputs(4, 6)
    enc = Encoder(max_batch=4, params=p)
    xd = cuda.tensor(x, dtype=cuda.bfloat16, device="cuda")
    td = cuda.tensor(t, dtype=cuda.float32, device="cuda")
    enc.train_step(xd, td, lr=1e-3)
    g = enc.grads().astype(np.float64)
    m = 0.1 * g
    v = 0.001 * g * g
    expect = p - 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.abs(enc.params() - expect).max() < 1e-6


def test_training_reduces_loss(cuda):
    """A learnable target (a fixed random linear map of pooled inputs)."""
    from n4b200.encoder import Encoder
    rng = np.random.default_rng(9)
    N = 256
    x = R.bf16(rng.normal(0.0, 0.5, size=(N, 32, 32, 24)))
    proj = rng.normal(0.0, 1.0, size=(4 * 4 * 3, 64)) / 8
    pooled = x.reshape(N, 4, 8, 4, 8, 3, 8).mean(axis=(2, 4, 6)).reshape(N, -1)
    t = pooled @ proj
    enc = Encoder(max_batch=64, seed=1)
    xd = cuda.tensor(x, dtype=cuda.bfloat16, device="cuda")
    td = cuda.tensor(t, dtype=cuda.float32, device="cuda")
    first = enc.train_step(xd[:64], td[:64], lr=0.0)
    from n4b200.encoder import train
    rep = train(enc, xd, td, epochs=30, batch=64, lr=1e-3)
    assert rep.losses[-1] < 0.2 * first


def test_warm_inputs_pool_the_fitting_grid(cuda):
    """n4_warm_inputs: threshold/shrink/log prologue, then 32x32x24 adaptive
    pooling of the masked log fitting grid (BF16)."""
    import n4b200
    import n4_oracle as O
    from n4b200.phantom import make_phantom
    for shape, shrink in (((128, 128, 96), 4), ((96, 112, 80), 2), ((64, 64, 48), 4)):
        ph = make_phantom(shape, seed=7)
        p = n4b200.N4Param(ShrinkFactor=shrink, low_value=0.0)
        got = n4b200.warm_inputs([(cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda"))], p)
        mean, mask_s = O.shrink_volume(ph.im, ph.mask, shrink, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            imlog = np.where((mask_s != 0) & (mean > 0.0), np.log(mean), np.nan)
        ref = R.pool_fitgrid(imlog)
        assert nrel(got[0].float().cpu().numpy(), ref) < 5e-3, shape
