"""Error bound of the engine's exp(x) - 1 for the convergence terms
(`expm1_conv`, csrc/n4_device.cuh): for |x| < 1/4 the Taylor series of
exp(x) - 1 through x^7 / 7!, evaluated in FP32 as
x + x^2 (1/2 + x (1/6 + x (1/24 + x (1/120 + x (1/720 + x / 5040))))) with
fused multiply-adds (emulated here: a product of two floats is exact in FP64),
against numpy's FP64 expm1.  Beyond 1/4 the engine calls expm1f."""
import numpy as np


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def expm1_conv_model(x):
    x = np.asarray(x, dtype=np.float32)
    c = [np.float32(1.0 / 5040.0), np.float32(1.0 / 720.0), np.float32(1.0 / 120.0),
         np.float32(1.0 / 24.0), np.float32(1.0 / 6.0), np.float32(0.5)]
    p = _fma32(x, np.full_like(x, c[0]), np.full_like(x, c[1]))
    for k in c[2:]:
        p = _fma32(p, x, np.full_like(x, k))
    return _fma32((x * x).astype(np.float32), p, x)


def test_relative_error_within_one_ulp_below_a_quarter():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-0.25, 0.25, 1 << 20),
                        rng.uniform(-1e-3, 1e-3, 1 << 18),
                        np.ldexp(rng.uniform(0.5, 1.0, 1 << 16), rng.integers(-40, -10, 1 << 16))]).astype(np.float32)
    x = x[np.abs(x) < 0.25]
    x = np.concatenate([x, -x])
    y = expm1_conv_model(x).astype(np.float64)
    ref = np.expm1(x.astype(np.float64))
    rel = np.abs(y - ref) / np.abs(ref)
    # one FP32 ulp of the result is at most 2^-23 relative
    assert rel.max() < 2.0 ** -23, rel.max()
    assert np.median(rel) < 2.0 ** -25


def test_zero_and_signs():
    x = np.array([0.0, -0.0, 1e-30, -1e-30, 0.2499, -0.2499], dtype=np.float32)
    y = expm1_conv_model(x)
    assert y[0] == 0.0 and y[1] == 0.0
    assert np.all(np.sign(y[2:]) == np.sign(x[2:]))
