"""Training data and end-to-end use of the learned warm start.

* ``phantoms_gpu`` — seeded phantoms generated on the GPU (same model as
  ``phantom.make_phantom``: nested jittered ellipsoids, exp of a cubic
  B-spline bias, Rician noise; torch's generator instead of numpy's, so the
  volumes differ from the numpy ones with the same seed).
* ``make_dataset`` — network inputs and labels: the label of a phantom is the
  first-level 4x4x4 lattice of the plain GPU N4 run to convergence with one
  fitting level at the run's shrink factor.
* ``train_encoder`` — Adam on MSE with the tensor-core encoder.
* ``WarmBatch`` — pool + predict + batched N4 with the predictions as warm
  lattices (the batch itself recorded as a CUDA graph).
"""
from __future__ import annotations

import numpy as np

from . import N4Batch, N4BatchGraph, N4Param
from .encoder import Encoder, pool_input, train
from .phantom import _axis_weights


def phantoms_gpu(n, shape, seed, sigma=0.03, grid=6, coeff_std=0.3, device="cuda"):
    """n phantoms [n, X, Y, Z] (im, mask) on the GPU."""
    import torch
    X, Y, Z = shape
    g = torch.Generator(device=device).manual_seed(int(seed))
    jitter = torch.rand((n, 3, 3), device=device, generator=g) * 0.2 + 0.9
    coeffs = torch.randn((n, grid, grid, grid), device=device, generator=g) * coeff_std
    u = [(torch.arange(d, device=device, dtype=torch.float32) + 0.5) / d - 0.5 for d in (X, Y, Z)]
    Wx, Wy, Wz = (torch.tensor(_axis_weights(d, grid), dtype=torch.float32, device=device) for d in (X, Y, Z))
    ims, masks = [], []
    for i in range(n):
        clean = torch.zeros((X, Y, Z), device=device)
        mask = None
        for k, (radius, value) in enumerate(((0.45, 0.35), (0.35, 0.70), (0.20, 1.00))):
            r = radius * jitter[i, k]
            d = (u[0] / r[0])[:, None, None] ** 2 + (u[1] / r[1])[None, :, None] ** 2 + (u[2] / r[2])[None, None, :] ** 2
            inside = d <= 1.0
            clean = torch.where(inside, torch.full_like(clean, value), clean)
            if k == 0:
                mask = inside
        b = torch.einsum("abc,xa,yb,zc->xyz", coeffs[i], Wx, Wy, Wz)
        biased = clean * torch.exp(b)
        n1 = torch.randn((X, Y, Z), device=device, generator=g)
        n2 = torch.randn((X, Y, Z), device=device, generator=g)
        ims.append(torch.sqrt((biased + sigma * n1) ** 2 + (sigma * n2) ** 2))
        masks.append(mask.float())
    return torch.stack(ims), torch.stack(masks)


def label_param(shrink):
    return N4Param(NumberOfFittingLevels=1, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                   low_value=0.0, ShrinkFactor=shrink)


def make_dataset(n, shape, seed, shrink=4, chunk=256, **gen):
    """(x [n,32,32,24] bf16, y [n,4,4,4] float) on the GPU."""
    import torch
    xs, ys = [], []
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        im, mask = phantoms_gpu(m, shape, seed + c0, **gen)
        res = N4Batch([(im[i], mask[i]) for i in range(m)], label_param(shrink))
        ys.append(torch.stack([r.lattice for r in res]))
        x = torch.empty((m, 32, 32, 24), dtype=torch.bfloat16, device=im.device)
        for i in range(m):
            pool_input(im[i], mask[i], 0.0, out=x[i])
        xs.append(x)
        del im, mask, res
    return torch.cat(xs), torch.cat(ys)


def train_encoder(n_train=4096, n_val=256, shape=(128, 128, 96), epochs=20, batch=64, lr=1e-3, seed=0,
                  shrink=4, **gen):
    """Generate data with the plain GPU N4 and train; returns (encoder, report dict)."""
    import time
    t0 = time.time()
    x, y = make_dataset(n_train, shape, seed, shrink, **gen)
    xv, yv = make_dataset(n_val, shape, seed + 1_000_000, shrink, **gen)
    t_data = time.time() - t0
    enc = Encoder(max_batch=batch, seed=seed)
    rep = train(enc, x, y.reshape(-1, 64), epochs=epochs, batch=batch, lr=lr, seed=seed,
                x_val=xv, y_val=yv.reshape(-1, 64))
    base = float((yv.reshape(-1, 64) - y.reshape(-1, 64).mean(0)).pow(2).mean())
    return enc, dict(n_train=n_train, n_val=n_val, epochs=epochs, data_seconds=t_data, train_seconds=rep.seconds,
                     loss_first_epoch=rep.losses[0], loss_last_epoch=rep.losses[-1], val_mse=rep.val_loss,
                     val_mse_of_mean_predictor=base)


class WarmBatch:
    """Warm-started batched N4 over fixed device buffers: every ``run()``
    pools the inputs, predicts first-level lattices with the encoder and
    launches the recorded batch graph with them as warm lattices."""

    def __init__(self, enc: Encoder, volumes, param, ctx=None, low_value=0.0):
        import torch
        self.enc = enc
        self.volumes = volumes
        self.low = low_value
        dev = volumes[0][0].device
        n = len(volumes)
        self.x = torch.empty((n, 32, 32, 24), dtype=torch.bfloat16, device=dev)
        self.warm = torch.zeros((n, 4, 4, 4), dtype=torch.float32, device=dev)
        self.graph = N4BatchGraph(volumes, param, warm_lattices=[self.warm[i] for i in range(n)], ctx=ctx)

    def run(self):
        for i, (im, mask) in enumerate(self.graph.inputs):
            pool_input(im, mask, self.low, out=self.x[i])
        self.warm.copy_(self.enc.predict(self.x))
        self.graph.launch()

    def sync(self):
        return self.graph.sync()
