"""Training data, training and evaluation of the learned warm start.

* ``phantoms_gpu`` — seeded phantoms generated on the GPU (same model as
  ``phantom.make_phantom``: nested jittered ellipsoids, exp of a cubic
  B-spline bias, Rician noise; torch's generator instead of numpy's, so the
  volumes differ from the numpy ones with the same seed).
* ``make_dataset`` — network inputs and labels: the input of a phantom is its
  masked log fitting grid pooled to 32x32x24 (``n4b200.warm_inputs``, the
  same pooling a warm-started run does internally); its label comes from the
  plain GPU N4 with one fitting level at the run's shrink factor, either the
  lattice it converges to (``label="end"``) or the lattice it holds one
  iteration before it stops (``label="pre"``, the default).  A warm start
  always runs at least one iteration, so from a perfect "pre" prediction the
  warm run repeats the plain run's last first-level iteration and continues
  exactly as the plain run does; from an "end" prediction it runs one
  iteration more than the plain run.
* ``train_encoder`` — Adam on MSE with the tensor-core encoder, optionally
  with the constant mode of the lattice weighted up (``gauge_weight``).
* ``evaluate`` — held-out phantoms corrected batched with and without the
  learned warm start (``N4Batch(..., encoder=...)``): iterations,
  volumes/s, warm starts kept, and the log-bias difference between the runs.

Why the constant mode matters.  The N4 residual ``logU - E(logU)`` is
unchanged when a constant is added to ``logU`` (the histogram, its bin range
and the sharpened map all shift with it), and so is every later update and
convergence value.  The constant of the log-bias lattice is therefore never
corrected: whatever constant the warm start hands over stays in the result,
plus the drift ``mean(residual)`` that every iteration adds.  Its error is
the whole raw log-bias difference between a warm and a plain run beyond the
(small) difference of their non-constant parts.

Command line (GPU)::

    python -m n4b200.warmstart train --out weights.npy      # 4096 x 128x128x96, 20 epochs
    python -m n4b200.warmstart eval --weights weights.npy   # 256 x 256x256x176
"""
from __future__ import annotations

import numpy as np

import os

from . import EvaluateBspline3D, N4Batch, N4Param, warm_inputs
from .encoder import Encoder, train
from .phantom import _axis_weights

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warmstart_encoder.npy")
TRAIN_GEN = dict(sigma=0.03, grid=6, coeff_std=0.3)


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


def eval_param(shrink=4, levels=4):
    """The 256x256x176 workload's parameters: 4 levels, <= 50 iterations,
    convergence 0.001, 200 bins, FWHM 0.15, Wiener 0.01."""
    return N4Param(NumberOfFittingLevels=levels, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                   low_value=0.0, ShrinkFactor=shrink)


def level1_labels(vols, shrink=4, label="pre"):
    """First-level 4x4x4 lattices [n,4,4,4] of the plain GPU N4 on ``vols``.

    ``label="end"``: the lattice one fitting level converges to (CV < 0.001,
    at most 50 iterations).  ``label="pre"``: the lattice one iteration
    before that (zero when the plain run stops after its first iteration);
    the volumes are rerun in groups of equal iteration count with that count
    minus one and no convergence test, which repeats the same iterations
    (the engine is deterministic)."""
    import torch
    res = N4Batch(vols, label_param(shrink))
    lat = torch.stack([r.lattice for r in res])
    if label == "end":
        return lat
    if label != "pre":
        raise ValueError(f"unknown label kind {label!r}")
    its = [int(r.report["iterations"][0]) for r in res]
    for n_it in sorted(set(its)):
        idx = [i for i, k in enumerate(its) if k == n_it]
        if n_it <= 1:
            lat[idx] = 0.0
            continue
        p = N4Param(NumberOfFittingLevels=1, MaximumNumberOfIterations=n_it - 1, ConvergenceThreshold=0.0,
                    low_value=0.0, ShrinkFactor=shrink)
        r2 = N4Batch([vols[i] for i in idx], p)
        lat[idx] = torch.stack([r.lattice for r in r2])
    return lat


def make_dataset(n, shape, seed, shrink=4, chunk=256, label="pre", **gen):
    """(x [n,32,32,24] bf16, y [n,4,4,4] float) on the GPU."""
    import torch
    xs, ys = [], []
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        im, mask = phantoms_gpu(m, shape, seed + c0, **gen)
        vols = [(im[i], mask[i]) for i in range(m)]
        ys.append(level1_labels(vols, shrink, label))
        xs.append(warm_inputs(vols, label_param(shrink)))
        del im, mask, vols
    return torch.cat(xs), torch.cat(ys)


def gauge_transform(weight: float) -> np.ndarray:
    """Symmetric 64x64 map T that multiplies the constant mode of a 4x4x4
    lattice (the unit vector u = ones / 8) by ``weight`` and leaves the
    orthogonal modes alone: T = I + (weight - 1) u u^T.  Training on T y
    weights the constant's squared error by weight^2 in the MSE; the trained
    head is then composed with T^-1 (``fold_output``) so that the network
    predicts lattices again."""
    u = np.full((64, 1), 1.0 / 8.0)
    return np.eye(64) + (float(weight) - 1.0) * (u @ u.T)


def fold_output(params: np.ndarray, T_inv: np.ndarray) -> np.ndarray:
    """Compose the linear head (the last 64x512 weights and 64 biases of the
    flat parameter vector) with ``T_inv`` on its output."""
    p = np.array(params, dtype=np.float64)
    nw, nb = 64 * 512, 64
    W = p[-(nw + nb):-nb].reshape(64, 512)
    b = p[-nb:]
    p[-(nw + nb):-nb] = (T_inv @ W).ravel()
    p[-nb:] = T_inv @ b
    return p.astype(np.float32)


def train_encoder(n_train=4096, n_val=256, shape=(256, 256, 176), epochs=20, batch=64, lr=1e-3, seed=0,
                  shrink=4, label="pre", gauge_weight=1.0, data=None, **gen):
    """Generate data with the plain GPU N4 and train; returns (encoder, report dict).

    ``data`` = (x, y, x_val, y_val) reuses a dataset from ``make_dataset``.
    With ``gauge_weight`` w != 1 the targets are T y (``gauge_transform``) and
    the trained head is folded with T^-1, so the constant mode's squared error
    counts w^2 times in the loss."""
    import time
    import torch
    gen = {**TRAIN_GEN, **gen}
    t0 = time.time()
    if data is None:
        x, y = make_dataset(n_train, shape, seed, shrink, label=label, **gen)
        xv, yv = make_dataset(n_val, shape, seed + 1_000_000, shrink, label=label, **gen)
    else:
        x, y, xv, yv = data
    torch.cuda.synchronize()
    t_data = time.time() - t0
    y = y.reshape(-1, 64)
    yv = yv.reshape(-1, 64)
    T = torch.tensor(gauge_transform(gauge_weight), dtype=torch.float32, device=y.device)
    enc = Encoder(max_batch=batch, seed=seed)
    rep = train(enc, x, (y @ T).contiguous(), epochs=epochs, batch=batch, lr=lr, seed=seed)
    if gauge_weight != 1.0:
        enc.set_params(fold_output(enc.params(), gauge_transform(1.0 / gauge_weight)))
    pred = enc.predict(xv).reshape(-1, 64)
    err = pred - yv
    base = float((yv - y.mean(0)).pow(2).mean())
    const_err = err.mean(1)
    return enc, dict(n_train=int(x.shape[0]), n_val=int(xv.shape[0]), shape=list(shape), label=label,
                     gauge_weight=gauge_weight, epochs=epochs, data_seconds=t_data, train_seconds=rep.seconds,
                     loss_first_epoch=rep.losses[0], loss_last_epoch=rep.losses[-1],
                     val_mse=float(err.pow(2).mean()), val_mse_of_mean_predictor=base,
                     val_rms_constant_error=float(const_err.pow(2).mean().sqrt()),
                     val_max_constant_error=float(const_err.abs().max()))


def evaluate(enc: Encoder, n_eval=256, shape=(256, 256, 176), seed=5_000_000, chunk=32, param=None, **gen):
    """Held-out phantoms corrected batched from zero and from the predicted
    lattices.  Returns mean iterations of both runs, device-timed volumes/s
    of both batched runs (pooling and prediction run inside the warm one),
    the share of warm starts kept, and the log-bias difference d between the
    two runs at full resolution: max |d| over the mask, max |d - mean_mask(d)|
    over the mask (a constant log bias is a global intensity scale, which the
    convergence measure std/mean of exp(change) does not see, so two runs
    stopping at CV < threshold may differ by one), and max |d| over the whole
    field of view (outside the mask the lattice is extrapolated)."""
    import torch
    gen = {**TRAIN_GEN, **gen}
    param = param or eval_param()
    dims = param.lattice_dims()
    it_plain, it_warm, lvl1_plain, lvl1_warm, kept, dmask, dcent, dfov = [], [], [], [], [], [], [], []
    ms_plain = ms_warm = 0.0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for c0 in range(0, n_eval, chunk):
        m = min(chunk, n_eval - c0)
        im, mask = phantoms_gpu(m, shape, seed + c0, **gen)
        vols = [(im[i], mask[i]) for i in range(m)]
        N4Batch(vols, param)                       # warm the context's workspaces
        torch.cuda.synchronize()
        N4Batch(vols, param, encoder=enc)
        torch.cuda.synchronize()
        ev[0].record()
        plain = N4Batch(vols, param, synchronous=False)
        ev[1].record()
        ev[2].record()
        warm = N4Batch(vols, param, encoder=enc, synchronous=False)
        ev[3].record()
        torch.cuda.synchronize()
        ms_plain += ev[0].elapsed_time(ev[1])
        ms_warm += ev[2].elapsed_time(ev[3])
        # reports (synchronous reruns are bitwise identical: the engine is deterministic)
        plain = N4Batch(vols, param)
        warm = N4Batch(vols, param, encoder=enc)
        for i, (a, b) in enumerate(zip(plain, warm)):
            it_plain.append(sum(a.report["iterations"][:a.report["levels"]]))
            it_warm.append(sum(b.report["iterations"][:b.report["levels"]]))
            lvl1_plain.append(a.report["iterations"][0])
            lvl1_warm.append(b.report["iterations"][0])
            kept.append(b.report["warm_start_used"])
            d = EvaluateBspline3D(b.lattice - a.lattice, dims, tuple(shape))
            inside = d[mask[i] != 0]
            dmask.append(float(inside.abs().max()))
            dcent.append(float((inside - inside.double().mean().float()).abs().max()))
            dfov.append(float(d.abs().max()))
        del im, mask, vols, plain, warm
    n = len(it_plain)
    q = lambda a, f: float(np.quantile(np.asarray(a), f))
    return dict(n_eval=n, shape=list(shape),
                iterations_plain=float(np.mean(it_plain)), iterations_warm=float(np.mean(it_warm)),
                level1_iterations_plain=float(np.mean(lvl1_plain)),
                level1_iterations_warm=float(np.mean(lvl1_warm)),
                warm_kept=float(np.mean(kept)),
                volumes_per_s_plain_batched=n / (ms_plain / 1000.0),
                volumes_per_s_warm_batched=n / (ms_warm / 1000.0),
                max_abs_log_bias_diff_mask=float(np.max(dmask)),
                median_abs_log_bias_diff_mask=q(dmask, 0.5),
                p90_abs_log_bias_diff_mask=q(dmask, 0.9),
                p99_abs_log_bias_diff_mask=q(dmask, 0.99),
                share_within_0_01=float(np.mean(np.asarray(dmask) <= 0.01)),
                max_abs_log_bias_diff_mask_mean_removed=float(np.max(dcent)),
                median_abs_log_bias_diff_mask_mean_removed=float(np.median(dcent)),
                max_abs_log_bias_diff_fov=float(np.max(dfov)))


def load_encoder(path=WEIGHTS, max_batch=64) -> Encoder:
    return Encoder(max_batch=max_batch, params=np.load(path))


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m n4b200.warmstart")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--n-train", type=int, default=4096)
    t.add_argument("--n-val", type=int, default=256)
    t.add_argument("--epochs", type=int, default=20)
    t.add_argument("--seed", type=int, default=0)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--n-eval", type=int, default=256)
    e.add_argument("--untrained", action="store_true", help="random-init encoder (the method without training)")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        enc, rep = train_encoder(n_train=a.n_train, n_val=a.n_val, epochs=a.epochs, seed=a.seed)
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        np.save(a.out, enc.params())
        rep["weights"] = a.out
        print(json.dumps(rep))
    else:
        enc = Encoder(max_batch=64, seed=0) if a.untrained else load_encoder(a.weights)
        print(json.dumps(evaluate(enc, n_eval=a.n_eval)))


if __name__ == "__main__":
    main()
