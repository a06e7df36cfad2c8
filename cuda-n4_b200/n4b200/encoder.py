"""Learned warm start for N4: training data, training loop and inference.

The encoder (``n4_encoder_*`` in ``include/n4b200.h``) maps the masked log
fitting grid, average-pooled to 32x32x24 (``n4b200.warm_inputs``), to the
first-level 4x4x4 log-bias lattice.  Training pairs come from the plain GPU N4 itself: for every seeded
phantom the label is the lattice of a one-level N4 run to convergence at the
run's shrink factor.  ``N4Batch(..., encoder=enc)`` and
``N4BatchGraph(..., encoder=enc)`` pool, predict and warm-start inside the
run; N4 still iterates to the same threshold and discards a warm start whose
first-iteration convergence value exceeds the zero-lattice one.

All network arithmetic runs in ``libn4b200.so`` (BF16 tensor-core kernels);
this module only orchestrates.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

IN_SHAPE = (32, 32, 24)
N_OUT = 64


def _decl():
    return _lib.load()


def layer_shapes():
    """(name, shape) of every parameter tensor, in the flat vector's order."""
    ch = [1, 16, 32, 64, 64]
    out = []
    for l in range(4):
        out.append((f"conv{l}.w", (ch[l + 1], ch[l], 3, 3, 3)))
        out.append((f"conv{l}.b", (ch[l + 1],)))
    out.append(("head.w", (N_OUT, 64 * 8)))
    out.append(("head.b", (N_OUT,)))
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases (seeded)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in layer_shapes():
        if name.endswith(".b"):
            parts.append(np.zeros(shape, np.float32))
        else:
            fan_in = int(np.prod(shape[1:]))
            bound = math.sqrt(6.0 / fan_in)
            if name.startswith("head"):
                bound = math.sqrt(3.0 / fan_in)
            parts.append(rng.uniform(-bound, bound, size=shape).astype(np.float32))
    flat = np.concatenate([p.ravel() for p in parts])
    assert flat.size == _decl().n4_encoder_num_params()
    return flat


class Encoder:
    def __init__(self, device: int = 0, max_batch: int = 64, seed: int = 0, params: np.ndarray | None = None):
        self.lib = _decl()
        self.h = C.c_void_p()
        self.device = device
        self.max_batch = max_batch
        check(self.lib.n4_encoder_create(C.byref(self.h), device, max_batch))
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if self.h:
            self.lib.n4_encoder_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nparam(self) -> int:
        return int(self.lib.n4_encoder_num_params())

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(self.lib.n4_encoder_set_params(self.h, p.ctypes.data, p.size))

    def params(self) -> np.ndarray:
        out = np.empty(self.nparam, np.float32)
        check(self.lib.n4_encoder_get_params(self.h, out.ctypes.data, None, out.size))
        return out

    def grads(self) -> np.ndarray:
        out = np.empty(self.nparam, np.float32)
        check(self.lib.n4_encoder_get_params(self.h, None, out.ctypes.data, out.size))
        return out

    def predict(self, x):
        """x: CUDA bf16 tensor [B, 32, 32, 24] -> CUDA float tensor [B, 4, 4, 4]."""
        import torch
        B = x.shape[0]
        out = torch.empty((B, 4, 4, 4), dtype=torch.float32, device=x.device)
        for b0 in range(0, B, self.max_batch):
            b1 = min(B, b0 + self.max_batch)
            check(self.lib.n4_encoder_predict(self.h, x[b0:b1].data_ptr(), b1 - b0, out[b0:b1].data_ptr(),
                                              torch.cuda.current_stream(x.device).cuda_stream))
        return out

    def train_step(self, x, target, lr: float, want_loss: bool = True) -> float:
        import torch
        loss = C.c_float()
        check(self.lib.n4_encoder_train_step(self.h, x.data_ptr(), target.data_ptr(), x.shape[0], float(lr),
                                             C.byref(loss) if want_loss else None,
                                             torch.cuda.current_stream(x.device).cuda_stream))
        return loss.value if want_loss else float("nan")


@dataclass
class TrainReport:
    losses: list
    val_loss: float
    seconds: float


def train(enc: Encoder, x, y, epochs: int = 20, batch: int = 64, lr: float = 1e-3, seed: int = 0,
          x_val=None, y_val=None) -> TrainReport:
    """Adam on MSE over (x [N,32,32,24] bf16, y [N,64] float), shuffled per epoch."""
    import time
    import torch
    g = torch.Generator().manual_seed(seed)
    n = x.shape[0]
    losses = []
    t0 = time.time()
    for _ in range(epochs):
        perm = torch.randperm(n, generator=g).to(x.device)
        tot, cnt = 0.0, 0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            l = enc.train_step(x[idx].contiguous(), y[idx].reshape(batch, N_OUT).contiguous(), lr)
            tot += l
            cnt += 1
        losses.append(tot / max(cnt, 1))
    torch.cuda.synchronize(x.device)
    secs = time.time() - t0
    val = float("nan")
    if x_val is not None:
        pred = enc.predict(x_val).reshape(-1, N_OUT)
        val = float(((pred - y_val.reshape(-1, N_OUT)) ** 2).mean())
    return TrainReport(losses, val, secs)
