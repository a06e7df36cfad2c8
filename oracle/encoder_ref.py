"""CPU reference of the warm-start encoder (test infrastructure only).

Forward and backward of the network behind ``n4_encoder_*`` in FP64 numpy,
with BF16 rounding applied exactly where the GPU kernels store BF16 values
(weights, activations, activation gradients), so that the GPU gradients can be
checked element by element.  Used only by ``tests/``.

Network: 4 conv layers (3x3x3, stride 2, padding 1; 1->16->32->64->64
channels), each followed by ReLU, then a linear layer 512 -> 64; loss MSE.
"""
from __future__ import annotations

import numpy as np

CH = [1, 16, 32, 64, 64]


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unflatten(p):
    out, o = {}, 0
    for l in range(4):
        n = CH[l + 1] * CH[l] * 27
        out[f"w{l}"] = p[o:o + n].reshape(CH[l + 1], CH[l], 3, 3, 3); o += n
        out[f"b{l}"] = p[o:o + CH[l + 1]]; o += CH[l + 1]
    out["wh"] = p[o:o + 64 * 512].reshape(64, 512); o += 64 * 512
    out["bh"] = p[o:o + 64]; o += 64
    assert o == p.size
    return out


def _cols(x):
    """im2col for k3 s2 p1: x [B,C,D,H,W] -> [B, od, oh, ow, C*27]."""
    B, C, D, H, W = x.shape
    od, oh, ow = (D - 1) // 2 + 1, (H - 1) // 2 + 1, (W - 1) // 2 + 1
    xp = np.zeros((B, C, D + 2, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1, 1:-1] = x
    cols = np.empty((B, od, oh, ow, C, 27))
    t = 0
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                cols[..., t] = xp[:, :, kd:kd + 2 * od:2, kh:kh + 2 * oh:2, kw:kw + 2 * ow:2].transpose(0, 2, 3, 4, 1)
                t += 1
    return cols.reshape(B, od, oh, ow, C * 27), (od, oh, ow)


def forward(p, x):
    """x [B,32,32,24] (BF16 values).  Returns (out [B,64], cache)."""
    P = unflatten(np.asarray(p, np.float64))
    a = bf16(x)[:, None]
    acts, colss = [a], []
    for l in range(4):
        cols, (od, oh, ow) = _cols(a)
        w = bf16(P[f"w{l}"]).reshape(CH[l + 1], -1)
        y = cols @ w.T + P[f"b{l}"]
        a = bf16(np.maximum(y, 0.0)).transpose(0, 4, 1, 2, 3)      # [B, Co, od, oh, ow]
        acts.append(a)
        colss.append(cols)
    feat = a.reshape(a.shape[0], -1)
    out = feat @ bf16(P["wh"]).T + P["bh"]
    return out, dict(P=P, acts=acts, cols=colss, feat=feat)


def backward(p, x, target):
    """Gradients of mean((out - target)^2) in the flat parameter order."""
    out, c = forward(p, x)
    P, acts = c["P"], c["acts"]
    B = out.shape[0]
    n = out.size
    dout = bf16(2.0 * (out - target.reshape(B, -1)) / n)
    g = {}
    g["wh"] = dout.T @ c["feat"]
    g["bh"] = dout.sum(axis=0)
    da = bf16(dout @ bf16(P["wh"])).reshape(acts[4].shape)
    for l in range(3, -1, -1):
        y = acts[l + 1]
        dy = np.where(y > 0, da, 0.0)                      # [B, Co, od, oh, ow]
        Co = CH[l + 1]
        dyf = dy.transpose(0, 2, 3, 4, 1).reshape(-1, Co)  # [B*pos, Co]
        cols = c["cols"][l].reshape(dyf.shape[0], -1)      # [B*pos, Ci*27]
        g[f"w{l}"] = (dyf.T @ cols).reshape(Co, CH[l], 3, 3, 3)
        g[f"b{l}"] = dyf.sum(axis=0)
        if l > 0:
            w = bf16(P[f"w{l}"]).reshape(Co, -1)
            dcols = (dyf @ w).reshape(c["cols"][l].shape[:-1] + (CH[l], 27))
            x_prev = acts[l]
            B_, Ci, D, H, W = x_prev.shape
            dxp = np.zeros((B_, Ci, D + 2, H + 2, W + 2))
            od, oh, ow = dcols.shape[1:4]
            t = 0
            for kd in range(3):
                for kh in range(3):
                    for kw in range(3):
                        dxp[:, :, kd:kd + 2 * od:2, kh:kh + 2 * oh:2, kw:kw + 2 * ow:2] += \
                            dcols[..., t].transpose(0, 4, 1, 2, 3)
                        t += 1
            da = bf16(dxp[:, :, 1:-1, 1:-1, 1:-1])
    flat = []
    for l in range(4):
        flat += [g[f"w{l}"].ravel(), g[f"b{l}"].ravel()]
    flat += [g["wh"].ravel(), g["bh"].ravel()]
    return np.concatenate(flat), out


def pool_fitgrid(imlog, shape=(32, 32, 24)):
    """Warm-start network input: adaptive mean over the finite entries of
    a masked log fitting grid (NaN outside the mask); 0 for empty cells."""
    X, Y, Z = imlog.shape
    out = np.zeros(shape)
    for i in range(shape[0]):
        x0, x1 = i * X // shape[0], -(-(i + 1) * X // shape[0])
        for j in range(shape[1]):
            y0, y1 = j * Y // shape[1], -(-(j + 1) * Y // shape[1])
            for k in range(shape[2]):
                z0, z1 = k * Z // shape[2], -(-(k + 1) * Z // shape[2])
                v = imlog[x0:x1, y0:y1, z0:z1]
                v = v[~np.isnan(v)]
                out[i, j, k] = v.mean() if v.size else 0.0
    return out
