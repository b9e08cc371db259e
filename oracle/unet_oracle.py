"""FP64 CPU reference of the learned preconditioner's network (test infrastructure only).

The learned part has no counterpart in the reference project; this file is its oracle.  The GPU
kernels (fluidisim_b200/csrc/fd3_unet.cuh) are checked against it; it is itself checked against
finite differences.  Only tests/ use it.

Layout: channels-last, one sample at a time, x[z, y, x, c].  Convolutions are 3x3x3 with zero
padding ("same"), weights w[tap, cout, cin] with tap = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1), and a
bias per output channel.  The network (`UNet`):

    x0 = input (3 channels: residual, solid mask, liquid mask)
    e0 = relu(conv(x0; 3 -> 16))                       full resolution
    e1 = relu(conv(pool(e0); 16 -> 32))                1/2
    b  = relu(conv(pool(e1); 32 -> 64))                1/4
    d1 = relu(conv(cat(up(b), e1); 96 -> 32))          1/2
    d0 = relu(conv(cat(up(d1), e0); 48 -> 16))         full
    y  = conv(d0; 16 -> 1)                             full, no activation

pool is the mean of 2 x 2 x 2 children, up the nearest-neighbour copy to the 8 children, cat the
channel concatenation (upsampled first, then the skip).
"""
from __future__ import annotations

import numpy as np

TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]

# (name, cin, cout, relu) in execution order
LAYERS = [("e0", 3, 16, True), ("e1", 16, 32, True), ("b", 32, 64, True), ("d1", 96, 32, True),
          ("d0", 48, 16, True), ("head", 16, 1, False)]


def shift(x, dz, dy, dx):
    """out[z, y, x] = x[z + dz, y + dy, x + dx], zero outside."""
    Z, Y, X = x.shape[:3]
    out = np.zeros_like(x)
    zs, zd = (slice(dz, Z), slice(0, Z - dz)) if dz >= 0 else (slice(0, Z + dz), slice(-dz, Z))
    ys, yd = (slice(dy, Y), slice(0, Y - dy)) if dy >= 0 else (slice(0, Y + dy), slice(-dy, Y))
    xs, xd = (slice(dx, X), slice(0, X - dx)) if dx >= 0 else (slice(0, X + dx), slice(-dx, X))
    out[zd, yd, xd] = x[zs, ys, xs]
    return out


def conv(x, w, b):
    y = np.zeros(x.shape[:3] + (w.shape[1],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += shift(x, dz, dy, dx) @ w[t].T
    return y + b


def conv_backward(x, w, gy):
    """(gx, gw, gb) of conv for the upstream gradient gy."""
    gx = np.zeros_like(x)
    gw = np.zeros_like(w)
    for t, (dz, dy, dx) in enumerate(TAPS):
        xs = shift(x, dz, dy, dx)
        gw[t] = gy.reshape(-1, gy.shape[-1]).T @ xs.reshape(-1, xs.shape[-1])
        gx += shift(gy @ w[t], -dz, -dy, -dx)
    return gx, gw, gy.reshape(-1, gy.shape[-1]).sum(axis=0)


def pool(x):
    Z, Y, X, C = x.shape
    return x.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(1, 3, 5))


def pool_backward(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)


def up_backward(g):
    Z, Y, X, C = g.shape
    return g.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(1, 3, 5))


def bf16(x):
    """Round to bfloat16 (round to nearest, ties to even), returned in float64."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _ident(x):
    return x


def init_params(seed: int = 0, scale: float = 1.0):
    """He-style initialisation: w ~ N(0, 2 / (27 cin)), bias 0 (the head's scaled down)."""
    rng = np.random.default_rng(seed)
    params = {}
    for name, cin, cout, relu in LAYERS:
        std = scale * np.sqrt(2.0 / (27 * cin)) * (1.0 if relu else 0.1)
        params[name + ".w"] = rng.normal(0.0, std, size=(27, cout, cin))
        params[name + ".b"] = np.zeros(cout)
    return params


class UNet:
    """Forward with the activations kept, and the backward pass.

    With round_bf16, every tensor the GPU stores in BF16 (inputs, weights, activations, pooled
    and upsampled tensors, activation gradients) is rounded to BF16 where the GPU rounds it; the
    arithmetic in between stays FP64.  That isolates the GPU's accumulation from its storage
    precision: the GPU must then agree to accumulation-order rounding."""

    def __init__(self, params, round_bf16: bool = False):
        self.r = bf16 if round_bf16 else _ident
        self.p = {k: (self.r(v) if k.endswith(".w") else v) for k, v in params.items()}

    def forward(self, x0):
        p, r = self.p, self.r
        c = {}
        c["x0"] = r(x0)
        c["e0"] = r(np.maximum(conv(c["x0"], p["e0.w"], p["e0.b"]), 0))
        c["p0"] = r(pool(c["e0"]))
        c["e1"] = r(np.maximum(conv(c["p0"], p["e1.w"], p["e1.b"]), 0))
        c["p1"] = r(pool(c["e1"]))
        c["b"] = r(np.maximum(conv(c["p1"], p["b.w"], p["b.b"]), 0))
        c["c1"] = np.concatenate([up(c["b"]), c["e1"]], axis=-1)
        c["d1"] = r(np.maximum(conv(c["c1"], p["d1.w"], p["d1.b"]), 0))
        c["c0"] = np.concatenate([up(c["d1"]), c["e0"]], axis=-1)
        c["d0"] = r(np.maximum(conv(c["c0"], p["d0.w"], p["d0.b"]), 0))
        c["y"] = conv(c["d0"], p["head.w"], p["head.b"])
        self.c = c
        return c["y"]

    def backward(self, gy):
        """Parameter gradients (and the input gradient) for dL/dy = gy."""
        p, c, g, r = self.p, self.c, {}, self.r
        gy = r(gy)
        gd0, g["head.w"], g["head.b"] = conv_backward(c["d0"], p["head.w"], gy)
        gd0 = r(gd0) * (c["d0"] > 0)
        gc0, g["d0.w"], g["d0.b"] = conv_backward(c["c0"], p["d0.w"], gd0)
        gc0 = r(gc0)
        nd1 = c["d1"].shape[-1]
        gd1 = r(up_backward(gc0[..., :nd1]) * (c["d1"] > 0))
        ge0 = gc0[..., nd1:]
        gc1, g["d1.w"], g["d1.b"] = conv_backward(c["c1"], p["d1.w"], gd1)
        gc1 = r(gc1)
        nb = c["b"].shape[-1]
        gb = r(up_backward(gc1[..., :nb]) * (c["b"] > 0))
        ge1 = gc1[..., nb:]
        gp1, g["b.w"], g["b.b"] = conv_backward(c["p1"], p["b.w"], gb)
        gp1 = r(gp1)
        ge1 = r((ge1 + pool_backward(gp1)) * (c["e1"] > 0))
        gp0, g["e1.w"], g["e1.b"] = conv_backward(c["p0"], p["e1.w"], ge1)
        gp0 = r(gp0)
        ge0 = r((ge0 + pool_backward(gp0)) * (c["e0"] > 0))
        gx0, g["e0.w"], g["e0.b"] = conv_backward(c["x0"], p["e0.w"], ge0)
        g["x0"] = gx0
        return g
