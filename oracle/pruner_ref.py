"""CPU restatement of the learned pruner's network (include/celv2_pruner.h), in numpy.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA forward / backward kernels (csrc/pruner.cu) and
of the features; nothing in the product path imports it. With `bf16=True` every GEMM operand is
rounded to BF16 (round to nearest even) as the tensor-core kernels round it, and the products
accumulate in float64 (the kernels: FP32); with `bf=False` it is the same network in float64 with
no rounding, whose gradients the finite-difference test checks.
"""
from __future__ import annotations

import numpy as np

FEATURES, OUTPUTS = 376, 24
SHAPES = [("W1", (16, 9)), ("b1", (16,)), ("W2", (32, 144)), ("b2", (32,)), ("W3", (32, 288)), ("b3", (32,)),
          ("W4", (64, 632)), ("b4", (64,)), ("W5", (OUTPUTS, 64)), ("b5", (OUTPUTS,))]
PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float32 (the value
    the tensor cores multiply; finite values only)."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    b = (b + (((b >> 16) & 1) + 0x7FFF)) & np.uint32(0xFFFF0000)
    return b.view(np.float32)


def _mm(a, b, rnd):
    if rnd:
        return (bf16(a).astype(np.float64) @ bf16(b).astype(np.float64)).astype(np.float32)
    return a.astype(np.float64) @ b.astype(np.float64)


def im2col(x: np.ndarray, s: int) -> np.ndarray:
    """x [B, H, W, C] -> [B * Ho * Wo, 9 * C], column (ky * 3 + kx) * C + c, padding 1, stride s."""
    B, H, W, C = x.shape
    Ho, Wo = (H - 1) // s + 1, (W - 1) // s + 1
    xp = np.zeros((B, H + 2, W + 2, C), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = np.empty((B, Ho, Wo, 3, 3, C), x.dtype)
    for ky in range(3):
        for kx in range(3):
            cols[:, :, :, ky, kx] = xp[:, ky:ky + s * (Ho - 1) + 1:s, kx:kx + s * (Wo - 1) + 1:s]
    return cols.reshape(B * Ho * Wo, 9 * C)


def col2im(d: np.ndarray, B: int, H: int, W: int, C: int, s: int) -> np.ndarray:
    Ho, Wo = (H - 1) // s + 1, (W - 1) // s + 1
    d = d.reshape(B, Ho, Wo, 3, 3, C)
    xp = np.zeros((B, H + 2, W + 2, C), d.dtype)
    for ky in range(3):
        for kx in range(3):
            xp[:, ky:ky + s * (Ho - 1) + 1:s, kx:kx + s * (Wo - 1) + 1:s] += d[:, :, :, ky, kx]
    return xp[:, 1:-1, 1:-1]


def forward(p: np.ndarray, x: np.ndarray, bf: bool = True):
    """(logits [B, OUTPUTS], cache)."""
    dt = np.float32 if bf else np.float64
    P = {k: v.astype(dt) for k, v in unpack(p).items()}
    x = x.astype(dt)
    B = x.shape[0]
    c = {}
    c["cols1"] = im2col(x[:, :256].reshape(B, 16, 16, 1), 1)
    c["a1"] = np.maximum(_mm(c["cols1"], P["W1"].T, bf) + P["b1"], 0).reshape(B, 16, 16, 16)
    c["cols2"] = im2col(c["a1"], 2)
    c["a2"] = np.maximum(_mm(c["cols2"], P["W2"].T, bf) + P["b2"], 0).reshape(B, 8, 8, 32)
    c["cols3"] = im2col(c["a2"], 2)
    c["a3"] = np.maximum(_mm(c["cols3"], P["W3"].T, bf) + P["b3"], 0).reshape(B, 512)
    c["h0"] = np.concatenate([c["a3"], x[:, 256:]], axis=1)
    c["a4"] = np.maximum(_mm(c["h0"], P["W4"].T, bf) + P["b4"], 0)
    logits = _mm(c["a4"], P["W5"].T, bf) + P["b5"]
    return logits.astype(dt), c


def backward(p: np.ndarray, c: dict, dlogits: np.ndarray, bf: bool = True) -> np.ndarray:
    """The gradient of every parameter, flattened like p."""
    dt = np.float32 if bf else np.float64
    P = {k: v.astype(dt) for k, v in unpack(p).items()}
    dlogits = dlogits.astype(dt)
    B = dlogits.shape[0]
    g = {}
    g["W5"] = _mm(dlogits.T, c["a4"], bf)
    g["b5"] = dlogits.sum(0)
    dz4 = _mm(dlogits, P["W5"], bf) * (c["a4"] > 0)
    g["W4"] = _mm(dz4.T, c["h0"], bf)
    g["b4"] = dz4.sum(0)
    dz3 = (_mm(dz4, P["W4"][:, :512], bf) * (c["a3"] > 0)).reshape(B * 16, 32)
    g["W3"] = _mm(dz3.T, c["cols3"], bf)
    g["b3"] = dz3.sum(0)
    dz2 = col2im(_mm(dz3, P["W3"], bf), B, 8, 8, 32, 2) * (c["a2"] > 0)
    dz2 = dz2.reshape(B * 64, 32)
    g["W2"] = _mm(dz2.T, c["cols2"], bf)
    g["b2"] = dz2.sum(0)
    dz1 = col2im(_mm(dz2, P["W2"], bf), B, 16, 16, 16, 2) * (c["a1"] > 0)
    dz1 = dz1.reshape(B * 256, 16)
    g["W1"] = _mm(dz1.T, c["cols1"], bf)
    g["b1"] = dz1.sum(0)
    return np.concatenate([g[name].reshape(-1) for name, _ in SHAPES]).astype(dt)


def bce(logits: np.ndarray, labels: np.ndarray, weights: np.ndarray):
    """(mean weighted binary cross-entropy, dlogits), as celv2_pruner_bce."""
    B = logits.shape[0]
    z = logits.astype(np.float64)
    loss = weights * (np.maximum(z, 0) - z * labels + np.log1p(np.exp(-np.abs(z))))
    d = weights * (1 / (1 + np.exp(-z)) - labels) / B
    return float(loss.sum() / B), d.astype(np.float32)
