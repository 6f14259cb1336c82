"""Float64 CPU reference of the learned scheduler's MLP -- TEST INFRASTRUCTURE.

Checks the hand-written CUDA forward/backward kernels (pumatch_b200/csrc/
pm_learn.cu): 16 -> 64 -> 64 -> 2, ReLU, weights rounded to bfloat16 (the GPU
computes with the BF16 copy of its FP32 master weights), loss = mean over
samples and outputs of the squared error.  Parameter layout (input-major):
W1[16][64] b1[64] W2[64][64] b2[64] W3[64][2] b3[2].
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 16, 64, 2
SHAPES = [("W1", (NIN, NH)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NOUT)), ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def to_bf16(w: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), as float64."""
    u = np.asarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat: np.ndarray):
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = flat[off:off + n].reshape(shape)
        off += n
    return out


def forward(flat: np.ndarray, x: np.ndarray) -> np.ndarray:
    p = unpack(to_bf16(flat))
    h1 = np.maximum(x.astype(np.float64) @ p["W1"] + p["b1"], 0.0)
    h2 = np.maximum(h1 @ p["W2"] + p["b2"], 0.0)
    return h2 @ p["W3"] + p["b3"]


def loss_and_grad(flat: np.ndarray, x: np.ndarray, t: np.ndarray):
    """MSE loss and its gradient w.r.t. the (bf16-rounded) parameters."""
    p = unpack(to_bf16(flat))
    x = x.astype(np.float64)
    t = t.astype(np.float64)
    n = x.shape[0]
    z1 = x @ p["W1"] + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"] + p["b2"]
    h2 = np.maximum(z2, 0.0)
    out = h2 @ p["W3"] + p["b3"]
    err = out - t
    loss = float((err ** 2).sum() / (n * NOUT))
    dout = 2.0 * err / (n * NOUT)
    g = {"W3": h2.T @ dout, "b3": dout.sum(0)}
    dz2 = (dout @ p["W3"].T) * (z2 > 0)
    g["W2"] = h1.T @ dz2
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"].T) * (z1 > 0)
    g["W1"] = x.T @ dz1
    g["b1"] = dz1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])
