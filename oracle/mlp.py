"""CPU oracle of the learned smoothing-length seed's network (8 -> 64 -> 64 -> 1).

TEST INFRASTRUCTURE ONLY: the product never imports this module.  The network
has no counterpart in the reference (density.metal:73-143 starts its
iteration from the particle's own h); this module restates, in numpy FP64,
exactly the arithmetic the GPU kernels perform, including where they round to
BF16 (the tensor-core operands), so the GPU gradients can be checked against
it:

  x   = (X[rows] - mean) * inv_dev              -> BF16 (operand of layer 1)
  z1  = x W1^T + b1      (W1 in BF16)           ; h1 = relu(z1) -> BF16
  z2  = h1 W2^T + b2     (W2 in BF16)           ; h2 = relu(z2) (FP32)
  yh  = h2 . w3 + b3                            ; t = (y[rows] - t_mean) / t_dev
  loss = 1/2 mean (yh - t)^2
  dy  = (yh - t) / B
  g2  = dy w3 (.) [z2 > 0]      -> BF16 for the MMAs; FP32 for db2
  g1  = (g2 W2) (.) [z1 > 0]    -> BF16 for dW1; FP32 for db1
  dW2 = g2^T h1 ; dW1 = g1^T x ; dw3 = h2^T dy ; db3 = sum dy

Parameter order: W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 8, 64
SIZES = (("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)), ("w3", (N_HID,)),
         ("b3", (1,)))
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SIZES])


def bf16(a) -> np.ndarray:
    """Round float32 values to BF16 (round to nearest even), returned as FP64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


def sample_rows(batch: int, salt: int, n: int, it: int = 0) -> np.ndarray:
    """Row r of a minibatch: ((it * batch + r) * 0x9E3779B97F4A7C15 ^ salt) mod n, modulo 2^64."""
    g = (np.uint64(it) * np.uint64(batch) + np.arange(batch, dtype=np.uint64))
    with np.errstate(over="ignore"):
        h = (g * np.uint64(0x9E3779B97F4A7C15)) ^ np.uint64(salt)
    return (h % np.uint64(n)).astype(np.int64)


def forward_backward(params: np.ndarray, X: np.ndarray, y: np.ndarray, norm: np.ndarray, rows: np.ndarray,
                     rounding: bool = True):
    """(loss, gradient) over the given rows; rounding=False drops the BF16
    rounding (plain FP64 backpropagation, for the finite-difference check)."""
    P = unpack(params)
    rnd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    B = rows.size
    mean, inv_dev = norm[:N_IN].astype(np.float64), norm[N_IN:2 * N_IN].astype(np.float64)
    t_mean, t_dev = float(norm[2 * N_IN]), float(norm[2 * N_IN + 1])
    if rounding:  # the kernel standardises in float32
        x = bf16((X[rows].astype(np.float32) - norm[:N_IN].astype(np.float32))
                 * norm[N_IN:2 * N_IN].astype(np.float32))
    else:
        x = (X[rows].astype(np.float64) - mean) * inv_dev
    W1 = bf16(P["W1"].astype(np.float32)) if rounding else P["W1"]
    W2 = bf16(P["W2"].astype(np.float32)) if rounding else P["W2"]
    z1 = x @ W1.T + P["b1"]
    h1 = rnd(np.maximum(z1, 0.0).astype(np.float32) if rounding else np.maximum(z1, 0.0))
    z2 = h1 @ W2.T + P["b2"]
    h2 = np.maximum(z2, 0.0)
    yh = h2 @ P["w3"] + P["b3"][0]
    t = (y[rows].astype(np.float64) - t_mean) / t_dev
    loss = 0.5 * float(np.mean((yh - t) ** 2))
    dy = (yh - t) / B
    g2 = dy[:, None] * P["w3"][None, :] * (z2 > 0)
    g2r = rnd(g2.astype(np.float32) if rounding else g2)
    g1 = (g2r @ W2) * (z1 > 0)
    g1r = rnd(g1.astype(np.float32) if rounding else g1)
    grad = dict(W1=g1r.T @ x, b1=g1.sum(0), W2=g2r.T @ h1, b2=g2.sum(0), w3=h2.T @ dy, b3=np.array([dy.sum()]))
    return loss, pack(grad)


def predict(params: np.ndarray, X: np.ndarray, norm: np.ndarray) -> np.ndarray:
    """Standardised-target predictions (no rounding), for inspection."""
    P = unpack(params)
    x = (X.astype(np.float64) - norm[:N_IN]) * norm[N_IN:2 * N_IN]
    h1 = np.maximum(x @ P["W1"].T + P["b1"], 0.0)
    h2 = np.maximum(h1 @ P["W2"].T + P["b2"], 0.0)
    return h2 @ P["w3"] + P["b3"][0]
