"""CPU oracle of the learned warm start's network (TEST INFRASTRUCTURE ONLY:
imported by tests/ and by the smoke check, never by the product path).

The network has no counterpart in the reference; this file restates, in
numpy, what the CUDA kernels of pdot.jl_b200/csrc/pdot_mlp.cu compute:

    X  = bf16((log(max(h, 1e-30)) + shift) * scale)
    Z1 = X W1^T + b1,  H1 = bf16(gelu(Z1))
    Z2 = H1 W2^T + b2, H2 = bf16(gelu(Z2))
    Y  = H2 W3^T + b3
    loss = mean over the batch rows and outputs of (Y - T)^2
    dY = 2 (Y - T) / (batch * outputs)
    dW3 = bf16(dY)^T H2,  db3 = sum_rows dY
    dZ2 = (bf16(dY) W3) * gelu'(Z2),  dW2 = bf16(dZ2)^T H1,  db2 = sum_rows dZ2
    dZ1 = (bf16(dZ2) W2) * gelu'(Z1), dW1 = bf16(dZ1)^T X,   db1 = sum_rows dZ1

with the weights rounded to BF16 for the products (the FP32 masters are the
parameters) and the products accumulated here in FP64 (the GPU accumulates in
FP32). With `bf16=False` nothing is rounded and the backward pass is the exact
gradient of the forward one, which the CPU tests check by finite differences.

Parameter vector layout (as pdot_mlp_get_parameters): W1 [H x I] row-major,
b1 [H], W2 [H x H], b2 [H], W3 [O x H], b3 [O].
"""
from __future__ import annotations

import math

import numpy as np

_SQRT1_2 = 1.0 / math.sqrt(2.0)
_INV_SQRT_2PI = 1.0 / math.sqrt(2.0 * math.pi)


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _erf(x):
    from scipy.special import erf

    return erf(x)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z * _SQRT1_2))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z * _SQRT1_2)) + z * _INV_SQRT_2PI * np.exp(-0.5 * z * z)


def unpack(theta: np.ndarray, I: int, H: int, O: int):
    sizes = [H * I, H, H * H, H, O * H, O]
    parts, off = [], 0
    for s in sizes:
        parts.append(np.asarray(theta[off : off + s], dtype=np.float64))
        off += s
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(H, I), b1, W2.reshape(H, H), b2, W3.reshape(O, H), b3


def features(hist: np.ndarray, shift: float, scale: float, round_bf16: bool = True) -> np.ndarray:
    x = (np.log(np.maximum(np.asarray(hist, dtype=np.float64), 1e-30)) + shift) * scale
    return bf16(x) if round_bf16 else x


def forward(theta, x, I, H, O, round_bf16: bool = True):
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(theta, I, H, O)
    z1 = x @ r(W1).T + b1
    h1 = r(gelu(z1))
    z2 = h1 @ r(W2).T + b2
    h2 = r(gelu(z2))
    y = h2 @ r(W3).T + b3
    return y, (x, z1, h1, z2, h2)


def loss_and_gradients(theta, x, target, I, H, O, round_bf16: bool = True):
    """(loss, gradient vector) in the parameter layout."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(theta, I, H, O)
    y, (x, z1, h1, z2, h2) = forward(theta, x, I, H, O, round_bf16)
    B = x.shape[0]
    diff = y - np.asarray(target, dtype=np.float64)
    loss = float(np.sum(diff * diff) / (B * O))
    dy = 2.0 * diff / (B * O)
    dyb = r(dy)
    gW3 = dyb.T @ h2
    gb3 = dy.sum(axis=0)
    dz2 = (dyb @ r(W3)) * gelu_grad(z2)
    dz2b = r(dz2)
    gW2 = dz2b.T @ h1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2b @ r(W2)) * gelu_grad(z1)
    dz1b = r(dz1)
    gW1 = dz1b.T @ x
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def adamw(theta, grad, m, v, step, lr, beta1, beta2, eps, weight_decay, I, H, O):
    """One AdamW step in place (decay on the weight matrices, not the biases)."""
    sizes = [H * I, H, H * H, H, O * H, O]
    c1 = 1.0 - beta1**step
    c2 = 1.0 - beta2**step
    off = 0
    for k, s in enumerate(sizes):
        sl = slice(off, off + s)
        m[sl] = beta1 * m[sl] + (1 - beta1) * grad[sl]
        v[sl] = beta2 * v[sl] + (1 - beta2) * grad[sl] ** 2
        wd = weight_decay if k % 2 == 0 else 0.0
        theta[sl] = theta[sl] - lr * ((m[sl] / c1) / (np.sqrt(v[sl] / c2) + eps) + wd * theta[sl])
        off += s
