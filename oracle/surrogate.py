"""Test infrastructure: FP64 CPU restatement of the surrogate network
(3d_fdtd_b200/csrc/surrogate.cu) -- MLP n_in -> H -> H -> H -> n_out, GELU,
MSE loss, backward, Adam.

With `bf16=True` the operands of every matrix product are rounded to bfloat16
(round to nearest even) where the GPU rounds them: the input, the weights, the
hidden activations and the back-propagated dZ; products and everything else
are FP64.  With `bf16=False` it is the exact FP64 network, whose gradients the
tests check against central finite differences.  Only tests import this.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unflatten(flat: np.ndarray, n_in: int, hid: int, n_out: int):
    """Flat [W1, b1, ..., W4, b4] (W [out][in]) -> list of (W, b)."""
    dims = [(hid, n_in), (hid, hid), (hid, hid), (n_out, hid)]
    out, off = [], 0
    for o, i in dims:
        W = flat[off:off + o * i].reshape(o, i).astype(np.float64)
        off += o * i
        b = flat[off:off + o].astype(np.float64)
        off += o
        out.append((W, b))
    return out


def flatten(params) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in params])


def forward(params, x, bf=True):
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    h = r(x)
    Zs, Hs = [], [h]
    for l, (W, b) in enumerate(params):
        z = h @ r(W).T + b
        if l < len(params) - 1:
            Zs.append(z)
            h = r(gelu(z))
            Hs.append(h)
        else:
            return z, Zs, Hs
    raise AssertionError


def gradients(params, x, t, bf=True):
    """Loss (mean squared error) and gradients [(dW, db)], and dL/dx."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    y, Zs, Hs = forward(params, x, bf)
    B, n = y.shape
    loss = float(((y - t) ** 2).sum() / (B * n))
    dz = 2.0 * (y - t) / (B * n)
    grads = [None] * len(params)
    for l in range(len(params) - 1, -1, -1):
        W, _ = params[l]
        dzr = r(dz)
        grads[l] = (dzr.T @ Hs[l], dz.sum(axis=0))
        dh = dzr @ r(W)
        if l > 0:
            dz = dh * gelu_grad(Zs[l - 1])
        else:
            dx = dh
    return loss, grads, dx


def input_gradient(params, x, dy, bf=True):
    """(dY/dX)^T dy."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    _, Zs, _ = forward(params, x, bf)
    dz = dy
    for l in range(len(params) - 1, -1, -1):
        dh = r(dz) @ r(params[l][0])
        if l > 0:
            dz = dh * gelu_grad(Zs[l - 1])
    return dh


def adam(params, grads, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (bias-corrected), returning new params and moments."""
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    out, mo, vo = [], [], []
    for (W, b), (gW, gb), (mW, mb), (vW, vb) in zip(params, grads, m, v):
        new = []
        for p, g, mm, vv in ((W, gW, mW, vW), (b, gb, mb, vb)):
            mm = b1 * mm + (1 - b1) * g
            vv = b2 * vv + (1 - b2) * g * g
            new.append((p - lr * (mm / c1) / (np.sqrt(vv / c2) + eps), mm, vv))
        out.append((new[0][0], new[1][0]))
        mo.append((new[0][1], new[1][1]))
        vo.append((new[0][2], new[1][2]))
    return out, mo, vo
