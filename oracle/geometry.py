"""Test infrastructure: CPU restatement of the spline taper rasteriser.

The engine's timefield3d_set_spline_taper has no reference counterpart; it
generalises timefield3d_set_taper (timefield3d.c:1511-1535) from straight
integer edges to a natural-cubic-spline width with sub-pixel fill.  This file
restates its fill rule in numpy (same IEEE operations, no fused multiply-add)
so that tests can compare the library's ep/mu arrays bit for bit; the spline
weights themselves are checked against scipy's natural CubicSpline.
Only tests import this module.
"""
from __future__ import annotations

import numpy as np


def spline_edges(W: np.ndarray, widths, center_x: float, disc: float):
    """Core x-extent [xl, xr) per plane from the weights W[k, c] (library order)."""
    w = np.zeros(W.shape[0])
    for c in range(W.shape[1]):          # same summation order as the library
        w = w + W[:, c] * widths[c]
    half = w / (2.0 * disc)
    return center_x - half, center_x + half


def raster(ep: np.ndarray, mu: np.ndarray, xl, xr, ep_core: float, mu_core: float, start_z: int, bottom: int,
           top: int) -> None:
    """Fill ep/mu, shaped (nz, ny, nx, 3) float32, in place: cell i of plane k
    covered by f = min(i+1, xr) - max(i, xl); f >= 1 -> the core value, 0 < f < 1
    -> old + f (core - old) in double, rounded to float."""
    nx = ep.shape[2]
    i = np.arange(nx, dtype=np.float64)
    for kk in range(len(xl)):
        k = start_z + kk
        f = np.minimum(i + 1.0, xr[kk]) - np.maximum(i, xl[kk])
        full = f >= 1.0
        part = (f > 0.0) & ~full
        for arr, core in ((ep, ep_core), (mu, mu_core)):
            blk = arr[k, bottom:top]                      # (rows, nx, 3) view
            old = blk[:, part, :].astype(np.float64)
            blk[:, part, :] = (old + f[part][None, :, None] * (core - old)).astype(np.float32)
            blk[:, full, :] = np.float32(core)
