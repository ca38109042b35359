"""Waveguide modes for the library's runs, from its own GPU mode solver.

strip_mode() builds the rectangular-core cross-section the reference builds
with mode_set_background + mode_make_rectangle (mode.c:2199-2218, 2308-2328)
and solves it with fdtd_mode_solve_beta_squared, the GPU FP64 port of the
reference's restarted Arnoldi beta^2 solver (mode.c:3461-3616), with the
settings the reference's mode files were made with: field confinement 2
(zero field on the window edge), no lateral symmetrisation, so the dominant
eigenvector is the fundamental quasi-TE mode of a Si strip.  The result is a
HostMode usable wherever the reference passes a `mode` (sources, monitors).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

REF_PI = 3.141592652   # the reference driver's pi (3d_fdtd.c:12)


def strip_mode(fd, mi: int, mj: int, disc: float, core: tuple[int, int, int, int], ep_clad: float,
               ep_core: float, lam: float, krylov: int = 20, tol: float = 1e-8):
    """(HostMode, beta): the dominant mode of an mi x mj window (cell disc um)
    with core cells [left, right) x [bottom, top) at wavelength lam um."""
    left, right, bottom, top = core
    ep = np.full((mj, mi, 3), ep_clad, dtype=np.complex128)
    ep[bottom:top, left:right, :] = ep_core
    m = fd.HostMode(np.zeros((mj, mi, 6), dtype=np.complex128), disc, ep, np.ones((mj, mi, 3)))
    omega = 2 * REF_PI / lam
    b = fd.lib.fdtd_mode_solve_beta_squared(C.byref(m.struct), omega, tol, None, 0, krylov, 2, 0)
    fd.check("fdtd_mode_solve_beta_squared")
    beta = complex(b.re, b.im)
    if not (beta.real > 0 and math.isfinite(beta.real)):
        raise RuntimeError(f"mode solver returned beta {beta}")
    return m, beta
