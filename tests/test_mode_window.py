"""Mode source and mode overlap on grids whose spacing differs from the mode's.

The GPU kernels visit only the window of plane cells that can map to a mode
sample (kernels.h `mode_window`); the oracle tests every cell of the plane.
With the grid spacing different from the mode's (ratio 0.5, 0.6, 2) and with
the mode centred near a corner, so that the window is clipped by the plane,
the FP64 fields after the sourced steps and every instantaneous and
accumulated overlap must agree with the oracle (fields: same arithmetic;
overlaps: summation order only, 1e-10 relative).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

from bindings import OracleGrid

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DP = C.POINTER(C.c_double)


def dptr(a):
    return a.ctypes.data_as(DP)


@pytest.mark.gpu
@pytest.mark.parametrize("dx,nx,ny,cx,cy", [
    (0.025, 64, 40, 32, 20),   # ratio 0.5: the 24 x 16 mode covers 48 x 32 cells
    (0.03, 48, 36, 24, 18),    # ratio 0.6
    (0.1, 24, 20, 12, 10),     # ratio 2: the mode covers 12 x 8 cells
    (0.025, 40, 28, 4, 25),    # ratio 0.5, centred near a corner: window clipped at low x and high y
])
def test_source_and_overlap_match_oracle(fd, orc, gpu, dx, nx, ny, cx, cy):
    nz, zs, zm, steps = 14, 4, 7, 12
    dt = 0.99 * dx / math.sqrt(3)
    grid = fd.Grid(nx, ny, nz, dx, fd.F64)
    fd.lib.timefield3d_set_background(grid.t, 2.085, 1.0)
    fd.lib.timefield3d_set_prism_permittivity(grid.t, 12.1, nx // 4, 3 * nx // 4, ny // 3, 2 * ny // 3, 0, nz)
    g = OracleGrid(orc, nx, ny, nz, dx)
    for c in range(3):
        g.ep[c][...] = grid.ep[..., c]
        g.mu[c][...] = grid.mu[..., c]
    mode = fd.read_mode_file(os.path.join(GOLDEN, "modes", "small_te0.txt.gz"))
    m = mode.copy()
    md = mode.copy()
    orc.orc_mode_power_normalize(dptr(md.fields.view(np.float64)), md.mi, md.mj, md.disc)
    omega = 2 * fd.REF_PI / 1.55
    cum = fd.Complex()
    ocum = np.zeros(2)
    for n in range(steps):
        amp = math.exp(-((n - 5) ** 2) / 8.0)
        phase = n * dt * omega
        fd.lib.timefield3d_mode_source(grid.t, cx, cy, zs, m.struct, phase, amp, 0)
        fd.call("timefield3d_apply_timestep_omp_full", grid.t, dt)
        orc.orc_mode_source(g.h, cx, cy, zs, dptr(md.fields.view(np.float64)), md.mi, md.mj, md.disc, phase, amp, 0)
        g.step(dt)
        o = fd.lib.timefield3d_mode_overlap(grid.t, cx, cy, zm, m.struct, phase, 0, C.byref(cum))
        fd.check("overlap")
        oinst = np.zeros(2)
        orc.orc_mode_overlap(g.h, cx, cy, zm, dptr(md.fields.view(np.float64)), md.mi, md.mj, md.disc, phase, 0,
                             dptr(ocum), dptr(oinst))
        assert abs(complex(o.re, o.im) - complex(*oinst)) <= 1e-10 * abs(complex(*oinst)) + 1e-300
    a, b = grid.fields(), g.fields()
    assert np.abs(b).max() > 0
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    assert abs(complex(cum.re, cum.im) - complex(*ocum)) <= 1e-10 * abs(complex(*ocum))
    assert abs(complex(*ocum)) > 0
