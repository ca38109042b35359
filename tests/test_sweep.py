"""Candidate sweeps in persistent launches (fdtd_sweep_run, yee_sweep.cu).

Several grids of different lengths advance together, each by its own step
count, in cooperative launches of S steps that run every grid's one-pass Yee
update, monitors and scheduled source.  Each grid must end exactly as the same
grid run alone with timefield3d_run on the one-pass kernel (FDTD_YEE_STREAM):
fields and monitors bit for bit, also for a second sweep that continues the
first (step counters, field-set parity and source planes handed over).  The
grid barrier's bounded wait is checked on a barrier nothing completes.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

DP = C.POINTER(C.c_double)
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def make_grid(fd, nz, T, boundary, lossy):
    nx, ny, dx = 48, 40, 0.05
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / 1.55
    g = fd.Grid(nx, ny, nz, dx, fd.F32)
    fd.lib.timefield3d_set_background(g.t, 2.085, 1.0)
    fd.lib.timefield3d_set_waveguide(g.t, 12.1, 19, 29, 0, nz, 17, 22)
    if lossy:
        fd.lib.timefield3d_set_prism_electric_conductivity(g.t, 0.3, 10, 20, 8, 16, nz // 3, nz // 2)
    if boundary == "cpml":
        fd.call("timefield3d_set_cpml", g.t, 6, 3, -1.0, 1.0, 0.0)
    else:
        fd.call("timefield3d_set_boundary", g.t, fd.PEC)
    fd.call("timefield3d_set_yee_variant", g.t, fd.YEE_STREAM)
    m = fd.read_mode_file(os.path.join(GOLDEN, "modes", "small_te0.txt.gz"))
    om = np.array([omega * 0.97, omega, omega * 1.03])
    mons = [fd.call("timefield3d_add_overlap_monitor", g.t, 24, 19, z, m.copy().struct, 0, 3, om.ctypes.data_as(DP))
            for z in (16, nz - 14)]
    amps = np.array([math.exp(-((n - 60) ** 2) / (2 * 20.0 ** 2)) for n in range(T)])
    phases = np.array([n * dt * omega for n in range(T)])
    fd.call("timefield3d_set_source_schedule", g.t, 24, 19, 12, m.copy().struct, 0, 0, T, amps.ctypes.data_as(DP),
            phases.ctypes.data_as(DP))
    return g, mons, dt


def monitors(fd, g, mons):
    out = []
    for mon in mons:
        acc = (fd.Complex * 3)()
        fd.call("timefield3d_read_overlap_monitor", g.t, mon, acc)
        out.append([[a.re, a.im] for a in acc])
    return np.array(out)


@pytest.mark.gpu
@pytest.mark.parametrize("boundary,lossy", [("cpml", False), ("pec", True)])
def test_sweep_equals_single_runs(fd, gpu, boundary, lossy):
    nzs, first, second = (44, 60, 76), (150, 97, 203), (40, 71, 0)
    T = 400
    alone = []
    for nz, a, b in zip(nzs, first, second):
        g, mons, dt = make_grid(fd, nz, T, boundary, lossy)
        fd.call("timefield3d_run", g.t, dt, a)
        if b:
            fd.call("timefield3d_run", g.t, dt, b)
        alone.append((g.fields(), monitors(fd, g, mons), fd.lib.timefield3d_step_count(g.t)))
        g.close()
    grids = [make_grid(fd, nz, T, boundary, lossy) for nz in nzs]
    arr = (fd.Timefield3d * 3)(*[g.t for g, _, _ in grids])
    dt = grids[0][2]
    for steps in (first, second):
        n = (C.c_int * 3)(*steps)
        fd.call("fdtd_sweep_run", arr, 3, dt, n, 64, 0, 1.0)
    for (g, mons, _), (f, m, cnt) in zip(grids, alone):
        assert fd.lib.timefield3d_step_count(g.t) == cnt
        assert np.abs(m).max() > 0
        assert np.array_equal(monitors(fd, g, mons), m)
        assert np.array_equal(g.fields(), f)


@pytest.mark.gpu
def test_sweep_barrier_gives_up_and_context_survives(fd, gpu):
    assert fd.lib.fdtd_sweep_barrier_selftest(0.05) == fd.FDTD_ERR_TIMEOUT
    fd.lib.fdtd_clear_error()
    g, mons, dt = make_grid(fd, 44, 64, "cpml", False)
    arr = (fd.Timefield3d * 1)(g.t)
    fd.call("fdtd_sweep_run", arr, 1, dt, (C.c_int * 1)(64), 32, 0, 1.0)
    assert np.abs(monitors(fd, g, mons)).max() > 0


def test_sweep_rejects_bad_arguments(fd):
    # refused on the host before any device work
    assert fd.lib.fdtd_sweep_run(None, 0, 0.01, None, 64, 0, 1.0) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()
    # at most 48 grids a call (their tile arguments sit in constant memory)
    grids = (fd.Timefield3d * 49)()
    steps = (C.c_int * 49)(*([1] * 49))
    assert fd.lib.fdtd_sweep_run(grids, 49, 0.01, steps, 64, 0, 1.0) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()
    assert fd.lib.fdtd_sweep_barrier_selftest(-1.0) in (fd.FDTD_ERR_ARG, fd.FDTD_ERR_NO_DEVICE)
    fd.lib.fdtd_clear_error()
