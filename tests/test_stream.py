"""The one-pass streaming FP32 Yee kernel (FDTD_YEE_STREAM, yee_stream.cu).

CPU: its tile plan (host computation) covers every interior (row, plane) of
the grid exactly once, within the block's row capacity, thread and shared
memory limits, with no more tiles than SMs.
GPU: it computes the same fields and monitors as the flat kernel pair (flat4:
separate E and H launches, the same per-cell expressions) up to FP32 rounding
-- the two compile to different multiply-add contractions, measured 2e-7 to 7e-7
of the peak field after 64-200 steps -- through timefield3d_run (captured
graphs, scheduled mode source, step-tail monitors) on the small taper, and on
the full 200x160x400 CPML grid.
Parity with the FP64 CPU restatement is in test_gpu_parity.py
(test_fused_f32_matches_oracle, variant "stream").
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

from make_golden import wg_geometry, wg_setup

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SMEM_MAX = 231424


def plan(fd, nx, ny, nz, L, lossy, nsm):
    ty, th, sm = C.c_int(), C.c_int(), C.c_longlong()
    n = fd.lib.fdtd_stream_plan(nx, ny, nz, L, lossy, nsm, None, 0, C.byref(ty), C.byref(th), C.byref(sm))
    if n < 0:
        return None
    buf = (C.c_int * (4 * n))()
    assert fd.lib.fdtd_stream_plan(nx, ny, nz, L, lossy, nsm, buf, n, C.byref(ty), C.byref(th), C.byref(sm)) == n
    return np.array(buf, dtype=np.int64).reshape(n, 4), ty.value, th.value, sm.value


@pytest.mark.parametrize("nx,ny,nz,L,lossy,nsm", [
    (200, 160, 400, 12, 0, 148),   # the Si taper workload
    (200, 160, 400, 12, 1, 148),
    (256, 128, 96, 12, 0, 148),    # shortest and longest candidates of the taper sweep
    (256, 128, 384, 12, 0, 148),
    (64, 64, 64, 8, 0, 148),
    (40, 28, 72, 6, 1, 148),
    (36, 21, 30, 5, 0, 148),       # odd CPML thickness: x-slab rows staged in 4-byte pieces
    (20, 16, 24, 4, 0, 148),
    (8, 3, 3, 0, 0, 1),            # one interior cell row
    (512, 40, 50, 0, 0, 132),
    (200, 160, 400, 12, 0, 18),    # one grid's share of an 8-grid sweep: more bands than tiles asked for
])
def test_stream_plan_covers_interior_once(fd, nx, ny, nz, L, lossy, nsm):
    p = plan(fd, nx, ny, nz, L, lossy, nsm)
    assert p is not None
    tiles, ty, threads, smem = p
    bands = len({t[0] for t in tiles})
    assert 1 <= len(tiles) <= max(nsm, bands)
    # 16 warps x 128 registers fit an SM; the cells of the x-slab quads (row
    # ends) get a thread each, in warps of their own
    qx = nx // 4
    if L:
        ql, qr = (L + 3) // 4, max((L + 3) // 4, min(qx, (nx - L) // 4))
        qi = qr - ql
        want = ((ty + 1) * qi + 31) // 32 * 32 + (ty + 1) * 4 * (qx - qi)
    else:
        want = (ty + 1) * qx
    assert threads % 32 == 0 and threads == (want + 31) // 32 * 32 and threads <= 512
    na = 12 if lossy else 9
    xw = (2 * L + 3) // 4 * 4   # staged x-slab auxiliaries per row, padded to 16 bytes
    ptab = 3 * 6 * 2 * L        # slab-cell profiles: 3 axes x 6 profiles x 2L cells
    assert smem == ((3 * na * (ty + 1) + 6 + 6 * (ty + 1)) * nx + 3 * 4 * (ty + 1) * xw + ptab) * 4 <= SMEM_MAX
    owned = np.zeros((nz, ny), dtype=np.int64)
    for j0, rows, k0, k1 in tiles:
        assert 1 <= rows <= ty and j0 >= 1 and j0 + rows <= ny - 1
        assert 1 <= k0 < k1 <= nz - 1
        owned[k0:k1, j0:j0 + rows] += 1
    assert (owned[1:-1, 1:-1] == 1).all() and owned.sum() == (nz - 2) * (ny - 2)
    if L:
        # bands are cut where the lower y slab ends and one row below where the
        # upper one begins: an interior band holds no y-slab row, and its halo
        # row (the row above its last) is no y-slab row either
        def slab(j):
            return j < L or j >= ny - L
        for j0, rows in {(t[0], t[1]) for t in tiles}:
            band = [slab(j) for j in range(j0, j0 + rows)]
            if not any(band):
                halo = j0 + rows
                assert not (slab(halo) and halo < ny - 1), (j0, rows)
            elif j0 < L:
                assert all(band), (j0, rows)
        # the first row past the lower slab and the row below the upper slab
        # start bands
        starts = {t[0] for t in tiles}
        if L < ny - L - 1:
            assert L in starts and ny - L - 1 in starts


def test_stream_plan_rejects_unsupported(fd):
    ty, th, sm = C.c_int(), C.c_int(), C.c_longlong()
    for args in ((37, 19, 45, 6, 0, 148),     # nx not a multiple of 4
                 (4096, 40, 40, 0, 0, 148),   # a row and its halo row need more than a block's threads
                 (40, 2, 40, 0, 0, 148),      # no interior row
                 (40, 20, 40, 0, 0, 0)):
        assert fd.lib.fdtd_stream_plan(*args, None, 0, C.byref(ty), C.byref(th), C.byref(sm)) == -1


def taper_run(fd, variant, T, steps):
    p = wg_setup()
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    b, t = p["core"]
    cx, cy = nx // 2, (b + t) // 2
    grid = fd.Grid(nx, ny, nz, dx, fd.F32)
    wg_geometry(fd.lib, grid.t, p, None, None)
    fd.call("timefield3d_set_cpml", grid.t, 6, 3, -1.0, 1.0, 0.0)
    fd.call("timefield3d_set_yee_variant", grid.t, variant)
    m = fd.read_mode_file(os.path.join(GOLDEN, "modes", "small_te0.txt.gz"))
    om = np.array([omega * 0.97, omega, omega * 1.03])
    dp = C.POINTER(C.c_double)
    mons = [fd.call("timefield3d_add_overlap_monitor", grid.t, cx, cy, z, m.copy().struct, 0, 3,
                    om.ctypes.data_as(dp)) for z in (p["launch_z"], p["out_z"])]
    amps = np.array([math.exp(-((n - 60) ** 2) / (2 * 20.0 ** 2)) for n in range(T)])
    phases = np.array([n * dt * omega for n in range(T)])
    fd.call("timefield3d_set_source_schedule", grid.t, cx, cy, p["src_z"], m.copy().struct, 0, 0, T,
            amps.ctypes.data_as(dp), phases.ctypes.data_as(dp))
    for s in steps:   # several runs: graph replays, a leftover odd count, a run after it
        fd.call("timefield3d_run", grid.t, dt, s)
    out = []
    for mon in mons:
        acc = (fd.Complex * 3)()
        fd.call("timefield3d_read_overlap_monitor", grid.t, mon, acc)
        out.append([[a.re, a.im] for a in acc])
    return grid.fields(), np.array(out)


@pytest.mark.gpu
def test_stream_matches_flat4_through_runs(fd, gpu):
    steps = (96, 33, 71)
    fa, ma = taper_run(fd, fd.YEE_FLAT4, sum(steps), steps)
    fb, mb = taper_run(fd, fd.YEE_STREAM, sum(steps), steps)
    assert np.abs(ma).max() > 0
    assert np.abs(fa - fb).max() <= 5e-6 * np.abs(fa).max()
    assert np.abs(ma - mb).max() <= 5e-6 * np.abs(ma).max()


@pytest.mark.gpu
def test_stream_matches_flat4_on_si_taper_grid(fd, gpu):
    # the bench workload's grid and materials, 64 steps of the scheduled TE0 source
    import bench
    out = []
    for variant in (fd.YEE_FLAT4, fd.YEE_STREAM):
        sim = bench.Taper(fd, 64, variant)
        sim.run()
        out.append((sim.grid.fields(), sim.amplitude_ratio()))
        sim.close()
    (fa, ta), (fb, tb) = out
    assert np.abs(fa).max() > 0
    assert np.abs(fa - fb).max() <= 5e-6 * np.abs(fa).max()
    assert np.abs(ta - tb).max() <= 5e-6 * np.abs(ta).max()
