"""Wavefront runs (FDTD_YEE_WAVE, csrc/yee_wave.cu).

CPU: the work-item table every launch follows -- each item's dependencies
finish (all their tickets) before the item's first ticket, with the counts the
kernel waits for; that ordering, with every block taking its tickets in
order and all blocks resident, is what guarantees progress.
GPU: a wavefront run gives fields and monitors bit-identical to the same run
on the per-step flat4 kernels (the per-cell code is shared), with CPML, PEC,
lossy material, a scheduled mode source, monitors, a run length that is not a
whole number of launches, and several launch / sweep lengths.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

from make_golden import wg_setup

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


def schedule(fd, nx, ny, nz, L, steps, sweep, group, job_z, nparts):
    jz = (C.c_int * max(1, len(job_z)))(*job_z)
    tickets = C.c_int()
    n = fd.lib.fdtd_wave_schedule(nx, ny, nz, L, steps, sweep, group, jz, len(job_z), nparts, None, 0,
                                  C.byref(tickets))
    assert n > 0
    out = np.zeros((n, 9), np.int32)
    assert fd.lib.fdtd_wave_schedule(nx, ny, nz, L, steps, sweep, group, jz, len(job_z), nparts,
                                     out.ctypes.data_as(IP), n, C.byref(tickets)) == n
    return out, tickets.value


@pytest.mark.parametrize("nx,ny,nz,L,steps,sweep,group,job_z,nparts", [
    (200, 160, 400, 12, 32, 8, 1, [25, 380], 30),   # the Si taper grid with its two monitors
    (200, 160, 400, 12, 32, 32, 4, [25, 380], 30),
    (40, 28, 72, 6, 32, 8, 1, [58], 4),
    (40, 28, 72, 6, 13, 3, 3, [16, 58, 58], 4),     # two monitors on one plane
    (24, 20, 28, 4, 32, 8, 2, [], 1),               # nz < 4 x sweep: sweeps do not overlap
    (32, 16, 10, 0, 7, 2, 5, [3], 2),               # no CPML
])
def test_schedule_orders_dependencies_first(fd, nx, ny, nz, L, steps, sweep, group, job_z, nparts):
    items, tickets = schedule(fd, nx, ny, nz, L, steps, sweep, group, job_z, nparts)
    t0 = items[:, 0]
    assert t0[0] == 0 and np.all(np.diff(t0) > 0)
    count = np.diff(np.append(t0, tickets))
    assert np.array_equal(count, (items[:, 2] + group - 1) // group)   # tickets of `group` blocks
    kind, k, ls = items[:, 1] & 3, (items[:, 1] >> 2) & 0x7FFF, items[:, 1] >> 17
    # every (step, field, plane) once, monitors once per (step, plane with monitors)
    mon_planes = sorted(set(job_z))
    assert np.sum(kind == 0) == np.sum(kind == 1) == steps * (nz - 2)
    assert np.sum(kind == 2) == steps * len(mon_planes)
    # the counter each item signals, as the kernel computes it
    ctr = np.where(kind == 2, 2 * steps * nz + ls * nz + k, (ls * 2 + kind) * nz + k)
    assert len(set(ctr.tolist())) == len(items)
    by_ctr = {int(c): i for i, c in enumerate(ctr)}
    parts = {z: nparts * job_z.count(z) for z in mon_planes}
    for i in range(len(items)):
        if kind[i] == 2:
            assert items[i, 2] == parts[int(k[i])]
        deps = [(items[i, 3 + 2 * d], items[i, 4 + 2 * d]) for d in range(3) if items[i, 3 + 2 * d] >= 0]
        want = []
        if kind[i] == 0 and ls[i] > 0:
            want = [(1, k[i], ls[i] - 1)] + ([(1, k[i] - 1, ls[i] - 1)] if k[i] > 1 else []) + \
                   ([(2, k[i], ls[i] - 1)] if int(k[i]) in parts else [])
        elif kind[i] == 1:
            want = [(0, k[i], ls[i])] + ([(0, k[i] + 1, ls[i])] if k[i] + 1 <= nz - 2 else [])
        elif kind[i] == 2:
            want = [(1, k[i], ls[i])]
        assert len(deps) == len(want), (i, deps, want)
        for (c, need), (wk, wkk, wls) in zip(deps, want):
            p = by_ctr[int(c)]
            assert (kind[p], k[p], ls[p]) == (wk, wkk, wls)
            assert need == count[p]                       # waits for every ticket of the producer
            assert t0[p] + count[p] <= t0[i]              # ... all of which come earlier


def test_schedule_rejects_bad_input(fd):
    t = C.c_int()
    jz = (C.c_int * 1)(0)   # plane 0 is not an updated plane
    assert fd.lib.fdtd_wave_schedule(40, 28, 72, 6, 8, 2, 1, jz, 1, 4, None, 0, C.byref(t)) == -1
    assert fd.lib.fdtd_wave_schedule(42, 28, 72, 6, 8, 2, 1, None, 0, 4, None, 0, C.byref(t)) == -1   # nx % 4
    assert fd.lib.fdtd_wave_schedule(40, 28, 72, 6, 0, 2, 1, None, 0, 4, None, 0, C.byref(t)) == -1   # no steps
    assert fd.lib.fdtd_wave_schedule(40, 28, 72, 6, 8, 2, 0, None, 0, 4, None, 0, C.byref(t)) == -1   # group 0


# ---------------------------------------------------------------------------
# GPU: wave == flat4, bit for bit
# ---------------------------------------------------------------------------
def taper_run(fd, variant, T, lossy=False, boundary="cpml", wave_steps=None, timing=0):
    p = wg_setup()
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    b, t = p["core"]
    g = fd.Grid(nx, ny, nz, dx, fd.F32)
    fd.lib.timefield3d_set_background(g.t, p["ep_clad"], 1.0)
    fd.lib.timefield3d_set_waveguide(g.t, p["ep_core"], 15, 25, 0, nz, b, t)
    if lossy:
        fd.lib.timefield3d_set_prism_electric_conductivity(g.t, 0.3, 10, 30, 8, 20, 30, 50)
    if boundary == "cpml":
        fd.call("timefield3d_set_cpml", g.t, 6, 3, -1.0, 1.0, 0.0)
    else:
        fd.call("timefield3d_set_boundary", g.t, fd.PEC)
    fd.call("timefield3d_set_yee_variant", g.t, variant)
    if wave_steps:
        fd.call("timefield3d_set_wave_steps", g.t, *wave_steps)
    path = os.path.join(os.path.dirname(__file__), "golden", "modes", "small_te0.txt.gz")
    m = fd.read_mode_file(path)
    om = np.array([omega * 0.98, omega, omega * 1.02])
    mons = [fd.call("timefield3d_add_overlap_monitor", g.t, nx // 2, (b + t) // 2, z, m.copy().struct, 0, 3,
                    om.ctypes.data_as(DP)) for z in (p["launch_z"], p["out_z"], p["out_z"])]
    amps = np.array([math.exp(-((n - 90) ** 2) / (2 * 30.0 ** 2)) for n in range(T)])
    phases = np.array([n * dt * omega for n in range(T)])
    fd.call("timefield3d_set_source_schedule", g.t, nx // 2, (b + t) // 2, p["src_z"], m.copy().struct, 0, 0, T,
            amps.ctypes.data_as(DP), phases.ctypes.data_as(DP))
    fd.call("timefield3d_set_kernel_timing", g.t, timing)
    fd.call("timefield3d_run", g.t, dt, T)
    ms, cnt = C.c_double(), C.c_longlong()
    fd.call("timefield3d_read_kernel_timing", g.t, C.byref(ms), C.byref(cnt))
    accs = []
    for mon in mons:
        acc = (fd.Complex * 3)()
        fd.call("timefield3d_read_overlap_monitor", g.t, mon, acc)
        accs.append([[a.re, a.im] for a in acc])
    assert fd.lib.timefield3d_step_count(g.t) == T
    out = (g.fields(), np.array(accs), cnt.value, ms.value)
    g.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("lossy,boundary", [(False, "cpml"), (True, "cpml"), (False, "pec")])
def test_wave_equals_flat4(fd, gpu, lossy, boundary):
    T = 200   # 3 launches of 64 steps + 8 per-step steps
    ref = taper_run(fd, fd.YEE_FLAT4, T, lossy, boundary)
    got = taper_run(fd, fd.YEE_WAVE, T, lossy, boundary)
    assert np.abs(ref[1]).max() > 0 and np.abs(ref[0]).max() > 0
    assert np.array_equal(ref[0], got[0])
    assert np.array_equal(ref[1], got[1])


@pytest.mark.gpu
@pytest.mark.parametrize("wave_steps", [(1, 1, 1), (16, 16, 3), (48, 5, 2), (96, 8, 8)])
def test_wave_launch_and_sweep_lengths(fd, gpu, wave_steps):
    T = 150
    ref = taper_run(fd, fd.YEE_FLAT4, T)
    got = taper_run(fd, fd.YEE_WAVE, T, wave_steps=wave_steps)
    assert np.array_equal(ref[0], got[0])
    assert np.array_equal(ref[1], got[1])


@pytest.mark.gpu
def test_wave_kernel_timing_counts_steps(fd, gpu):
    T = 100   # 3 launches of 32 steps, the first and the third timed with period 2
    _, _, cnt, ms = taper_run(fd, fd.YEE_WAVE, T, wave_steps=(32, 8, 1), timing=2)
    assert cnt == 64 and ms > 0
    _, _, cnt, ms = taper_run(fd, fd.YEE_WAVE, T, wave_steps=(32, 8, 1), timing=1)
    assert cnt == 96 and ms > 0


def test_wave_steps_argument_checks(fd):
    g = fd.Grid(24, 20, 28, 0.02, fd.F32)
    assert fd.lib.timefield3d_set_wave_steps(g.t, 0, 1, 1) == fd.FDTD_ERR_ARG
    assert fd.lib.timefield3d_set_wave_steps(g.t, 8, 9, 1) == fd.FDTD_ERR_ARG
    assert fd.lib.timefield3d_set_wave_steps(g.t, 5000, 8, 1) == fd.FDTD_ERR_ARG
    assert fd.lib.timefield3d_set_wave_steps(g.t, 64, 8, 0) == fd.FDTD_ERR_ARG
    assert fd.lib.timefield3d_set_wave_steps(g.t, 64, 8, 65) == fd.FDTD_ERR_ARG
    assert fd.lib.timefield3d_set_wave_steps(g.t, 64, 8, 2) == fd.FDTD_OK
    fd.lib.fdtd_clear_error()
