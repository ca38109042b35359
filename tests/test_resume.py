"""Checkpoint / resume, host-side allocation-failure injection and run-to-run
determinism of the FP32 CPML path (scheduled mode source, overlap monitors)."""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

from make_golden import wg_setup

DP = C.POINTER(C.c_double)


def setup(fd, T):
    p = wg_setup()
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    b, t = p["core"]
    g = fd.Grid(nx, ny, nz, dx, fd.F32)
    fd.lib.timefield3d_set_background(g.t, p["ep_clad"], 1.0)
    fd.lib.timefield3d_set_waveguide(g.t, p["ep_core"], 15, 25, 0, nz, b, t)
    fd.call("timefield3d_set_cpml", g.t, 6, 3, -1.0, 1.0, 0.0)
    path = os.path.join(os.path.dirname(__file__), "golden", "modes", "small_te0.txt.gz")
    m = fd.read_mode_file(path)
    om = np.array([omega * 0.98, omega, omega * 1.02])
    mon = fd.call("timefield3d_add_overlap_monitor", g.t, nx // 2, (b + t) // 2, p["out_z"], m.copy().struct, 0, 3,
                  om.ctypes.data_as(DP))
    amps = np.array([math.exp(-((n - 120) ** 2) / (2 * 40.0 ** 2)) for n in range(T)])
    phases = np.array([n * dt * omega for n in range(T)])
    fd.call("timefield3d_set_source_schedule", g.t, nx // 2, (b + t) // 2, p["src_z"], m.copy().struct, 0, 0, T,
            amps.ctypes.data_as(DP), phases.ctypes.data_as(DP))
    return g, mon, dt


def monitor(fd, g, mon):
    acc = (fd.Complex * 3)()
    fd.call("timefield3d_read_overlap_monitor", g.t, mon, acc)
    return np.array([[a.re, a.im] for a in acc])


@pytest.mark.gpu
def test_resume_equals_uninterrupted_run(fd, gpu, tmp_path):
    T = 160
    ck = str(tmp_path / "run.ckpt").encode()
    a, mon_a, dt = setup(fd, T)
    fd.call("timefield3d_run", a.t, dt, 96)
    fd.call("timefield3d_checkpoint_save", a.t, ck)
    fd.call("timefield3d_run", a.t, dt, T - 96)
    b, mon_b, _ = setup(fd, T)
    fd.call("timefield3d_checkpoint_load", b.t, ck)
    assert fd.lib.timefield3d_step_count(b.t) == 96
    fd.call("timefield3d_run", b.t, dt, T - 96)
    assert np.abs(monitor(fd, a, mon_a)).max() > 0
    assert np.array_equal(monitor(fd, a, mon_a), monitor(fd, b, mon_b))
    assert np.array_equal(a.fields(), b.fields())


@pytest.mark.gpu
def test_checkpoint_rejects_another_grid(fd, gpu, tmp_path):
    ck = str(tmp_path / "x.ckpt").encode()
    a, _, dt = setup(fd, 40)
    fd.call("timefield3d_run", a.t, dt, 32)
    fd.call("timefield3d_checkpoint_save", a.t, ck)
    other = fd.Grid(24, 20, 30, 0.05, fd.F32)
    assert fd.lib.timefield3d_checkpoint_load(other.t, ck) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()
    with open(tmp_path / "junk.ckpt", "wb") as fh:
        fh.write(b"not a checkpoint")
    assert fd.lib.timefield3d_checkpoint_load(a.t, str(tmp_path / "junk.ckpt").encode()) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()


@pytest.mark.gpu
def test_injected_allocation_failure_is_reported_and_recoverable(fd, gpu):
    g = fd.Grid(20, 16, 24, 0.05, fd.F32)
    fd.lib.fdtd_inject_allocation_failures(1)
    r = fd.lib.timefield3d_upload_materials(g.t)
    assert r == fd.FDTD_ERR_ALLOC, fd.lib.fdtd_last_error_message()
    fd.lib.fdtd_inject_allocation_failures(0)
    fd.lib.fdtd_clear_error()
    h = fd.Grid(20, 16, 24, 0.05, fd.F32)
    fd.call("timefield3d_set_source_value", h.t, 10, 8, 12, 2, 1.0)
    fd.call("timefield3d_run", h.t, 0.99 * 0.05 / math.sqrt(3), 40)
    assert np.abs(h.fields()).max() > 0


@pytest.mark.gpu
def test_runs_are_deterministic(fd, gpu):
    out = []
    for _ in range(2):
        g, mon, dt = setup(fd, 160)
        fd.call("timefield3d_run", g.t, dt, 160)
        out.append((g.fields(), monitor(fd, g, mon)))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.gpu
def test_truncated_checkpoint_leaves_grid_unchanged(fd, gpu, tmp_path):
    # a file cut inside the field data: the load is refused and nothing of the
    # grid (fields, monitors, step count) changes
    T = 120
    ck = tmp_path / "full.ckpt"
    a, mon_a, dt = setup(fd, T)
    fd.call("timefield3d_run", a.t, dt, 64)
    fd.call("timefield3d_checkpoint_save", a.t, str(ck).encode())
    raw = ck.read_bytes()
    field_bytes = 6 * a.nx * a.ny * a.nz * 4
    cut = tmp_path / "cut.ckpt"
    cut.write_bytes(raw[: len(raw) - field_bytes // 2 - 12 * 4096])
    b, mon_b, _ = setup(fd, T)
    fd.call("timefield3d_run", b.t, dt, 24)
    before = (b.fields(), monitor(fd, b, mon_b), fd.lib.timefield3d_step_count(b.t))
    assert fd.lib.timefield3d_checkpoint_load(b.t, str(cut).encode()) == fd.FDTD_ERR_ARG
    assert b"truncated" in fd.lib.fdtd_last_error_message()
    fd.lib.fdtd_clear_error()
    after = (b.fields(), monitor(fd, b, mon_b), fd.lib.timefield3d_step_count(b.t))
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
    assert before[2] == after[2] == 24


@pytest.mark.gpu
def test_load_into_grid_that_already_ran(fd, gpu, tmp_path):
    # the target grid has run other steps first (its CPML auxiliaries, source
    # plane and monitors hold other values); after the load it continues
    # exactly like the saved run
    T = 160
    ck = str(tmp_path / "run.ckpt").encode()
    a, mon_a, dt = setup(fd, T)
    fd.call("timefield3d_run", a.t, dt, 80)
    fd.call("timefield3d_checkpoint_save", a.t, ck)
    fd.call("timefield3d_run", a.t, dt, T - 80)
    b, mon_b, _ = setup(fd, T)
    fd.call("timefield3d_run", b.t, dt, 131)
    fd.call("timefield3d_checkpoint_load", b.t, ck)
    assert fd.lib.timefield3d_step_count(b.t) == 80
    fd.call("timefield3d_run", b.t, dt, T - 80)
    assert np.array_equal(monitor(fd, a, mon_a), monitor(fd, b, mon_b))
    assert np.array_equal(a.fields(), b.fields())


@pytest.mark.gpu
def test_load_without_cpml_state_zeroes_auxiliaries(fd, gpu, tmp_path):
    # a checkpoint of a grid that had not stepped yet holds no CPML auxiliaries;
    # loading it into a grid that ran must leave that grid's auxiliaries zero,
    # so the run equals one from a fresh grid
    T = 100
    ck = str(tmp_path / "fresh.ckpt").encode()
    a, mon_a, dt = setup(fd, T)
    fd.call("timefield3d_checkpoint_save", a.t, ck)
    fd.call("timefield3d_run", a.t, dt, T)
    b, mon_b, _ = setup(fd, T)
    fd.call("timefield3d_run", b.t, dt, 77)
    fd.call("timefield3d_checkpoint_load", b.t, ck)
    assert fd.lib.timefield3d_step_count(b.t) == 0
    fd.call("timefield3d_run", b.t, dt, T)
    assert np.array_equal(monitor(fd, a, mon_a), monitor(fd, b, mon_b))
    assert np.array_equal(a.fields(), b.fields())
