"""GPU engine vs the CPU checkers, through the C ABI (reference entry points).

FP64 grids reproduce the reference's arithmetic: stencil and Mur boundary are
compared bit for bit; quantities that pass through a plane reduction (mode
overlaps) differ only by summation order and are held to 1e-10 relative.
FP32 grids are held to the stated FP32 tolerances.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

from bindings import OracleGrid
from make_golden import c0_drive, c0_setup, wg_geometry, wg_setup

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DT_FACTOR = 0.99 / math.sqrt(3)


def lossy_problem(lib, t):
    lib.timefield3d_set_background(t, 1.0, 1.0)
    lib.timefield3d_set_prism_permittivity(t, 4.0, 5, 12, 4, 10, 6, 15)
    lib.timefield3d_set_top_half_plane(t, 2.25, 1.3, 10)
    lib.timefield3d_set_prism_electric_conductivity(t, 0.4, 6, 11, 5, 9, 7, 12)
    lib.timefield3d_set_background_magnetic_conductivity(t, 0.05)


SRC = ((9, 7, 11, 2, 1.0), (8, 6, 10, 4, 0.5), (12, 8, 14, 0, -0.3))


def drive(n):
    return math.exp(-((n - 50) ** 2) / (2 * 15.0 ** 2)) * math.sin(0.9 * n)


def oracle_copy(orc, grid):
    g = OracleGrid(orc, grid.nx, grid.ny, grid.nz, grid.disc)
    for c in range(3):
        g.ep[c][...] = grid.ep[..., c]
        g.mu[c][...] = grid.mu[..., c]
    for m in range(6):
        g.sig[m][...] = grid.sig[..., m]
    return g


def run_pair(fd, orc, precision, boundary, steps=150, dims=(18, 14, 22), cpml=None):
    nx, ny, nz = dims
    dx = 0.02
    dt = DT_FACTOR * dx
    grid = fd.Grid(nx, ny, nz, dx, precision)
    lossy_problem(fd.lib, grid.t)
    g = oracle_copy(orc, grid)
    if boundary == fd.CPML:
        L, order, smax, kmax, amax = cpml
        fd.call("timefield3d_set_cpml", grid.t, L, order, smax, kmax, amax)
        g.set_boundary(orc.CPML)
        g.set_cpml(L, order, smax, kmax, amax, dt)
    for n in range(steps):
        J = drive(n)
        for (i, j, k, m, s) in SRC:
            fd.call("timefield3d_set_source_value", grid.t, i, j, k, m, s * J)
            g.src[m][k, j, i] = np.float32(s * J)
        fd.call("timefield3d_apply_timestep_omp_full", grid.t, dt)
        g.step(dt)
    return grid.fields(), g.fields()


def test_mur_f64_bitexact(fd, orc, gpu):
    a, b = run_pair(fd, orc, fd.F64, fd.MUR)
    assert np.abs(b).max() > 1e-3
    assert np.array_equal(a, b)


def test_mur_f32_close(fd, orc, gpu):
    a, b = run_pair(fd, orc, fd.F32, fd.MUR)
    err = np.abs(a - b).max() / np.abs(b).max()
    assert err < 2e-5, err


@pytest.mark.parametrize("cpml", [(4, 3, -1.0, 1.0, 0.0), (3, 2, 40.0, 3.0, 0.2)])
def test_cpml_f64_matches_oracle(fd, orc, gpu, cpml):
    a, b = run_pair(fd, orc, fd.F64, fd.CPML, cpml=cpml, dims=(20, 16, 24))
    assert np.abs(b).max() > 1e-3
    assert np.array_equal(a, b)


def test_cpml_f32_close(fd, orc, gpu):
    a, b = run_pair(fd, orc, fd.F32, fd.CPML, cpml=(4, 3, -1.0, 1.0, 0.0), dims=(20, 16, 24))
    err = np.abs(a - b).max() / np.abs(b).max()
    assert err < 2e-5, err


def fused_problem(lib, t, dims, lossy):
    nx, ny, nz = dims
    lib.timefield3d_set_background(t, 1.0, 1.0)
    lib.timefield3d_set_prism_permittivity(t, 4.0, nx // 4, 3 * nx // 4, ny // 4, 3 * ny // 4, nz // 4, nz // 2)
    lib.timefield3d_set_top_half_plane(t, 2.25, 1.0, 2 * ny // 3)
    if lossy:
        lib.timefield3d_set_prism_electric_conductivity(t, 0.4, nx // 3, nx // 2, ny // 3, ny // 2, nz // 3, nz // 2)


@pytest.mark.parametrize("variant", ["flat", "flat4", "fused", "stream"])
@pytest.mark.parametrize("dims,boundary,lossy", [
    ((37, 19, 45), "cpml", False),   # width not a multiple of 4: cp.async staging when fused
    ((33, 17, 40), "pec", False),
    ((64, 40, 150), "cpml", True),   # TMA staging when fused, lossy coefficients, several z-chunks
    ((48, 24, 40), "cpml", False),
    ((72, 20, 36), "pec", False),    # partial edge tile
    ((36, 21, 30), "cpml", True),    # nine 4-cell groups per row: rows start inside a warp
])
def test_fused_f32_matches_oracle(fd, orc, gpu, dims, boundary, lossy, variant):
    """FP32 fast path (mu = 1, no magnetic loss), both kernel designs, against the FP64 restatement."""
    nx, ny, nz = dims
    dx = 0.02
    dt = DT_FACTOR * dx
    grid = fd.Grid(nx, ny, nz, dx, fd.F32)
    fd.call("timefield3d_set_yee_variant", grid.t,
            {"flat": fd.YEE_FLAT, "flat4": fd.YEE_FLAT4, "fused": fd.YEE_FUSED, "stream": fd.YEE_STREAM}[variant])
    fused_problem(fd.lib, grid.t, dims, lossy)
    g = oracle_copy(orc, grid)
    if boundary == "cpml":
        fd.call("timefield3d_set_cpml", grid.t, 6, 3, -1.0, 2.0, 0.1)
        g.set_boundary(orc.CPML)
        g.set_cpml(6, 3, -1.0, 2.0, 0.1, dt)
    else:
        fd.call("timefield3d_set_boundary", grid.t, fd.PEC)
        g.set_boundary(orc.PEC)
    src = [(nx // 2, ny // 2, nz // 3, 2, 1.0), (nx // 2 - 3, ny // 2 + 1, nz // 3, 4, 0.5),
           (nx // 3, ny // 3, 2 * nz // 3, 0, -0.7)]
    steps = 160
    launches = []
    for n in range(steps):
        J = drive(n)
        for (i, j, k, m, s) in src:
            fd.lib.timefield3d_set_source_value(grid.t, i, j, k, m, s * J)
            g.src[m][k, j, i] = np.float32(s * J)
        l0 = fd.lib.fdtd_launch_count()
        fd.lib.timefield3d_apply_timestep_omp_full(grid.t, dt)
        launches.append(fd.lib.fdtd_launch_count() - l0)
        g.step(dt)
    fd.check("fused loop")
    # Yee kernels (1 fused or stream; 2 flat or flat4) + the step counter; the
    # stream kernel needs nx % 4 == 0 and otherwise leaves the step to the flat pair
    one_pass = variant == "fused" or (variant == "stream" and nx % 4 == 0)
    assert max(launches[5:]) == (2 if one_pass else 3)
    a, b = grid.fields(), g.fields()
    err = np.abs(a - b).max() / np.abs(b).max()
    assert np.abs(b).max() > 1e-3
    assert err < 5e-5, err


def test_c0_probes_golden(fd, gpu):
    """64^3 dipole, 1000 FP64 steps: probe series equal the reference's."""
    gold = np.load(os.path.join(GOLDEN, "c0_probes.npz"))
    p = c0_setup()
    N = p["n"]
    grid = fd.Grid(N, N, N, p["dx"])
    fd.lib.timefield3d_set_background(grid.t, 1.0, 1.0)
    a, b = p["cube"]
    fd.lib.timefield3d_set_prism_permittivity(grid.t, p["eps"], a, b, a, b, a, b)
    ids = [[fd.call("timefield3d_add_probe", grid.t, i, j, k, m, p["steps"]) for m in range(3)]
           for (i, j, k) in p["probes"]]
    si, sj, sk = p["src"]
    for n in range(p["steps"]):
        fd.lib.timefield3d_set_source_value(grid.t, si, sj, sk, 2, c0_drive(n, p))
        fd.lib.timefield3d_apply_timestep_omp_full(grid.t, p["dt"])
    fd.check("c0 loop")
    out = np.zeros_like(gold["probes"])
    buf = np.zeros(p["steps"])
    for q in range(4):
        for m in range(3):
            fd.call("timefield3d_read_probe", grid.t, ids[q][m], buf.ctypes.data_as(C.POINTER(C.c_double)),
                    p["steps"])
            out[:, q, m] = buf
    assert np.array_equal(out, gold["probes"])


# ---------------------------------------------------------------------------
# the reference driver's sequence on a small taper (golden from the reference)
# ---------------------------------------------------------------------------
def gpu_wg_forward(fd, precision, steps=None):
    p = wg_setup()
    gold = np.load(os.path.join(GOLDEN, "wg_small.npz"))
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    T = steps or p["steps"]
    grid = fd.Grid(nx, ny, nz, dx, precision)
    lib = fd.lib
    wg_geometry(lib, grid.t, p, None, None)
    S = p["seg_num"] + 1
    Lc = (C.c_int * S)(*p["left"])
    Rc = (C.c_int * S)(*p["right"])
    b, t = p["core"]
    z0, z1 = p["taper"]
    taper = fd.call("adjoint3d_taper_new", p["ep_core"], 1.0, p["seg_num"], z0, z1, Lc, Rc, b, t, p["steps"])
    fd.call("adjoint3d_taper_insert", grid.t, taper)
    assert np.array_equal(grid.ep, gold["eps"])
    path = os.path.join(GOLDEN, "modes", "small_te0.txt.gz")
    launch, outm = fd.read_mode_file(path), fd.read_mode_file(path)
    cx, cy = nx // 2, (b + t) // 2
    cums = [fd.Complex() for _ in range(3)]
    inst = np.zeros((T, 3, 2))
    for n in range(T):
        amp = math.exp(-((n - 120) ** 2) / (2 * 40.0 ** 2)) if n < 300 else 0.0
        phase = n * dt * omega
        lib.timefield3d_mode_source(grid.t, cx, cy, p["src_z"], launch.struct, phase, amp, 0)
        lib.timefield3d_apply_timestep_omp_full(grid.t, dt)
        lib.timefield3d_update_fourier_fields_y_slice_omp(grid.t, phase, cy)
        for q, (z, m, rev) in enumerate(((p["launch_z"], launch, 0), (p["launch_z"], launch, 1),
                                         (p["out_z"], outm, 0))):
            o = lib.timefield3d_mode_overlap(grid.t, cx, cy, z, m.struct, phase, rev, C.byref(cums[q]))
            inst[n, q] = (o.re, o.im)
        lib.adjoint3d_taper_store_forward_fields(taper, grid.t, n)
    fd.check("forward loop")
    cum = np.array([[c.re, c.im] for c in cums])
    return dict(p=p, gold=gold, grid=grid, taper=taper, launch=launch, outm=outm, inst=inst, cum=cum,
                dt=dt, omega=omega, cx=cx, cy=cy)


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def test_wg_forward_f64_golden(fd, gpu):
    r = gpu_wg_forward(fd, fd.F64)
    gold, p, grid = r["gold"], r["p"], r["grid"]
    assert rel(r["inst"], gold["inst"]) < 1e-10
    assert rel(r["cum"], gold["cum"]) < 1e-10
    f = grid.fields()
    assert rel(f[p["out_z"]], gold["fwd_z"]) < 1e-10
    assert rel(f[:, r["cy"]], gold["fwd_y"]) < 1e-10
    four = grid.fourier()[:, r["cy"]]
    assert rel(four, gold["fourier"]) < 1e-10
    fd.lib.adjoint3d_taper_free(r["taper"])


def test_wg_forward_f32_transmission(fd, gpu):
    """FP32 fields, FP64 overlaps: launched/transmitted amplitudes within 1e-3 of the reference."""
    r = gpu_wg_forward(fd, fd.F32)
    gold = r["gold"]
    for q in (0, 2):
        c, g = complex(*r["cum"][q]), complex(*gold["cum"][q])
        assert abs(c - g) / abs(g) < 1e-3, (q, c, g)
    t32 = complex(*r["cum"][2]) / complex(*r["cum"][0])
    tg = complex(*gold["cum"][2]) / complex(*gold["cum"][0])
    assert abs(t32 - tg) / abs(tg) < 1e-3
    fd.lib.adjoint3d_taper_free(r["taper"])


def test_wg_adjoint_gradient_golden(fd, orc, gpu):
    r = gpu_wg_forward(fd, fd.F64)
    gold, p, grid, taper, outm = r["gold"], r["p"], r["grid"], r["taper"], r["outm"]
    lib = fd.lib
    # rotate the output mode as the driver does (3d_fdtd.c:144-148), complex_mul per entry
    rot = orc.cexp(float(gold["tphase"]) + fd.REF_PI / 2)
    fr, fi = outm.fields.real.copy(), outm.fields.imag.copy()
    outm.fields.real[...] = rot.real * fr - rot.imag * fi
    outm.fields.imag[...] = rot.real * fi + rot.imag * fr
    lib.timefield3d_zero_fields(grid.t)
    T = p["steps"]
    for n in range(T - 1, -1, -1):
        phase = (n + 1) * r["dt"] * r["omega"]
        lib.timefield3d_mode_source_adjoint(grid.t, r["cx"], r["cy"], p["out_z"], outm.struct, phase, 0)
        lib.timefield3d_apply_timestep_omp_full(grid.t, r["dt"])
        lib.adjoint3d_taper_store_adjoint_fields(taper, grid.t, n)
    fd.check("adjoint loop")
    f = grid.fields()
    assert rel(f[p["out_z"]], gold["adj_z"]) < 1e-10
    assert rel(f[:, r["cy"]], gold["adj_y"]) < 1e-10
    fd.call("adjoint3d_taper_calculate_ep_gradient", taper)
    n = gold["ep_grad"].size
    eg = np.ctypeslib.as_array(taper.ep_gradient, shape=(n,))
    assert rel(eg, gold["ep_grad"]) < 1e-9
    fd.call("adjoint3d_taper_calculate_gradients_from_ep_gradient", taper, p["ep_core"] - p["ep_clad"])
    S = p["seg_num"] + 1
    assert rel(np.ctypeslib.as_array(taper.left_grad, shape=(S,)), gold["left_grad"]) < 1e-9
    assert rel(np.ctypeslib.as_array(taper.right_grad, shape=(S,)), gold["right_grad"]) < 1e-9
    fd.lib.adjoint3d_taper_free(taper)


def test_wg_adjoint_gradient_f32_fields(fd, orc, gpu):
    """The reference's gradient path (adjoint3d.c:339-418) on FP32 fields: the
    ep gradient and the vertex gradients within 1e-2 of the FP64 reference."""
    r = gpu_wg_forward(fd, fd.F32)
    gold, p, grid, taper, outm = r["gold"], r["p"], r["grid"], r["taper"], r["outm"]
    lib = fd.lib
    rot = orc.cexp(float(gold["tphase"]) + fd.REF_PI / 2)
    fr, fi = outm.fields.real.copy(), outm.fields.imag.copy()
    outm.fields.real[...] = rot.real * fr - rot.imag * fi
    outm.fields.imag[...] = rot.real * fi + rot.imag * fr
    lib.timefield3d_zero_fields(grid.t)
    T = p["steps"]
    for n in range(T - 1, -1, -1):
        phase = (n + 1) * r["dt"] * r["omega"]
        lib.timefield3d_mode_source_adjoint(grid.t, r["cx"], r["cy"], p["out_z"], outm.struct, phase, 0)
        lib.timefield3d_apply_timestep_omp_full(grid.t, r["dt"])
        lib.adjoint3d_taper_store_adjoint_fields(taper, grid.t, n)
    fd.check("adjoint loop")
    fd.call("adjoint3d_taper_calculate_ep_gradient", taper)
    n = gold["ep_grad"].size
    assert rel(np.ctypeslib.as_array(taper.ep_gradient, shape=(n,)), gold["ep_grad"]) < 1e-2
    fd.call("adjoint3d_taper_calculate_gradients_from_ep_gradient", taper, p["ep_core"] - p["ep_clad"])
    S = p["seg_num"] + 1
    assert rel(np.ctypeslib.as_array(taper.left_grad, shape=(S,)), gold["left_grad"]) < 1e-2
    assert rel(np.ctypeslib.as_array(taper.right_grad, shape=(S,)), gold["right_grad"]) < 1e-2
    fd.lib.adjoint3d_taper_free(taper)


def test_kernel_timing_run_equals_untimed(fd, gpu):
    """Timed graphs (event pairs around each Yee update), on every replay or on
    one replay in 3, compute the same fields as the untimed run."""
    outs = []
    # 100 steps = 3 graph replays of 32 steps + 4 single steps
    for period, timed_steps in ((0, 0), (1, 96), (3, 32)):
        grid = fd.Grid(24, 20, 28, 0.02, fd.F32)
        lossy_problem(fd.lib, grid.t)
        fd.call("timefield3d_set_cpml", grid.t, 4, 3, -1.0, 1.0, 0.0)
        fd.call("timefield3d_set_source_value", grid.t, 10, 9, 14, 2, 1.0)
        fd.call("timefield3d_set_kernel_timing", grid.t, period)
        l0 = fd.lib.fdtd_launch_count()
        fd.call("timefield3d_run", grid.t, DT_FACTOR * 0.02, 100)
        ms, cnt = C.c_double(), C.c_longlong()
        fd.call("timefield3d_read_kernel_timing", grid.t, C.byref(ms), C.byref(cnt))
        launches = fd.lib.fdtd_launch_count() - l0
        assert launches >= 100 * 2
        assert cnt.value == timed_steps
        assert (ms.value > 0) == (timed_steps > 0)
        outs.append(grid.fields())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    assert fd.lib.timefield3d_set_kernel_timing(grid.t, -1) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()


def test_run_graph_equals_stepwise(fd, gpu):
    """timefield3d_run (scheduled source, graphs, monitors, bound store) equals the per-call path."""
    p = wg_setup()
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    T = 150
    b, t = p["core"]
    cx, cy = nx // 2, (b + t) // 2
    path = os.path.join(GOLDEN, "modes", "small_te0.txt.gz")
    amps = np.array([math.exp(-((n - 60) ** 2) / (2 * 20.0 ** 2)) for n in range(T)])
    phases = np.array([n * dt * omega for n in range(T)])
    outs = []
    for mode_run in (False, True):
        grid = fd.Grid(nx, ny, nz, dx)
        wg_geometry(fd.lib, grid.t, p, None, None)
        m = fd.read_mode_file(path)
        om = np.array([omega * 0.97, omega, omega * 1.03])
        mon = fd.call("timefield3d_add_overlap_monitor", grid.t, cx, cy, p["out_z"], m.copy().struct, 0, 3,
                      om.ctypes.data_as(C.POINTER(C.c_double)))
        if mode_run:
            fd.call("timefield3d_set_source_schedule", grid.t, cx, cy, p["src_z"], m.struct, 0, 0, T,
                    amps.ctypes.data_as(C.POINTER(C.c_double)), phases.ctypes.data_as(C.POINTER(C.c_double)))
            fd.call("timefield3d_run", grid.t, dt, T)
        else:
            for n in range(T):
                fd.lib.timefield3d_mode_source(grid.t, cx, cy, p["src_z"], m.struct, phases[n], amps[n], 0)
                fd.lib.timefield3d_apply_timestep_omp_full(grid.t, dt)
            fd.check("stepwise")
        acc = (fd.Complex * 3)()
        fd.call("timefield3d_read_overlap_monitor", grid.t, mon, acc)
        assert fd.lib.timefield3d_step_count(grid.t) == T
        outs.append((grid.fields(), np.array([[a.re, a.im] for a in acc])))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.abs(outs[0][1]).max() > 0


def test_bounded_wait_times_out_and_context_survives(fd, gpu):
    """A device wait on a barrier nothing arrives on gives up after its limit,
    reports FDTD_ERR_TIMEOUT like a pipeline timeout, and the GPU keeps working."""
    el = C.c_double()
    r = fd.lib.fdtd_wait_selftest(0.05, C.byref(el))
    assert r == fd.FDTD_ERR_TIMEOUT, fd.lib.fdtd_last_error_message()
    assert 0.05 <= el.value < 1.0, el.value
    fd.lib.fdtd_clear_error()
    # the context is still usable: a small FP64 run completes without error
    grid = fd.Grid(12, 12, 12, 0.02)
    fd.call("timefield3d_set_source_value", grid.t, 6, 6, 6, 2, 1.0)
    fd.call("timefield3d_run", grid.t, DT_FACTOR * 0.02, 10)
    fd.call("timefield3d_synchronize", grid.t)
    assert np.abs(grid.fields()).max() > 0
