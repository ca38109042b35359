"""Spline taper: natural-cubic-spline width, sub-pixel fill, device raster.

timefield3d_set_spline_taper has no reference counterpart; it generalises
timefield3d_set_taper (timefield3d.c:1511-1535).  Pins: the spline weights
against scipy's natural CubicSpline; the fill against the numpy restatement in
oracle/geometry.py (bit for bit); integer edges against the reference's own
timefield3d_set_taper (bit for bit); the device raster against the host path
(fields after stepping, bit for bit).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

import geometry

DP = C.POINTER(C.c_double)


def basis(fd, K, z0, z1):
    W = np.zeros((z1 - z0, K))
    fd.call("fdtd_spline_basis", K, z0, z1, W.ctypes.data_as(DP))
    return W


@pytest.mark.parametrize("K,z0,z1", [(2, 5, 30), (5, 0, 41), (20, 30, 370), (7, 3, 9)])
def test_spline_basis_is_natural_cubic_spline(fd, K, z0, z1):
    W = basis(fd, K, z0, z1)
    knots = np.linspace(0.0, z1 - 1 - z0, K)
    want = CubicSpline(knots, np.eye(K), bc_type="natural")(np.arange(z1 - z0, dtype=float))
    assert np.abs(W - want).max() < 1e-12
    assert np.abs(W.sum(axis=1) - 1).max() < 1e-12     # reproduces constants


def taper_problem(fd, g):
    fd.lib.timefield3d_set_background(g.t, 2.085, 1.0)
    fd.lib.timefield3d_set_prism_permittivity(g.t, 4.0, 0, 40, 0, 6, 0, 50)   # non-uniform "old" values
    fd.lib.timefield3d_set_top_half_plane(g.t, 3.0, 1.0, 15)


def test_spline_fill_matches_restatement(fd):
    g = fd.Grid(40, 20, 50, 0.05, fd.F32)
    taper_problem(fd, g)
    rng = np.random.default_rng(3)
    widths = rng.uniform(0.3, 1.5, 6)
    ep0, mu0 = g.ep.copy(), g.mu.copy()
    args = (12.1, 1.0, 6, widths.ctypes.data_as(DP), 20.3, 8, 44, 4, 13)
    fd.call("timefield3d_set_spline_taper", g.t, *args)
    xl, xr = geometry.spline_edges(basis(fd, 6, 8, 44), widths, 20.3, 0.05)
    geometry.raster(ep0, mu0, xl, xr, 12.1, 1.0, 8, 4, 13)
    assert np.array_equal(g.ep, ep0) and np.array_equal(g.mu, mu0)
    frac = (ep0[8:44, 4:13] != np.float32(12.1)) & (ep0[8:44, 4:13] != np.float32(2.085)) \
        & (ep0[8:44, 4:13] != np.float32(4.0)) & (ep0[8:44, 4:13] != np.float32(3.0))
    assert frac.any()                                   # partial cells exist


def test_integer_edges_equal_reference_taper(fd, ref):
    """Constant width 1.0 um at 0.05 um, centre 20: edges at cells 10 and 30,
    the same cells the reference's integer taper fills."""
    nx, ny, nz = 40, 20, 50
    g = fd.Grid(nx, ny, nz, 0.05, fd.F32)
    taper_problem(fd, g)
    widths = np.full(4, 1.0)
    fd.call("timefield3d_set_spline_taper", g.t, 12.1, 1.0, 4, widths.ctypes.data_as(DP), 20.0, 8, 44, 4, 13)
    tf = ref.lib.timefield3d_new(nx, ny, nz, 0.05)
    ref.lib.timefield3d_set_background(tf, 2.085, 1.0)
    ref.lib.timefield3d_set_prism_permittivity(tf, 4.0, 0, 40, 0, 6, 0, 50)
    ref.lib.timefield3d_set_top_half_plane(tf, 3.0, 1.0, 15)
    ref.lib.timefield3d_set_taper(tf, 12.1, 1.0, 10, 30, 10, 30, 8, 44, 4, 13)
    assert np.array_equal(g.ep, ref.eps(tf)) and np.array_equal(g.mu, ref.mus(tf))
    ref.lib.timefield3d_free(tf)


def test_spline_rejects_core_outside_grid(fd):
    g = fd.Grid(20, 10, 20, 0.05, fd.F32)
    widths = np.array([0.5, 2.0])                      # 2 um = 40 cells > 20
    r = fd.lib.timefield3d_set_spline_taper(g.t, 12.1, 1.0, 2, widths.ctypes.data_as(DP), 10.0, 2, 18, 2, 6)
    assert r == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()


@pytest.mark.gpu
def test_spline_device_raster_equals_host_path(fd, gpu):
    """Grid A rasterises after its materials are on the GPU (device path, one
    kernel); grid B before (host arrays, uploaded).  Same fields after 60 steps."""
    dx, dt = 0.05, 0.99 * 0.05 / 3 ** 0.5
    rng = np.random.default_rng(7)
    widths = rng.uniform(0.4, 1.4, 5)
    args = (12.1, 1.0, 5, widths.ctypes.data_as(DP), 19.7, 6, 40, 5, 12)
    out = []
    for device_path in (True, False):
        g = fd.Grid(40, 20, 48, dx, fd.F32)
        taper_problem(fd, g)
        fd.call("timefield3d_set_cpml", g.t, 4, 3, -1.0, 1.0, 0.0)
        if device_path:
            fd.call("timefield3d_upload_materials", g.t)
            l0 = fd.lib.fdtd_launch_count()
        fd.call("timefield3d_set_spline_taper", g.t, *args)
        if device_path:
            assert fd.lib.fdtd_launch_count() - l0 == 1
        fd.call("timefield3d_set_source_value", g.t, 20, 9, 10, 1, 1.0)
        fd.call("timefield3d_run", g.t, dt, 60)
        out.append((g.fields(), g.ep.copy()))
    assert np.array_equal(out[0][1], out[1][1])
    assert np.abs(out[0][0]).max() > 0
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.gpu
def test_spline_adjoint_gradient_matches_finite_differences(fd, gpu):
    """Forward pulse + CW adjoint as the reference driver runs them
    (3d_fdtd.c:97-165): the spline-weighted field-product gradient of
    F = |O_out(omega)| against centred differences (+-5 nm on the three
    interior control widths, sub-pixel geometry).  The reference's formula
    leaves out a global constant (time step, overlap normalisation, omega), so
    one scale is fitted; measured on B200: cosine 0.9998, 2.4 % residual."""
    import math
    import os
    from make_golden import wg_setup
    p = wg_setup()
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    T, K = 400, 5
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    b, t = p["core"]
    cx, cy = nx // 2, (b + t) // 2
    z0, z1 = p["taper"]
    W0 = np.array([0.5, 0.6, 0.55, 0.66, 0.7])
    mode_path = os.path.join(os.path.dirname(__file__), "golden", "modes", "small_te0.txt.gz")
    amps = np.array([math.exp(-((n - 120) ** 2) / (2 * 40.0 ** 2)) if n < 300 else 0.0 for n in range(T)])
    phases = np.array([n * dt * omega for n in range(T)])
    keep = []

    def build(widths):
        g = fd.Grid(nx, ny, nz, dx, fd.F32)
        fd.lib.timefield3d_set_background(g.t, p["ep_clad"], 1.0)
        fd.lib.timefield3d_set_waveguide(g.t, p["ep_core"], 15, 25, 0, z0, b, t)
        fd.lib.timefield3d_set_waveguide(g.t, p["ep_core"], 13, 27, z1, nz, b, t)
        w = np.ascontiguousarray(widths, float)
        fd.call("timefield3d_set_spline_taper", g.t, p["ep_core"], 1.0, K, w.ctypes.data_as(DP), 20.0, z0, z1, b, t)
        fd.call("timefield3d_set_cpml", g.t, 6, 3, -1.0, 1.0, 0.0)
        keep.append(g)
        return g

    def forward(widths, store=None):
        g = build(widths)
        launch, outm = fd.read_mode_file(mode_path), fd.read_mode_file(mode_path)
        keep.extend([launch, outm])
        om = np.array([omega])
        mon = fd.call("timefield3d_add_overlap_monitor", g.t, cx, cy, p["out_z"], outm.struct, 0, 1,
                      om.ctypes.data_as(DP))
        fd.call("timefield3d_set_source_schedule", g.t, cx, cy, p["src_z"], launch.struct, 0, 0, T,
                amps.ctypes.data_as(DP), phases.ctypes.data_as(DP))
        if store:
            fd.call("fdtd_spline_store_bind", store, g.t, 0, 0, 1)
        fd.call("timefield3d_run", g.t, dt, T)
        acc = (fd.Complex * 1)()
        fd.call("timefield3d_read_overlap_monitor", g.t, mon, acc)
        if store:
            fd.call("fdtd_spline_store_unbind", store, g.t)
        return complex(acc[0].re, acc[0].im), outm

    g0 = build(W0)
    store = fd.lib.fdtd_spline_store_new(g0.t, K, W0.ctypes.data_as(DP), 20.0, z0, z1, b, t, T)
    assert store
    O, outm = forward(W0, store)
    tph = math.atan2(O.imag, O.real) % (2 * fd.REF_PI)
    outm.fields *= complex(math.cos(tph + fd.REF_PI / 2), math.sin(tph + fd.REF_PI / 2))
    ga = build(W0)
    aph = np.array([(T - n) * dt * omega for n in range(T)])
    ones = np.ones(T)
    fd.call("timefield3d_set_source_schedule", ga.t, cx, cy, p["out_z"], outm.struct, 0, 1, T,
            ones.ctypes.data_as(DP), aph.ctypes.data_as(DP))
    fd.call("fdtd_spline_store_bind", store, ga.t, 1, T - 1, -1)
    fd.call("timefield3d_run", ga.t, dt, T)
    fd.call("fdtd_spline_store_unbind", store, ga.t)
    grad = np.zeros(K)
    cells = np.zeros(2 * (t - b) * (z1 - z0))
    fd.call("fdtd_spline_store_gradient", store, p["ep_core"] - p["ep_clad"], grad.ctypes.data_as(DP),
            cells.ctypes.data_as(DP))
    # the reduction is the spline-weighted sum of the cell products
    W = basis(fd, K, z0, z1)
    rows = cells.reshape(z1 - z0, t - b, 2).sum(axis=(1, 2))
    assert np.allclose(grad, W.T @ rows * (p["ep_core"] - p["ep_clad"]) / (2 * dx), rtol=1e-12, atol=0)
    delta = 0.005
    fdg = []
    for c in range(1, K - 1):
        Wp, Wm = W0.copy(), W0.copy()
        Wp[c] += delta
        Wm[c] -= delta
        fdg.append((abs(forward(Wp)[0]) - abs(forward(Wm)[0])) / (2 * delta))
    a, f = grad[1:K - 1], np.array(fdg)
    cos = a @ f / np.linalg.norm(a) / np.linalg.norm(f)
    s = a @ f / (a @ a)
    assert cos > 0.999, (a, f)
    assert np.abs(s * a - f).max() / np.abs(f).max() < 0.05, (a, f, s)
    fd.lib.fdtd_spline_store_free(store)
