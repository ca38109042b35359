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
