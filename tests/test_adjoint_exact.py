"""Exact discrete-adjoint gradient of a spline taper against finite differences.

Objective: F = |O_out(omega)|, the output monitor's overlap with its mode
(accumulated as timefield3d.c:3176-3239 does it, every step).  The gradient
dF/d(control width) comes from one forward run (edge fields stored) and one
adjoint run scheduled by timefield3d_set_exact_adjoint_schedule, reduced by
fdtd_spline_store_gradient_exact.  It is the derivative of the simulated
objective itself -- no constant is fitted or left out: central differences
with a step small enough not to carry an edge across a cell boundary (+-0.5 nm)
agree with it to rounding.  The sub-pixel fill is piecewise linear in the
width, so a +-5 nm step can move an edge across a cell boundary, and its
central difference then measures the secant across that kink; the same
adjoint fields applied to the step's actual permittivity change
(fdtd_spline_store_gradient_step, which uses the edge cells' neighbours) give
that secant, and must agree with the +-5 nm central difference to 1e-2
relative on every checked control width.  This replaces the reference driver's CW adjoint
(3d_fdtd.c:143-187), whose field-product formula (adjoint3d.c:339-418) leaves
out the step size, the overlap normalisation and a one-step time alignment.

Workloads: the small Si taper of the golden fixtures (40x28x72, dx 50 nm, 6-cell
CPML, 400 steps, 5 control widths), FP64 and FP32; and the 200x160x400 Si taper
(dx 25 nm, 12-cell CPML, 6000 steps) with 20 control widths drawn uniform in
0.5-3.0 um (seed 1) and sorted, differences on control points 3, 10 and 17,
FP32 fields with FP64 monitors.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
DP = C.POINTER(C.c_double)
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class TaperCase:
    """One spline-taper geometry: builds grids, runs forward / adjoint / FD."""

    def __init__(self, fd, prec, nx, ny, nz, dx, T, core, z0, z1, cx, wg_in, wg_out, src_z, out_z, L, lam,
                 mode_in, mode_out, ep_core=12.1, ep_clad=2.085, amp=None):
        self.fd, self.prec = fd, prec
        self.nx, self.ny, self.nz, self.dx, self.T = nx, ny, nz, dx, T
        self.core, self.z0, self.z1, self.cx = core, z0, z1, cx
        self.wg_in, self.wg_out, self.src_z, self.out_z, self.L = wg_in, wg_out, src_z, out_z, L
        self.ep_core, self.ep_clad = ep_core, ep_clad
        self.dt = 0.99 * dx / math.sqrt(3)
        self.omega = 2 * fd.REF_PI / lam
        self.mode_in, self.mode_out = mode_in, mode_out
        self.amps = amp
        self.phases = np.array([n * self.dt * self.omega for n in range(T)])
        self.keep = []

    def grid(self, widths):
        fd = self.fd
        b, t = self.core
        g = fd.Grid(self.nx, self.ny, self.nz, self.dx, self.prec)
        fd.lib.timefield3d_set_background(g.t, self.ep_clad, 1.0)
        fd.lib.timefield3d_set_waveguide(g.t, self.ep_core, self.wg_in[0], self.wg_in[1], 0, self.z0, b, t)
        fd.lib.timefield3d_set_waveguide(g.t, self.ep_core, self.wg_out[0], self.wg_out[1], self.z1, self.nz, b, t)
        w = np.ascontiguousarray(widths, float)
        fd.call("timefield3d_set_spline_taper", g.t, self.ep_core, 1.0, len(w), w.ctypes.data_as(DP), self.cx,
                self.z0, self.z1, b, t)
        fd.call("timefield3d_set_cpml", g.t, self.L, 3, -1.0, 1.0, 0.0)
        return g

    def forward(self, widths, store=None):
        """O_out(omega) of a forward run (and the edge store, when given)."""
        fd = self.fd
        b, t = self.core
        cy = (b + t) // 2
        g = self.grid(widths)
        om = np.array([self.omega])
        mon = fd.call("timefield3d_add_overlap_monitor", g.t, int(self.cx), cy, self.out_z, self.mode_out.struct, 0, 1,
                      om.ctypes.data_as(DP))
        fd.call("timefield3d_set_source_schedule", g.t, int(self.cx), cy, self.src_z, self.mode_in.struct, 0, 0, self.T,
                self.amps.ctypes.data_as(DP), self.phases.ctypes.data_as(DP))
        if store:
            fd.call("fdtd_spline_store_bind", store, g.t, 0, 0, 1)
        fd.call("timefield3d_run", g.t, self.dt, self.T)
        acc = (fd.Complex * 1)()
        fd.call("timefield3d_read_overlap_monitor", g.t, mon, acc)
        if store:
            fd.call("fdtd_spline_store_unbind", store, g.t)
        g.close()
        return complex(acc[0].re, acc[0].im)

    def gradient(self, widths, step=None):
        """(F, dF/dw) by the exact adjoint, and the step form for +-step when given."""
        fd = self.fd
        b, t = self.core
        cy = (b + t) // 2
        g0 = self.grid(widths)
        w = np.ascontiguousarray(widths, float)
        store = fd.lib.fdtd_spline_store_new(g0.t, len(w), w.ctypes.data_as(DP), self.cx, self.z0, self.z1, b, t,
                                             self.T)
        assert store
        self.keep.append(g0)
        O = self.forward(widths, store)
        weight = np.conj(O) / abs(O)                 # F = |O|: dF = Re(conj(O)/|O| dO)
        ga = self.grid(widths)
        fd.call("timefield3d_set_exact_adjoint_schedule", ga.t, int(self.cx), cy, self.out_z, self.mode_out.struct, 0,
                self.T, self.omega, self.dt, float(weight.real), float(weight.imag))
        fd.call("fdtd_spline_store_bind", store, ga.t, 1, self.T, -1)
        fd.call("timefield3d_run", ga.t, self.dt, self.T + 1)
        fd.call("fdtd_spline_store_unbind", store, ga.t)
        grad = np.zeros(len(w))
        fd.call("fdtd_spline_store_gradient_exact", store, self.ep_core - self.ep_clad, grad.ctypes.data_as(DP),
                None)
        sgrad = None
        if step:
            sgrad = np.zeros(len(w))
            fd.call("fdtd_spline_store_gradient_step", store, self.ep_core - self.ep_clad, step,
                    sgrad.ctypes.data_as(DP))
        fd.lib.fdtd_spline_store_free(store)
        ga.close()
        return abs(O), grad, sgrad

    def fd_gradient(self, widths, c, delta):
        wp, wm = np.array(widths, float), np.array(widths, float)
        wp[c] += delta
        wm[c] -= delta
        return (abs(self.forward(wp)) - abs(self.forward(wm))) / (2 * delta)


def small_case(fd, prec):
    from make_golden import wg_setup
    p = wg_setup()
    T = p["steps"]
    amps = np.array([math.exp(-((n - 120) ** 2) / (2 * 40.0 ** 2)) if n < 300 else 0.0 for n in range(T)])
    path = os.path.join(GOLDEN, "modes", "small_te0.txt.gz")
    return TaperCase(fd, prec, p["nx"], p["ny"], p["nz"], p["dx"], T, p["core"], p["taper"][0], p["taper"][1], 20.0,
                     p["wg_in"], p["wg_out"], p["src_z"], p["out_z"], 6, p["lam"], fd.read_mode_file(path),
                     fd.read_mode_file(path), p["ep_core"], p["ep_clad"], amps)


def test_exact_adjoint_is_the_derivative_small_taper_f64(fd, gpu):
    case = small_case(fd, fd.F64)
    W0 = np.array([0.5, 0.6, 0.55, 0.66, 0.7])
    F, g, _ = case.gradient(W0)
    assert F > 0
    for c in (1, 2, 3):
        fdg = case.fd_gradient(W0, c, 0.0005)
        assert abs(g[c] - fdg) <= 1e-3 * abs(fdg), (c, g[c], fdg)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_exact_adjoint_step_matches_5nm_differences_small_taper(fd, gpu, prec):
    case = small_case(fd, fd.F64 if prec == "f64" else fd.F32)
    W0 = np.array([0.5, 0.6, 0.55, 0.66, 0.7])
    F, g, gs = case.gradient(W0, step=0.005)
    assert F > 0
    for c in (1, 2, 3):
        fdg = case.fd_gradient(W0, c, 0.005)
        assert abs(gs[c] - fdg) <= 1e-2 * abs(fdg), (c, gs[c], g[c], fdg)


def test_exact_adjoint_step_matches_5nm_differences_si_taper_20_widths(fd, gpu):
    import bench
    Wk = bench.W
    rng = np.random.default_rng(1)
    widths = np.sort(rng.uniform(0.5, 3.0, 20))
    amp, phase = bench.source_tables(Wk["time_steps"], 0.99 * Wk["dx"] / math.sqrt(3))
    modes = os.path.join(GOLDEN, "modes")
    case = TaperCase(fd, fd.F32, Wk["nx"], Wk["ny"], Wk["nz"], Wk["dx"], Wk["time_steps"],
                     (Wk["core_y"][0], Wk["core_y"][1]), Wk["taper_z"][0], Wk["taper_z"][1], float(Wk["cx"]),
                     Wk["w_in"], Wk["w_out"], Wk["src_z"], Wk["out_z"], Wk["cpml"], Wk["lam0"],
                     fd.read_mode_file(os.path.join(modes, "c1_in_te0.txt.gz")),
                     fd.read_mode_file(os.path.join(modes, "c1_out_te0.txt.gz")), Wk["ep_core"], Wk["ep_clad"], amp)
    F, g, gs = case.gradient(widths, step=0.005)
    assert F > 0
    bad = []
    for c in (3, 10, 17):
        fdg = case.fd_gradient(widths, c, 0.005)
        if not abs(gs[c] - fdg) <= 1e-2 * abs(fdg):
            bad.append((c, gs[c], g[c], fdg))
    assert not bad, bad
