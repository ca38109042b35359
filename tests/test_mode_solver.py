"""GPU FP64 mode solver against the reference's Arnoldi beta^2 solver.

fdtd_mode_apply_beta_squared must equal mode_apply_beta_squared_operator
(mode.c:2796-2943) bit for bit; fdtd_mode_solve_beta_squared must find the
same mode as mode_solve_beta_squared (mode.c:3461-3616): n_eff within the
solver tolerance and the H-normalised fields equal up to a global phase.
Both solvers stop when |n_eff| changes by less than tol between restarts, so
their answers agree to about that tolerance, not to rounding.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from bindings import Complex as RComplex

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
OMEGA = 2 * 3.141592652 / 1.55   # the reference driver's omega (3d_fdtd.c:12,37)


def ref_strip(R, mi, mj, disc, core, pml=None, ep_clad=2.085, ep_core=12.1):
    """A strip cross-section built with the reference's own mode API."""
    m = R.lib.mode_new(mi, mj, disc)
    R.lib.mode_set_background(m, RComplex(ep_clad, 0), RComplex(1, 0))
    left, right, bottom, top = core
    R.lib.mode_make_rectangle(m, RComplex(ep_core, 0), RComplex(1, 0), left, right, bottom, top)
    if pml is not None:
        R.lib.mode_set_pml(m, *pml)
    return m


def ours(fd, m):
    """The same struct (same arrays) as the engine's ctypes type."""
    return fd.Mode.from_buffer_copy(m)


def betas():
    out = {}
    with open(os.path.join(GOLDEN, "modes", "betas.txt")) as fh:
        for line in fh:
            name, val = line.split()
            out[name] = complex(val.replace("i", "j"))
    return out


def aligned_error(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - c b| / max |a| with the complex c that best maps b onto a."""
    c = np.vdot(b.ravel(), a.ravel()) / np.vdot(b.ravel(), b.ravel())
    return float(np.abs(a - c * b).max() / np.abs(a).max())


@pytest.mark.gpu
def test_beta2_operator_bitexact(fd, ref, gpu):
    R = ref
    mi, mj, disc = 20, 14, 0.05
    m = ref_strip(R, mi, mj, disc, (6, 14, 5, 9), pml=(0.8, 2, 3))
    a = R.mode_array(m)
    rng = np.random.default_rng(11)
    for comp in (3, 4):
        a[..., comp] = rng.standard_normal((mj, mi)) + 1j * rng.standard_normal((mj, mi))
    want_m = R.lib.mode_apply_beta_squared_operator(m, OMEGA)
    got_m = R.lib.mode_new(mi, mj, disc)
    fd.call("fdtd_mode_apply_beta_squared", ours(fd, m), OMEGA, ours(fd, got_m))
    want, got = R.mode_array(want_m).copy(), R.mode_array(got_m).copy()
    assert np.abs(want[..., 3:5]).max() > 0
    assert np.array_equal(got, want)
    for x in (m, want_m, got_m):
        R.lib.mode_free(x)


@pytest.mark.gpu
def test_mode_solver_matches_reference_solver(fd, ref, gpu):
    """500 x 250 nm Si strip in SiO2, 0.05 um grid: both solvers, same inputs."""
    R = ref
    cfg = (24, 16, 0.05, (7, 17, 6, 11))
    m_ref = ref_strip(R, *cfg)
    b_ref = R.lib.mode_solve_beta_squared(C.byref(m_ref), OMEGA, 1e-5, None, 0, 20, 2, 0)
    m_gpu = ref_strip(R, *cfg)
    s = ours(fd, m_gpu)
    b = fd.lib.fdtd_mode_solve_beta_squared(C.byref(s), OMEGA, 1e-5, None, 0, 20, 2, 0)
    fd.check("mode solve")
    assert fd.lib.fdtd_mode_solve_restarts() > 0
    n_ref, n = b_ref.re / OMEGA, b.re / OMEGA
    assert abs(n - n_ref) < 2e-5, (n, n_ref)
    assert abs(b.im) < 1e-9 and abs(b_ref.im) < 1e-9
    A, B = R.mode_array(m_ref).copy(), R.mode_array(m_gpu).copy()
    for comp in range(6):
        err = aligned_error(A[..., comp], B[..., comp]) if np.abs(A[..., comp]).max() > 0 else 0.0
        assert err < 5e-3, (comp, err)
    assert aligned_error(A, B) < 5e-3
    R.lib.mode_free(m_ref)
    R.lib.mode_free(m_gpu)


@pytest.mark.gpu
def test_mode_solver_matches_golden_taper_input(fd, gpu):
    """64 x 48 window of the taper's 500 x 225 nm input end (0.025 um grid):
    beta and fields against the reference solver's recorded output."""
    g = fd.read_mode_file(os.path.join(GOLDEN, "modes", "c1_in_te0.txt.gz"))
    m = fd.HostMode(np.zeros_like(g.fields), g.disc, g.ep, g.mu)
    b = fd.lib.fdtd_mode_solve_beta_squared(C.byref(m.struct), OMEGA, 1e-5, None, 0, 20, 2, 0)
    fd.check("mode solve")
    b_gold = betas()["c1_in_te0"]
    assert abs(b.re / OMEGA - b_gold.real / OMEGA) < 2e-5, (b.re, b_gold)
    # the file holds 6 decimals; compare the dominant components
    for comp in (0, 1, 3, 4):
        assert aligned_error(g.fields[..., comp], m.fields[..., comp]) < 5e-3, comp


def eigen_residual(fd, g, fields, beta) -> float:
    """|B h - beta^2 h| / |beta^2 h| over interior (Hx, Hy), B the GPU operator."""
    m = fd.HostMode(fields.copy(), g.disc, g.ep, g.mu)
    out = fd.HostMode(np.zeros_like(fields), g.disc, g.ep, g.mu)
    fd.call("fdtd_mode_apply_beta_squared", m.struct, OMEGA, out.struct)
    lam = beta * beta
    h, bh = fields[1:-1, 1:-1, 3:5], out.fields[1:-1, 1:-1, 3:5]
    return float(np.linalg.norm(bh - lam * h) / np.linalg.norm(lam * h))


@pytest.mark.gpu
def test_mode_solver_converges_wide_output_end(fd, gpu):
    """3 um x 225 nm output end (160 x 48, near-degenerate lateral modes).  The
    reference's recorded mode stopped on its |n_eff| criterion with an
    eigen-residual of ~1e-2; at a tight tolerance the GPU solver reaches an
    eigenvector (residual < 1e-5) with n_eff within 1e-4 of the reference's."""
    g = fd.read_mode_file(os.path.join(GOLDEN, "modes", "c1_out_te0.txt.gz"))
    b_gold = betas()["c1_out_te0"]
    assert eigen_residual(fd, g, g.fields, b_gold) > 1e-3
    m = fd.HostMode(np.zeros_like(g.fields), g.disc, g.ep, g.mu)
    b = fd.lib.fdtd_mode_solve_beta_squared(C.byref(m.struct), OMEGA, 1e-10, None, 0, 20, 2, 0)
    fd.check("mode solve")
    beta = complex(b.re, b.im)
    assert eigen_residual(fd, g, m.fields, beta) < 1e-5
    assert abs(beta.real - b_gold.real) / OMEGA < 1e-4


def test_mode_solver_rejects_bad_arguments(fd):
    """Argument checks run before any device work (no GPU needed)."""
    z = fd.HostMode(np.zeros((4, 4, 6), complex), 0.05)
    b = fd.lib.fdtd_mode_solve_beta_squared(C.byref(z.struct), -1.0, 1e-5, None, 0, 20, 2, 0)
    assert (b.re, b.im) == (0.0, 0.0)
    assert fd.lib.fdtd_last_error() in (fd.FDTD_ERR_ARG, fd.FDTD_ERR_NO_DEVICE)
    fd.lib.fdtd_clear_error()
