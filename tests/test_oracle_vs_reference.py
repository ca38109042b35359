"""Pins the CPU restatement (oracle/liboracle.so) to the reference itself.

The reference's own C (oracle/_ref/libref.so, compiled unchanged from its
sources) and our SoA restatement run the same inputs side by side; every
comparison here is bit-exact, since both compute in IEEE double with the same
operation order.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from bindings import Complex, OracleGrid, Reference

DT_FACTOR = 0.99 / math.sqrt(3)


def _copy_materials(tf, g: OracleGrid):
    ep, mu, sg = Reference.eps(tf), Reference.mus(tf), Reference.sig(tf)
    for c in range(3):
        g.ep[c][...] = ep[..., c]
        g.mu[c][...] = mu[..., c]
    for m in range(6):
        g.sig[m][...] = sg[..., m]


def _ref_mode(ref, fd, path):
    """Load a mode file with the reference's own loader (mode.c:949)."""
    import gzip
    import os
    import shutil
    import tempfile
    tmp = tempfile.mkdtemp()
    try:
        txt = os.path.join(tmp, "m.txt")
        with gzip.open(path, "rb") as fi, open(txt, "wb") as fo:
            shutil.copyfileobj(fi, fo)
        return ref.load_mode(txt)
    finally:
        shutil.rmtree(tmp)


def test_mur_step_lossy_bitexact(ref, orc):
    nx, ny, nz, dx = 18, 14, 22, 0.02
    dt = DT_FACTOR * dx
    ref.set_threads(nz // 2)
    tf = ref.timefield3d_new(nx, ny, nz, dx)
    ref.timefield3d_set_background(tf, 1.0, 1.0)
    ref.timefield3d_set_prism_permittivity(tf, 4.0, 5, 12, 4, 10, 6, 15)
    ref.timefield3d_set_top_half_plane(tf, 2.25, 1.3, 10)
    ref.timefield3d_set_prism_electric_conductivity(tf, 0.4, 6, 11, 5, 9, 7, 12)
    ref.timefield3d_set_background_magnetic_conductivity(tf, 0.05)
    g = OracleGrid(orc, nx, ny, nz, dx)
    _copy_materials(tf, g)
    src = Reference.sources(tf)
    for n in range(150):
        J = math.exp(-((n - 50) ** 2) / (2 * 15.0 ** 2)) * math.sin(0.9 * n)
        for (i, j, k, m, s) in ((9, 7, 11, 2, 1.0), (8, 6, 10, 4, 0.5), (12, 8, 14, 0, -0.3)):
            src[k, j, i, m] = np.float32(s * J)
            g.src[m][k, j, i] = np.float32(s * J)
        ref.timefield3d_apply_timestep_omp_full(tf, dt)
        g.step(dt)
    a, b = Reference.fields(tf), g.fields()
    assert np.abs(a).max() > 1e-3
    assert np.array_equal(a, b)
    ref.timefield3d_free(tf)


def test_initial_field_small_grid_bitexact(ref, orc):
    """A field set directly in the host array propagates identically (12^3, 6 threads)."""
    nx, ny, nz, dx = 12, 12, 12, 0.02
    dt = DT_FACTOR * dx
    ref.set_threads(nz // 2)
    tf = ref.timefield3d_new(nx, ny, nz, dx)
    g = OracleGrid(orc, nx, ny, nz, dx)
    _copy_materials(tf, g)
    Reference.fields(tf)[6, 6, 6, 2] = 1.0
    g.f[2][6, 6, 6] = 1.0
    for _ in range(20):
        ref.timefield3d_apply_timestep_omp_full(tf, dt)
        g.step(dt)
    assert np.array_equal(Reference.fields(tf), g.fields())
    ref.timefield3d_free(tf)


def test_cexp_series(ref, orc):
    for x in np.linspace(0.0, 2 * math.pi, 37):
        r = ref.complex_exp(Complex(0.0, float(x)))
        assert orc.cexp(float(x)) == complex(r.re, r.im)
    for ph in (0.0, 1.0, 6.283185304, 6.3, 100.123, 2467.5):
        red = orc.orc_reduce_phase(ph)
        assert red == ph - int(ph / (2 * 3.141592652)) * 2 * 3.141592652


@pytest.fixture(scope="module")
def wg(ref, fd):
    import os
    from make_golden import wg_geometry, wg_setup
    p = wg_setup()
    path = os.path.join(os.path.dirname(__file__), "golden", "modes", "small_te0.txt.gz")
    return p, wg_geometry, path


def test_mode_source_overlap_dft_bitexact(ref, orc, fd, wg):
    p, wg_geometry, path = wg
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = DT_FACTOR * dx
    omega = 2 * 3.141592652 / p["lam"]
    ref.set_threads(8)
    tf = ref.timefield3d_new(nx, ny, nz, dx)
    wg_geometry(ref.lib, tf, p, None, None)
    g = OracleGrid(orc, nx, ny, nz, dx)
    _copy_materials(tf, g)
    rm = _ref_mode(ref, fd, path)
    om = np.ascontiguousarray(Reference.mode_array(rm)).copy()     # (mj, mi, 6) complex
    rm2 = _ref_mode(ref, fd, path)
    om2 = om.copy()
    mi, mj, md = rm.i, rm.j, rm.disc
    b, t = p["core"]
    cx, cy = nx // 2, (b + t) // 2
    cum_r = [Complex(), Complex()]
    cum_o = [np.zeros(2), np.zeros(2)]
    acc = np.zeros(nx * nz * 6 * 2)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    for n in range(60):
        amp = math.exp(-((n - 25) ** 2) / (2 * 10.0 ** 2))
        phase = n * dt * omega
        ref.timefield3d_mode_source(tf, cx, cy, p["src_z"], rm, phase, amp, 0)
        orc.orc_mode_source(g.h, cx, cy, p["src_z"], P(om.view(np.float64)), mi, mj, md, phase, amp, 0)
        if n == 0:
            assert np.array_equal(Reference.sources(tf)[p["src_z"]], np.stack([s[p["src_z"]] for s in g.src], -1))
        ref.timefield3d_apply_timestep_omp_full(tf, dt)
        g.step(dt)
        ref.timefield3d_update_fourier_fields_y_slice_omp(tf, phase, cy)
        orc.orc_dft_y_slice(g.h, phase, cy, P(acc))
        for q, rev in enumerate((0, 1)):
            o = ref.timefield3d_mode_overlap(tf, cx, cy, p["launch_z"], rm2, phase, rev, C.byref(cum_r[q]))
            inst = np.zeros(2)
            orc.orc_mode_overlap(g.h, cx, cy, p["launch_z"], P(om2.view(np.float64)), mi, mj, md, phase, rev,
                                 P(cum_o[q]), P(inst))
            assert (o.re, o.im) == (inst[0], inst[1])
    assert np.array_equal(Reference.fields(tf), g.fields())
    for q in range(2):
        assert (cum_r[q].re, cum_r[q].im) == tuple(cum_o[q])
    n6 = nx * ny * nz * 6
    ff = np.ctypeslib.as_array(C.cast(tf.fourier_fields, C.POINTER(C.c_double)), shape=(2 * n6,))
    ref_slice = ff.view(np.complex128).reshape(nz, ny, nx, 6)[:, cy]
    ours = acc.view(np.complex128).reshape(nz, nx, 6)
    assert np.array_equal(ref_slice, ours)
    # the mode was normalised in place identically
    assert np.array_equal(Reference.mode_array(rm), om)
    # adjoint source
    ref.timefield3d_mode_source_adjoint(tf, cx, cy, p["out_z"], rm, 1.234, 0)
    orc.orc_mode_source_adjoint(g.h, cx, cy, p["out_z"], P(om.view(np.float64)), mi, mj, md, 1.234, 0)
    assert np.array_equal(Reference.sources(tf)[p["out_z"]], np.stack([s[p["out_z"]] for s in g.src], -1))
    ref.timefield3d_free(tf)


def test_taper_store_and_gradients_bitexact(ref, orc):
    nx, ny, nz, dx = 30, 12, 40, 0.05
    T, seg = 25, 3
    left = [10, 9, 8, 9]
    right = [20, 21, 23, 22]
    Lc = (C.c_int * 4)(*left)
    Rc = (C.c_int * 4)(*right)
    tp = ref.adjoint3d_taper_new(12.1, 1.0, seg, 8, 29, Lc, Rc, 4, 8, T)
    tf = ref.timefield3d_new(nx, ny, nz, dx)
    g = OracleGrid(orc, nx, ny, nz, dx)
    rng = np.random.default_rng(3)
    fl = Reference.fields(tf)
    H, L = 4, 21
    fwd = np.zeros(T * L * H * 2 * 3)
    adj = np.zeros_like(fwd)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    li, ri = (C.c_int * 4)(*left), (C.c_int * 4)(*right)
    for t in range(T):
        vals = rng.standard_normal(fl.shape)
        fl[...] = vals
        for m in range(6):
            g.f[m][...] = vals[..., m]
        ref.adjoint3d_taper_store_forward_fields(tp, tf, t)
        orc.orc_taper_store(g.h, seg, 8, 29, 4, 8, li, ri, t, P(fwd))
        vals = rng.standard_normal(fl.shape)
        fl[...] = vals
        for m in range(6):
            g.f[m][...] = vals[..., m]
        ref.adjoint3d_taper_store_adjoint_fields(tp, tf, t)
        orc.orc_taper_store(g.h, seg, 8, 29, 4, 8, li, ri, t, P(adj))
    ref.adjoint3d_taper_calculate_ep_gradient(tp)
    eg = np.zeros(2 * H * L)
    orc.orc_taper_ep_gradient(H, L, T, P(fwd), P(adj), P(eg))
    assert np.array_equal(np.ctypeslib.as_array(tp.ep_gradient, shape=(2 * H * L,)), eg)
    ref.adjoint3d_taper_calculate_gradients_from_ep_gradient(tp, 10.0)
    lg, rg = np.zeros(seg + 1), np.zeros(seg + 1)
    orc.orc_taper_vertex_gradient(seg, H, L, P(eg), 10.0, P(lg), P(rg))
    assert np.array_equal(np.ctypeslib.as_array(tp.left_grad, shape=(seg + 1,)), lg)
    assert np.array_equal(np.ctypeslib.as_array(tp.right_grad, shape=(seg + 1,)), rg)
    ref.timefield3d_free(tf)
