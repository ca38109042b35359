"""The C ABI without a GPU: exports, host-side reference logic, error conventions.

Host-side parts of the reference surface (rasterisers, taper vertex gradients
and edge updates, the permittivity slice writer, mode files) are compared with
the reference's own compiled C where it is available.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fdtd_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b((?:timefield3d|adjoint3d|fdtd)_[A-Za-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(fd):
    names = declared_functions()
    assert len(names) >= 90
    missing = [n for n in names if not hasattr(fd.lib, n)]
    assert not missing, missing
    # and the Python mirror binds every one of them
    assert set(names) <= set(fd.SIGNATURES), set(names) - set(fd.SIGNATURES)


def test_rasterisers_match_reference(fd, ref):
    dims = (30, 24, 40, 0.02)
    g = fd.Grid(*dims)
    tf = ref.timefield3d_new(*dims)
    for lib, t in ((fd.lib, g.t), (ref.lib, tf)):
        lib.timefield3d_set_background(t, 2.085, 1.0)
        lib.timefield3d_set_top_half_plane(t, 1.93 ** 2, 1.0, 15)
        lib.timefield3d_set_taper(t, 12.1, 1.0, 10, 18, 6, 22, 3, 30, 8, 14)
        lib.timefield3d_set_taper(t, 12.1, 1.0, 12, 16, 15, 14, 30, 36, 8, 14)
        lib.timefield3d_set_waveguide(t, 12.1, 12, 16, 30, 40, 8, 14)
        lib.timefield3d_set_prism_permittivity(t, 7.0, -3, 4, 2, 50, 0, 5)
        lib.timefield3d_set_prism_electric_conductivity(t, 0.5, 2, 5, 3, 7, 1, 9)
        lib.timefield3d_set_background_magnetic_conductivity(t, 0.125)
    from bindings import Reference
    assert np.array_equal(g.ep, Reference.eps(tf))
    assert np.array_equal(g.mu, Reference.mus(tf))
    assert np.array_equal(g.sig, Reference.sig(tf))
    ref.timefield3d_free(tf)


def test_taper_insert_and_slice_writer_match_reference(fd, ref):
    from bindings import Reference
    dims = (40, 20, 60, 0.02)
    left, right = [12, 10, 9, 11, 12], [28, 29, 31, 30, 28]
    out = []
    ours = fd.Grid(*dims)       # owns the host arrays for the whole test
    for lib, t in ((fd.lib, ours.t), (ref.lib, ref.timefield3d_new(*dims))):
        lib.timefield3d_set_background(t, 2.085, 1.0)
        tp = lib.adjoint3d_taper_new(12.1, 1.0, 4, 10, 50, (C.c_int * 5)(*left), (C.c_int * 5)(*right), 8, 12, 5)
        lib.adjoint3d_taper_insert(t, tp)
        path = tempfile.mktemp(suffix=".bin")
        lib.timefield3d_file_write_permittivity_y_slice(t, path.encode(), 5, 35, 10, 50, 10, 2.085, 12.1)
        out.append((np.ctypeslib.as_array(t.ep, shape=(3 * 40 * 20 * 60,)).copy(), open(path, "rb").read()))
        os.unlink(path)
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
@pytest.mark.parametrize("kind", ["asymmetric", "symmetric"])
def test_taper_updates_match_reference(fd, ref, seed, kind, capfd):
    rng = np.random.default_rng(seed)
    seg, H, L = 6, 5, 36
    left = [20 - int(x) for x in rng.integers(0, 4, seg + 1)]
    right = [30 + int(x) for x in rng.integers(0, 4, seg + 1)]
    eg = rng.standard_normal(2 * H * L) * 10 ** rng.uniform(-3, 1)
    res = []
    for lib in (fd.lib, ref.lib):
        tp = lib.adjoint3d_taper_new(12.1, 1.0, seg, 4, 4 + L, (C.c_int * (seg + 1))(*left),
                                     (C.c_int * (seg + 1))(*right), 2, 2 + H, 3)
        np.ctypeslib.as_array(tp.ep_gradient, shape=(2 * H * L,))[:] = eg
        lib.adjoint3d_taper_calculate_gradients_from_ep_gradient(tp, 10.015)
        lg = np.ctypeslib.as_array(tp.left_grad, shape=(seg + 1,)).copy()
        rg = np.ctypeslib.as_array(tp.right_grad, shape=(seg + 1,)).copy()
        goal = float(rng.uniform(0.01, 2.0)) if lib is fd.lib else goal_saved
        goal_saved = goal
        fn = lib.adjoint3d_taper_update_asymmetric if kind == "asymmetric" else lib.adjoint3d_taper_update_symmetric
        flag = fn(tp, goal, 0.025, 4)
        res.append((lg, rg, flag, np.ctypeslib.as_array(tp.left, shape=(seg + 1,)).copy(),
                    np.ctypeslib.as_array(tp.right, shape=(seg + 1,)).copy()))
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a, b)
    out = capfd.readouterr().out
    assert out.count("zeroed out index") % 2 == 0   # both implementations print the same lines


def test_wg_golden_host_update(fd):
    """Vertex gradients and the asymmetric update on the reference's recorded ep-gradient."""
    from make_golden import wg_setup
    gold = np.load(os.path.join(ROOT, "tests", "golden", "wg_small.npz"))
    p = wg_setup()
    S = p["seg_num"] + 1
    b, t = p["core"]
    z0, z1 = p["taper"]
    tp = fd.lib.adjoint3d_taper_new(p["ep_core"], 1.0, p["seg_num"], z0, z1, (C.c_int * S)(*p["left"]),
                                    (C.c_int * S)(*p["right"]), b, t, p["steps"])
    np.ctypeslib.as_array(tp.ep_gradient, shape=(gold["ep_grad"].size,))[:] = gold["ep_grad"]
    fd.lib.adjoint3d_taper_calculate_gradients_from_ep_gradient(tp, p["ep_core"] - p["ep_clad"])
    assert np.array_equal(np.ctypeslib.as_array(tp.left_grad, shape=(S,)), gold["left_grad"])
    assert np.array_equal(np.ctypeslib.as_array(tp.right_grad, shape=(S,)), gold["right_grad"])
    flag = fd.lib.adjoint3d_taper_update_asymmetric(tp, float(gold["goal"]), p["dx"], 4)
    assert flag == int(gold["flag"])
    assert np.array_equal(np.ctypeslib.as_array(tp.left, shape=(S,)), gold["new_left"])
    assert np.array_equal(np.ctypeslib.as_array(tp.right, shape=(S,)), gold["new_right"])
    fd.lib.adjoint3d_taper_free(tp)


def test_mode_file_parser_matches_reference_loader(fd, ref):
    import gzip
    import shutil
    from bindings import Reference
    src = os.path.join(ROOT, "tests", "golden", "modes", "small_te0.txt.gz")
    tmp = tempfile.mkdtemp()
    txt = os.path.join(tmp, "m.txt")
    with gzip.open(src, "rb") as fi, open(txt, "wb") as fo:
        shutil.copyfileobj(fi, fo)
    rm = ref.load_mode(txt)
    ours = fd.read_mode_file(src)
    assert (ours.mi, ours.mj, ours.disc) == (rm.i, rm.j, rm.disc)
    assert np.array_equal(ours.fields, Reference.mode_array(rm))
    shutil.rmtree(tmp)


def test_errors_are_recorded_not_fatal(fd):
    t = fd.lib.timefield3d_new(0, 4, 4, 0.1)
    assert fd.lib.fdtd_last_error() == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()
    g = fd.Grid(8, 8, 8, 0.1)
    assert fd.lib.timefield3d_set_cpml(g.t, 10, 3, -1.0, 1.0, 0.0) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()
    assert fd.lib.timefield3d_set_precision(g.t, 7) == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()
    fd.lib.timefield3d_TE_gaussian_source(g.t, 1, 1, 1, 0.5, 4.0, 0.0, 1.0)
    assert fd.lib.fdtd_last_error() == fd.FDTD_ERR_UNSUPPORTED
    fd.lib.fdtd_clear_error()
    # a struct the library never created
    bogus = fd.Timefield3d()
    fd.lib.timefield3d_apply_timestep_omp_full(bogus, 0.01)
    assert fd.lib.fdtd_last_error() == fd.FDTD_ERR_ARG
    fd.lib.fdtd_clear_error()


def test_device_calls_fail_loudly_without_gpu(fd, capfd):
    if fd.lib.fdtd_device_count() > 0:
        pytest.skip("a GPU is present")
    fd.lib.fdtd_clear_error()
    g = fd.Grid(8, 8, 8, 0.1)
    fd.lib.timefield3d_apply_timestep_omp_full(g.t, 0.01)
    assert fd.lib.fdtd_last_error() == fd.FDTD_ERR_NO_DEVICE
    assert "no CPU fallback" in capfd.readouterr().err
    fd.lib.fdtd_clear_error()
    with pytest.raises(fd.FdtdError):
        fd.call("timefield3d_run", g.t, 0.01, 10)
