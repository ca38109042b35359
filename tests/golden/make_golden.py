"""Generates the golden vectors in tests/golden/ by running the reference itself.

    python tests/golden/make_golden.py

Needs oracle/_ref/libref.so (the reference's C sources compiled unchanged by
`make -C oracle ref`); run it where those sources exist.  The outputs are small
.npz files that the tests read on any machine, including ones without the
reference.  Mode profiles in tests/golden/modes/ come from oracle/_ref/modegen
(see make_modes.sh).

Fixtures
  c0_probes.npz   64^3 dipole run (the plain-FDTD workload, Mur boundary since the
                  reference has no CPML): Ex/Ey/Ez at 4 seeded interior points,
                  every step for 1000 steps, FP64.
  wg_small.npz    small Si waveguide taper with the reference's own driver
                  sequence (3d_fdtd.c:105-187) shrunk: mode source, three mode
                  overlaps, y-slice DFT, taper edge store, adjoint run, ep
                  gradient, vertex gradients and the asymmetric edge update.
"""
from __future__ import annotations

import ctypes as C
import gzip
import math
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from bindings import Complex, Reference  # noqa: E402

REF_PI = 3.141592652


def splitmix64(seed: int):
    s = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        s = (s + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        yield z ^ (z >> 31)


def c0_setup():
    """Parameters of the 64^3 dipole workload (shared with the tests)."""
    n, dx = 64, 0.020
    dt = 0.99 * dx / math.sqrt(3)
    lam0, bw = 1.55, 0.3
    w0 = 2 * math.pi / lam0
    dw = 2 * math.pi * bw / lam0 ** 2
    sigma_n = (2 * math.sqrt(2 * math.log(2)) / dw) / dt
    n0 = 3 * sigma_n
    g = splitmix64(0)
    pts = [tuple(9 + next(g) % 46 for _ in range(3)) for _ in range(4)]
    return dict(n=n, dx=dx, dt=dt, w0=w0, sigma_n=sigma_n, n0=n0, steps=1000, cube=(22, 42), eps=4.0,
                src=(32, 32, 32), probes=pts)


def c0_drive(n: int, p: dict) -> float:
    return math.exp(-((n - p["n0"]) ** 2) / (2 * p["sigma_n"] ** 2)) * math.sin(p["w0"] * n * p["dt"])


def make_c0(R: Reference) -> None:
    p = c0_setup()
    N = p["n"]
    tf = R.timefield3d_new(N, N, N, p["dx"])
    R.timefield3d_set_background(tf, 1.0, 1.0)
    a, b = p["cube"]
    R.timefield3d_set_prism_permittivity(tf, p["eps"], a, b, a, b, a, b)
    src = Reference.sources(tf)
    fl = Reference.fields(tf)
    si, sj, sk = p["src"]
    out = np.zeros((p["steps"], 4, 3))
    for n in range(p["steps"]):
        src[sk, sj, si, 2] = np.float32(c0_drive(n, p))
        R.timefield3d_apply_timestep_omp_full(tf, p["dt"])
        for q, (i, j, k) in enumerate(p["probes"]):
            out[n, q] = fl[k, j, i, 0:3]
    R.timefield3d_free(tf)
    np.savez_compressed(os.path.join(HERE, "c0_probes.npz"), probes=out, points=np.array(p["probes"]),
                        dt=p["dt"], dx=p["dx"])
    print("c0_probes.npz", np.abs(out).max())


def wg_setup():
    """Small taper problem on the 0.05 um grid of modes/small_te0.txt.gz."""
    return dict(nx=40, ny=28, nz=72, dx=0.05, steps=400, lam=1.55, core=(11, 16), src_z=12, launch_z=16,
                out_z=58, taper=(24, 48), seg_num=4, left=[15, 14, 12, 12, 13], right=[25, 26, 27, 28, 27],
                wg_in=(15, 25), wg_out=(13, 27), ep_core=12.1, ep_clad=2.085)


def wg_geometry(lib, tf, p, left, right):
    lib.timefield3d_set_background(tf, p["ep_clad"], 1.0)
    b, t = p["core"]
    z0, z1 = p["taper"]
    lib.timefield3d_set_waveguide(tf, p["ep_core"], p["wg_in"][0], p["wg_in"][1], 0, z0, b, t)
    lib.timefield3d_set_waveguide(tf, p["ep_core"], p["wg_out"][0], p["wg_out"][1], z1, p["nz"], b, t)


def make_wg(R: Reference) -> None:
    p = wg_setup()
    modefile = os.path.join(HERE, "modes", "small_te0.txt.gz")
    tmp = tempfile.mkdtemp()
    try:
        txt = os.path.join(tmp, "m.txt")
        with gzip.open(modefile, "rb") as fi, open(txt, "wb") as fo:
            shutil.copyfileobj(fi, fo)
        launch = R.load_mode(txt)
        out_mode = R.load_mode(txt)
    finally:
        shutil.rmtree(tmp)
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * REF_PI / p["lam"]
    T = p["steps"]
    tf = R.timefield3d_new(nx, ny, nz, dx)
    wg_geometry(R.lib, tf, p, None, None)
    L = (C.c_int * (p["seg_num"] + 1))(*p["left"])
    Rr = (C.c_int * (p["seg_num"] + 1))(*p["right"])
    b, t = p["core"]
    z0, z1 = p["taper"]
    taper = R.adjoint3d_taper_new(p["ep_core"], 1.0, p["seg_num"], z0, z1, L, Rr, b, t, T)
    R.adjoint3d_taper_insert(tf, taper)
    ep0 = Reference.eps(tf).copy()
    cx, cy = nx // 2, (b + t) // 2
    launched, reflected, transmitted = Complex(), Complex(), Complex()
    inst = np.zeros((T, 3, 2))
    fl = Reference.fields(tf)
    for n in range(T):
        amp = math.exp(-((n - 120) ** 2) / (2 * 40.0 ** 2)) if n < 300 else 0.0
        phase = n * dt * omega
        R.timefield3d_mode_source(tf, cx, cy, p["src_z"], launch, phase, amp, 0)
        R.timefield3d_apply_timestep_omp_full(tf, dt)
        R.timefield3d_update_fourier_fields_y_slice_omp(tf, phase, cy)
        for q, (z, mode, rev, acc) in enumerate(((p["launch_z"], launch, 0, launched),
                                                 (p["launch_z"], launch, 1, reflected),
                                                 (p["out_z"], out_mode, 0, transmitted))):
            o = R.timefield3d_mode_overlap(tf, cx, cy, z, mode, phase, rev, C.byref(acc))
            inst[n, q] = (o.re, o.im)
        R.adjoint3d_taper_store_forward_fields(taper, tf, n)
    fwd_z, fwd_y = fl[p["out_z"]].copy(), fl[:, cy].copy()
    n6 = nx * ny * nz * 6
    ff = np.ctypeslib.as_array(C.cast(tf.fourier_fields, C.POINTER(C.c_double)), shape=(2 * n6,))
    fourier = ff.view(np.complex128).reshape(nz, ny, nx, 6)[:, cy, :, :].copy()
    cum = np.array([[launched.re, launched.im], [reflected.re, reflected.im], [transmitted.re, transmitted.im]])
    # adjoint run (3d_fdtd.c:144-165)
    tphase = math.atan2(transmitted.im, transmitted.re)
    if tphase < 0:
        tphase += 2 * REF_PI
    rot = R.complex_exp(Complex(0.0, tphase + REF_PI / 2))
    R.mode_smul(rot, out_mode)
    R.timefield3d_zero_fields(tf)
    for n in range(T - 1, -1, -1):
        phase = (n + 1) * dt * omega
        R.timefield3d_mode_source_adjoint(tf, cx, cy, p["out_z"], out_mode, phase, 0)
        R.timefield3d_apply_timestep_omp_full(tf, dt)
        R.adjoint3d_taper_store_adjoint_fields(taper, tf, n)
    adj_z, adj_y = fl[p["out_z"]].copy(), fl[:, cy].copy()
    R.adjoint3d_taper_calculate_ep_gradient(taper)
    H, Lz = t - b, z1 - z0
    ep_grad = np.ctypeslib.as_array(taper.ep_gradient, shape=(2 * H * Lz,)).copy()
    ep_diff = p["ep_core"] - p["ep_clad"]
    R.adjoint3d_taper_calculate_gradients_from_ep_gradient(taper, ep_diff)
    S = p["seg_num"] + 1
    lg = np.ctypeslib.as_array(taper.left_grad, shape=(S,)).copy()
    rg = np.ctypeslib.as_array(taper.right_grad, shape=(S,)).copy()
    goal = 0.2 * (math.hypot(launched.re, launched.im) - math.hypot(transmitted.re, transmitted.im))
    flag = R.adjoint3d_taper_update_asymmetric(taper, goal, dx, 4)
    new_left = np.ctypeslib.as_array(taper.left, shape=(S,)).copy()
    new_right = np.ctypeslib.as_array(taper.right, shape=(S,)).copy()
    np.savez_compressed(os.path.join(HERE, "wg_small.npz"), eps=ep0, inst=inst, cum=cum, fourier=fourier,
                        fwd_z=fwd_z, fwd_y=fwd_y, adj_z=adj_z, adj_y=adj_y, ep_grad=ep_grad, left_grad=lg,
                        right_grad=rg, goal=goal, flag=flag, new_left=new_left, new_right=new_right,
                        tphase=tphase, dt=dt)
    print("wg_small.npz", cum, ep_grad[:4], lg, rg, new_left, new_right, flag)


if __name__ == "__main__":
    R = Reference()
    R.set_threads(8)   # every z-slab keeps >= 2 planes on these grids
    make_c0(R)
    make_wg(R)
