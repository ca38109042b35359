"""The CPU restatement against golden vectors recorded from the reference itself.

tests/golden/*.npz were written by tests/golden/make_golden.py running the
reference's own compiled C; these checks need no reference on the machine.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from bindings import OracleGrid
from make_golden import c0_drive, c0_setup, wg_geometry, wg_setup

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))


def test_c0_probes_oracle(orc):
    gold = np.load(os.path.join(GOLDEN, "c0_probes.npz"))
    p = c0_setup()
    N = p["n"]
    assert [tuple(x) for x in gold["points"]] == p["probes"]
    g = OracleGrid(orc, N, N, N, p["dx"])
    a, b = p["cube"]
    for c in range(3):
        g.ep[c][a:b, a:b, a:b] = 4.0
    orc.orc_step_threads(os.cpu_count() or 1)
    si, sj, sk = p["src"]
    out = np.zeros_like(gold["probes"])
    for n in range(p["steps"]):
        g.src[2][sk, sj, si] = np.float32(c0_drive(n, p))
        g.step(p["dt"])
        for q, (i, j, k) in enumerate(p["probes"]):
            out[n, q] = [g.f[m][k, j, i] for m in range(3)]
    orc.orc_step_threads(1)
    assert np.abs(out).max() > 1e-6
    assert np.array_equal(out, gold["probes"])


def oracle_wg_forward(orc, fd, p, steps=None):
    """The reference driver's forward loop (3d_fdtd.c:105-126) in the restatement."""
    from bindings import Reference  # noqa: F401  (layout only)
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * 3.141592652 / p["lam"]
    T = steps or p["steps"]
    mode = fd.read_mode_file(os.path.join(GOLDEN, "modes", "small_te0.txt.gz"))
    ml = mode.fields.copy()
    mo = mode.fields.copy()
    mi, mj, md = mode.mi, mode.mj, mode.disc
    g = OracleGrid(orc, nx, ny, nz, dx)
    gold = np.load(os.path.join(GOLDEN, "wg_small.npz"))
    for c in range(3):
        g.ep[c][...] = gold["eps"][..., c]
    b, t = p["core"]
    cx, cy = nx // 2, (b + t) // 2
    cums = [np.zeros(2) for _ in range(3)]
    inst = np.zeros((T, 3, 2))
    acc = np.zeros(nx * nz * 6 * 2)
    for n in range(T):
        amp = math.exp(-((n - 120) ** 2) / (2 * 40.0 ** 2)) if n < 300 else 0.0
        phase = n * dt * omega
        orc.orc_mode_source(g.h, cx, cy, p["src_z"], P(ml.view(np.float64)), mi, mj, md, phase, amp, 0)
        g.step(dt)
        orc.orc_dft_y_slice(g.h, phase, cy, P(acc))
        for q, (z, m, rev) in enumerate(((p["launch_z"], ml, 0), (p["launch_z"], ml, 1), (p["out_z"], mo, 0))):
            o = np.zeros(2)
            orc.orc_mode_overlap(g.h, cx, cy, z, P(m.view(np.float64)), mi, mj, md, phase, rev, P(cums[q]), P(o))
            inst[n, q] = o
    return g, inst, np.array(cums), acc.view(np.complex128).reshape(nz, nx, 6)


def test_wg_forward_oracle(orc, fd):
    p = wg_setup()
    gold = np.load(os.path.join(GOLDEN, "wg_small.npz"))
    g, inst, cums, four = oracle_wg_forward(orc, fd, p)
    b, t = p["core"]
    cy = (b + t) // 2
    f = g.fields()
    # the mode file is read by our own parser here, the reference's fscanf there:
    # both give the nearest double to each printed decimal
    assert np.array_equal(inst, gold["inst"])
    assert np.array_equal(cums, gold["cum"])
    assert np.array_equal(four, gold["fourier"])
    assert np.array_equal(f[p["out_z"]], gold["fwd_z"])
    assert np.array_equal(f[:, cy], gold["fwd_y"])
