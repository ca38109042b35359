"""Known-answer test of the CPML that shares no formula with the CPU
restatement: the field a 12-cell CPML (the bench's: grading order 3, kappa 1,
alpha 0, default sigma_max) reflects back into the domain.

The reference has no CPML (its absorbing boundary is the first-order Mur ABC,
timefield3d.c:2275-2721), so parity with the restatement alone would let a
formula error shared by both pass.  Here a broadband Ez point pulse (derivative
of a Gaussian: no net charge, so no static field stays behind) runs on a 56^3
grid with the CPML and on the same interior enlarged by 64 cells on every side
with PEC walls, far enough that nothing comes back from them within the run.
The difference of the two at probes two cells from the CPML is the reflected
field; it must stay 60 dB below the incident peak there.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, L, PAD, T, DX = 56, 12, 64, 220, 0.025
SIG = 8.0   # pulse width in steps: spectrum peaks near 0.7 um and covers 1.5-1.6 um


def pulse(n):
    t = (n - 5 * SIG) / SIG
    return -t * math.exp(-0.5 * t * t)


def probes():
    c = N // 2
    # normal incidence on the z0 face, two oblique points, and one near a corner
    return [(c, c, L + 2), (c - 10, c, L + 2), (c, c - 12, L + 2), (L + 2, L + 2, L + 2)]


def run(fd, prec, size, off, cpml):
    dt = 0.99 * DX / math.sqrt(3)
    g = fd.Grid(size, size, size, DX, prec)
    fd.lib.timefield3d_set_background(g.t, 1.0, 1.0)
    if cpml:
        fd.call("timefield3d_set_cpml", g.t, L, 3, -1.0, 1.0, 0.0)
    else:
        fd.call("timefield3d_set_boundary", g.t, fd.PEC)
    ids = [[fd.call("timefield3d_add_probe", g.t, i + off, j + off, k + off, m, T) for m in range(3)]
           for (i, j, k) in probes()]
    c = N // 2 + off
    for n in range(T):
        fd.call("timefield3d_set_source_value", g.t, c, c, c, 2, pulse(n))
        fd.call("timefield3d_apply_timestep_omp_full", g.t, dt)
    rec = np.zeros((T, len(ids), 3))
    for q, row in enumerate(ids):
        for m, pid in enumerate(row):
            buf = np.zeros(T)
            fd.call("timefield3d_read_probe", g.t, pid, buf.ctypes.data_as(fd.dp), T)
            rec[:, q, m] = buf
    g.close()
    return rec


@pytest.fixture(scope="module")
def free_space(fd, gpu):
    return run(fd, fd.F64, N + 2 * PAD, PAD, False)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_cpml_reflection_below_minus_60_db(fd, gpu, free_space, prec):
    got = run(fd, fd.F64 if prec == "f64" else fd.F32, N, 0, True)
    for q in range(len(probes())):
        inc = np.abs(free_space[:, q, :]).max()
        refl = np.abs(got[:, q, :] - free_space[:, q, :]).max()
        assert inc > 0
        db = 20 * math.log10(max(refl, 1e-300) / inc)
        assert db <= -60.0, (probes()[q], db)
