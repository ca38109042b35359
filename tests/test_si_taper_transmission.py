"""FP32 transmission of the Si taper workload against the same workload in FP64.

The workload is the bench's: 200x160x400 cells, dx 25 nm, 12-cell CPML, TE0
mode source with the 1.55 um Gaussian pulse, 6000 steps, mode-overlap monitors
at the launch and output planes for 11 wavelengths over 1.50-1.60 um.  The
quantity is the reference driver's complex ratio t = O_out / O_in
(3d_fdtd.c:139-142, overlaps accumulated as in timefield3d.c:3176-3239).  The
engine's FP64 path is bit-exact to the CPU restatement on CPML grids
(test_gpu_parity.py), so it stands in for the FP64 oracle at this size, which
the CPU restatement would need hours for.  Bound: |t32 - t64| / |t64| <= 1e-3
at every wavelength.
"""
from __future__ import annotations

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


def test_si_taper_transmission_f32_within_1e3_of_f64(fd, gpu):
    t = {}
    for prec in (fd.F32, fd.F64):
        sim = bench.Taper(fd, bench.W["time_steps"], 0, prec)
        sim.run()
        t[prec] = sim.amplitude_ratio()
        sim.close()
    t32, t64 = t[fd.F32], t[fd.F64]
    assert np.all(np.abs(t64) > 0.9), np.abs(t64)   # the taper transmits: |t| near 1, T ~ 0.96
    rel = np.abs(t32 - t64) / np.abs(t64)
    assert rel.max() <= 1e-3, rel
