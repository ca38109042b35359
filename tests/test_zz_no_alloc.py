"""fdtd_mode_overlap_plane_noalloc: the mode overlap for callers that cannot
allocate device memory (stream-capture regions, fixed memory budgets, loops
that cannot take cudaMalloc's synchronisation).  Its scratch is a fixed
file-scope device array, so it must agree with the regular entry point
(timefield3d_mode_overlap, which reduces into library-allocated scratch) on
consecutive calls, with the array holding the previous call's contents.

Collected last on purpose (tests/test_zz_*): it loads torch's CUDA runtime next
to the library's, and it must pass both alone and after the other tests.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import pytest

from make_golden import wg_geometry, wg_setup

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_overlap_matches_regular_entry_point(fd, gpu, prec):
    import torch
    precision = fd.F64 if prec == "f64" else fd.F32
    np_dtype = np.float64 if prec == "f64" else np.float32
    p = wg_setup()
    nx, ny, nz, dx = p["nx"], p["ny"], p["nz"], p["dx"]
    dt = 0.99 * dx / math.sqrt(3)
    omega = 2 * fd.REF_PI / p["lam"]
    grid = fd.Grid(nx, ny, nz, dx, precision)
    wg_geometry(fd.lib, grid.t, p, None, None)
    mode = fd.read_mode_file(os.path.join(GOLDEN, "modes", "small_te0.txt.gz"))
    b, t = p["core"]
    cx, cy = nx // 2, (b + t) // 2
    for n in range(120):
        amp = math.exp(-((n - 50) ** 2) / (2 * 20.0 ** 2))
        fd.lib.timefield3d_mode_source(grid.t, cx, cy, p["src_z"], mode.struct, n * dt * omega, amp, 0)
        fd.lib.timefield3d_apply_timestep_omp_full(grid.t, dt)
    fd.check("run")
    f = grid.fields()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    result = torch.zeros(2, dtype=torch.float64, device=dev)
    # two calls in a row (different planes / directions): the second reuses the
    # fixed scratch the first one filled
    for z, rev in ((p["launch_z"], 0), (p["out_z"], 1)):
        acc = fd.Complex()
        ref = fd.lib.timefield3d_mode_overlap(grid.t, cx, cy, z, mode.struct, 0.0, rev, C.byref(acc))
        fd.check("timefield3d_mode_overlap")
        # the FP32 grid's host mirror holds its float values exactly
        planes = [torch.from_numpy(np.ascontiguousarray(f[z, :, :, m].astype(np_dtype))).to(dev)
                  for m in (0, 1, 3, 4)]
        md = torch.from_numpy(mode.fields.copy()).to(dev)      # normalised in place by the call above
        rc = fd.lib.fdtd_mode_overlap_plane_noalloc(
            planes[0].data_ptr(), planes[1].data_ptr(), planes[2].data_ptr(), planes[3].data_ptr(), precision,
            nx, ny, cx, cy, md.data_ptr(), mode.mi, mode.mj, dx / mode.disc, rev, dx, result.data_ptr(),
            stream.cuda_stream)
        assert rc == fd.FDTD_OK, fd.lib.fdtd_last_error_message()
        torch.cuda.synchronize(dev)
        got = complex(*result.cpu().numpy())
        want = complex(ref.re, ref.im)
        assert abs(want) > 0
        assert abs(got - want) <= 1e-10 * abs(want), (z, got, want)


def test_noalloc_overlap_rejects_oversized_plane(fd, gpu):
    dummy = C.c_void_p(16)
    rc = fd.lib.fdtd_mode_overlap_plane_noalloc(dummy, dummy, dummy, dummy, fd.F64, 4, 9000, 2, 2, dummy, 2, 2,
                                                1.0, 0, 0.05, dummy, None)
    assert rc == fd.FDTD_ERR_ARG
    assert "8192" in fd.lib.fdtd_last_error_message().decode()
    fd.lib.fdtd_clear_error()


def test_noalloc_overlap_rejects_misaligned_pointers(fd, gpu):
    # refused on the host before any launch: result / mode must be 16-byte aligned,
    # field planes aligned to their element size (nothing is dereferenced).  The
    # plane is also taller than the scratch allows, so a library without the
    # alignment check would still refuse the call (for the row count) rather
    # than launch on these addresses.
    ok16, off8, off4 = C.c_void_p(256), C.c_void_p(264), C.c_void_p(260)
    cases = [
        (ok16, ok16, fd.F64, off8),   # result at 8 bytes past a 16-byte boundary
        (ok16, off8, fd.F64, ok16),   # mode_fields likewise
        (off4, ok16, fd.F64, ok16),   # a double plane at 4 bytes
        (C.c_void_p(258), ok16, fd.F32, ok16),   # a float plane at 2 bytes
    ]
    for plane, mode_ptr, prec, result in cases:
        rc = fd.lib.fdtd_mode_overlap_plane_noalloc(plane, ok16, ok16, ok16, prec, 4, 9000, 2, 2, mode_ptr, 2, 2,
                                                    1.0, 0, 0.05, result, None)
        assert rc == fd.FDTD_ERR_ARG
        assert "aligned" in fd.lib.fdtd_last_error_message().decode()
        fd.lib.fdtd_clear_error()
