"""Python mirror of libfdtd_b200's C ABI (include/fdtd_b200.h).

The engine is the shared library 3d_fdtd_b200/lib/libfdtd_b200.so, built by
3d_fdtd_b200/build.py.  This module binds it with ctypes under the reference's
own function names (timefield3d_*, adjoint3d_taper_*), so tests and the bench
drive exactly the entry points a C caller of the reference would link.  It has
no compute of its own: when the library is missing, importing this package
raises, and device entry points report FDTD_ERR_NO_DEVICE without a GPU.

Import with ``importlib.import_module("3d_fdtd_b200")`` (the directory name
starts with a digit).
"""
from __future__ import annotations

import ctypes as C
import gzip
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libfdtd_b200.so")

FDTD_OK, FDTD_ERR_NO_DEVICE, FDTD_ERR_CUDA, FDTD_ERR_ARG, FDTD_ERR_ALLOC = 0, 1, 2, 3, 4
FDTD_ERR_UNSUPPORTED, FDTD_ERR_TIMEOUT, FDTD_ERR_NONFINITE = 5, 6, 7
F64, F32 = 0, 1
MUR, CPML, PEC = 0, 1, 2
YEE_AUTO, YEE_FLAT, YEE_FUSED, YEE_FLAT4, YEE_WAVE, YEE_STREAM = 0, 1, 2, 3, 4, 5

# the reference's constants (3d_fdtd.c:12, timefield3d.c:3)
REF_PI = 3.141592652


class Complex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class Matrix(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("m", C.POINTER(Complex))]


class Mode(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("disc", C.c_double),
                ("pml", Matrix), ("ep", Matrix), ("mu", Matrix), ("fields", Matrix)]


class Timefield3d(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("k", C.c_int), ("disc", C.c_double),
                ("ep", C.POINTER(C.c_float)), ("mu", C.POINTER(C.c_float)),
                ("sig", C.POINTER(C.c_float)), ("fields", C.POINTER(C.c_double)),
                ("old_fields", C.POINTER(C.c_double)),
                ("fourier_fields", C.POINTER(Complex)), ("sources", C.POINTER(C.c_float))]


class Taper(C.Structure):
    _fields_ = [("ep", C.c_double), ("mu", C.c_double), ("seg_num", C.c_int), ("start", C.c_int),
                ("end", C.c_int), ("bottom", C.c_int), ("top", C.c_int), ("duration", C.c_int),
                ("left", C.POINTER(C.c_int)), ("right", C.POINTER(C.c_int)),
                ("forward_fields", C.POINTER(C.c_double)), ("adjoint_fields", C.POINTER(C.c_double)),
                ("ep_gradient", C.POINTER(C.c_double)), ("left_grad", C.POINTER(C.c_double)),
                ("right_grad", C.POINTER(C.c_double))]


T, M, P = Timefield3d, Mode, Taper
d, i, f, ll = C.c_double, C.c_int, C.c_float, C.c_longlong
dp, ip, cp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(Complex)

# name -> (restype, argtypes), in the order of include/fdtd_b200.h
SIGNATURES = {
    "timefield3d_new": (T, [i, i, i, d]),
    "timefield3d_free": (None, [T]),
    "timefield3d_copy": (T, [T]),
    "timefield3d_zero_fields": (None, [T]),
    "timefield3d_get_fields": (dp, [T]),
    "timefield3d_get_edge_fields": (dp, [T]),
    "timefield3d_update_old_edge_fields": (None, [T]),
    **{f"timefield3d_plot_{n}": (None, [T, i]) for n in (
        "Ex_x_slice", "Ex_y_slice", "Ex_z_slice", "Ey_x_slice", "Ey_y_slice", "Ey_z_slice",
        "Ez_x_slice", "Ez_y_slice", "Ez_z_slice", "Ex_x_slice_fourier", "Ex_y_slice_fourier",
        "Ex_z_slice_fourier", "permittivity_x_slice", "permittivity_y_slice", "permittivity_z_slice")},
    "timefield3d_set_background": (None, [T, f, f]),
    "timefield3d_set_top_half_plane": (None, [T, f, f, i]),
    "timefield3d_set_background_permittivity": (None, [T, f]),
    "timefield3d_set_background_permeability": (None, [T, f]),
    "timefield3d_set_background_electric_conductivity": (None, [T, f]),
    "timefield3d_set_background_magnetic_conductivity": (None, [T, f]),
    "timefield3d_set_background_complex_permittivity": (None, [T, d, f, f]),
    "timefield3d_set_prism_permittivity": (None, [T, f, i, i, i, i, i, i]),
    "timefield3d_set_prism_electric_conductivity": (None, [T, f, i, i, i, i, i, i]),
    "timefield3d_set_prism_complex_permittivity": (None, [T, d, f, f, i, i, i, i, i, i]),
    "timefield3d_set_waveguide": (None, [T, f, i, i, i, i, i, i]),
    "timefield3d_set_taper": (None, [T, d, d, i, i, i, i, i, i, i, i]),
    "timefield3d_apply_H_timestep": (None, [T, d]),
    "timefield3d_apply_E_timestep": (None, [T, d]),
    "timefield3d_apply_H_timestep_zsection": (None, [T, d, i, i]),
    "timefield3d_apply_E_timestep_zsection": (None, [T, d, i, i]),
    "timefield3d_apply_H_first_order_abc": (None, [T, dp, d]),
    "timefield3d_apply_E_first_order_abc": (None, [T, dp, d]),
    "timefield3d_apply_H_first_order_abc_zsection": (None, [T, d, i, i]),
    "timefield3d_apply_E_first_order_abc_zsection": (None, [T, d, i, i]),
    "timefield3d_apply_timestep": (None, [T, d]),
    "timefield3d_apply_timestep_omp": (None, [T, d]),
    "timefield3d_apply_timestep_omp_full": (None, [T, d]),
    "timefield3d_update_fourier_fields": (None, [T, d]),
    "timefield3d_update_fourier_fields_y_slice": (None, [T, d, i]),
    "timefield3d_update_fourier_fields_zsection": (None, [T, d, i, i]),
    "timefield3d_update_fourier_fields_y_slice_zsection": (None, [T, d, i, i, i]),
    "timefield3d_update_fourier_fields_omp": (None, [T, d]),
    "timefield3d_update_fourier_fields_y_slice_omp": (None, [T, d, i]),
    "timefield3d_mode_source": (None, [T, i, i, i, M, d, d, i]),
    "timefield3d_mode_source_adjoint": (None, [T, i, i, i, M, d, i]),
    "timefield3d_TE_gaussian_source": (None, [T, i, i, i, d, d, d, d]),
    "timefield3d_TM_gaussian_source": (None, [T, i, i, i, d, d, d, d]),
    "timefield3d_mode_overlap": (Complex, [T, i, i, i, M, d, i, cp]),
    "timefield3d_file_write_permittivity_y_slice": (None, [T, C.c_char_p, i, i, i, i, i, d, d]),
    "adjoint3d_taper_new": (P, [d, d, i, i, i, ip, ip, i, i, i]),
    "adjoint3d_taper_insert": (None, [T, P]),
    "adjoint3d_taper_store_forward_fields": (None, [P, T, i]),
    "adjoint3d_taper_store_adjoint_fields": (None, [P, T, i]),
    "adjoint3d_taper_calculate_ep_gradient": (None, [P]),
    "adjoint3d_taper_calculate_gradients_from_ep_gradient": (None, [P, d]),
    "adjoint3d_taper_update_symmetric": (i, [P, d, d, i]),
    "adjoint3d_taper_update_asymmetric": (i, [P, d, d, i]),
    "adjoint3d_taper_free": (None, [P]),
    "fdtd_last_error": (i, []),
    "fdtd_last_error_message": (C.c_char_p, []),
    "fdtd_error_string": (C.c_char_p, [i]),
    "fdtd_clear_error": (None, []),
    "fdtd_device_count": (i, []),
    "fdtd_version": (C.c_char_p, []),
    "timefield3d_set_precision": (i, [T, i]),
    "timefield3d_set_boundary": (i, [T, i]),
    "timefield3d_set_yee_variant": (i, [T, i]),
    "timefield3d_set_cpml": (i, [T, i, i, d, d, d]),
    "timefield3d_sync_host": (i, [T]),
    "timefield3d_sync_device": (i, [T]),
    "timefield3d_synchronize": (i, [T]),
    "timefield3d_set_source_value": (i, [T, i, i, i, i, f]),
    "timefield3d_get_field_value": (d, [T, i, i, i, i]),
    "timefield3d_add_probe": (i, [T, i, i, i, i, i]),
    "timefield3d_read_probe": (i, [T, i, dp, i]),
    "timefield3d_clear_probes": (i, [T]),
    "timefield3d_add_overlap_monitor": (i, [T, i, i, i, M, i, i, dp]),
    "timefield3d_read_overlap_monitor": (i, [T, i, cp]),
    "timefield3d_clear_monitors": (i, [T]),
    "timefield3d_step_count": (ll, [T]),
    "timefield3d_set_source_schedule": (i, [T, i, i, i, M, i, i, i, dp, dp]),
    "timefield3d_clear_source_schedule": (i, [T]),
    "timefield3d_set_exact_adjoint_schedule": (i, [T, i, i, i, M, i, i, d, d, d, d]),
    "adjoint3d_taper_bind_store": (i, [P, T, i, i, i]),
    "adjoint3d_taper_unbind_store": (i, [P, T]),
    "timefield3d_run": (i, [T, d, i]),
    "timefield3d_release_mode": (i, [M]),
    "adjoint3d_taper_sync_host": (i, [P]),
    "fdtd_set_device": (i, [i]),
    "fdtd_launch_count": (ll, []),
    "fdtd_wait_selftest": (i, [d, dp]),
    "fdtd_mode_solve_beta_squared": (Complex, [C.POINTER(Mode), d, d, C.POINTER(Mode), i, i, i, i]),
    "fdtd_mode_solve_restarts": (i, []),
    "fdtd_mode_apply_beta_squared": (i, [Mode, d, Mode]),
    "fdtd_spline_basis": (i, [i, i, i, dp]),
    "timefield3d_checkpoint_save": (i, [T, C.c_char_p]),
    "timefield3d_checkpoint_load": (i, [T, C.c_char_p]),
    "fdtd_inject_allocation_failures": (None, [i]),
    "fdtd_mlp_new": (C.c_void_p, [i, i, i, C.c_ulonglong]),
    "fdtd_mlp_param_count": (ll, [C.c_void_p]),
    "fdtd_mlp_get_params": (i, [C.c_void_p, C.POINTER(C.c_float)]),
    "fdtd_mlp_set_params": (i, [C.c_void_p, C.POINTER(C.c_float)]),
    "fdtd_mlp_forward": (i, [C.c_void_p, C.POINTER(C.c_float), i, C.POINTER(C.c_float)]),
    "fdtd_mlp_gradients": (i, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), i, C.POINTER(C.c_float),
                               C.POINTER(C.c_double)]),
    "fdtd_mlp_train_step": (i, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), i, C.c_float,
                                C.POINTER(C.c_double)]),
    "fdtd_mlp_input_gradient": (i, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), i,
                                    C.POINTER(C.c_float)]),
    "fdtd_mlp_free": (None, [C.c_void_p]),
    "fdtd_gemm_bf16": (i, [C.c_void_p, i, C.c_void_p, i, i, i, i, C.c_void_p, i, C.c_float, C.c_float, C.c_void_p,
                           i, C.c_void_p, i, C.c_void_p, i, C.c_void_p, C.c_void_p]),
    "timefield3d_set_spline_taper": (i, [T, d, d, i, dp, d, i, i, i, i]),
    "fdtd_spline_store_new": (C.c_void_p, [T, i, dp, d, i, i, i, i, i]),
    "fdtd_spline_store_bind": (i, [C.c_void_p, T, i, i, i]),
    "fdtd_spline_store_unbind": (i, [C.c_void_p, T]),
    "fdtd_spline_store_gradient": (i, [C.c_void_p, d, dp, dp]),
    "fdtd_spline_store_gradient_exact": (i, [C.c_void_p, d, dp, dp]),
    "fdtd_spline_store_gradient_step": (i, [C.c_void_p, d, d, dp]),
    "fdtd_spline_store_free": (None, [C.c_void_p]),
    "timefield3d_get_stream": (C.c_void_p, [T]),
    "timefield3d_upload_materials": (i, [T]),
    "timefield3d_set_kernel_timing": (i, [T, i]),
    "timefield3d_set_wave_steps": (i, [T, i, i, i]),
    "fdtd_wave_schedule": (i, [i, i, i, i, i, i, i, ip, i, i, ip, i, ip]),
    "timefield3d_read_kernel_timing": (i, [T, dp, C.POINTER(ll)]),
    "fdtd_sweep_run": (i, [C.POINTER(T), i, d, ip, i, i, d]),
    "fdtd_sweep_barrier_selftest": (i, [d]),
    "fdtd_stream_plan": (i, [i, i, i, i, i, i, ip, i, ip, ip, C.POINTER(C.c_longlong)]),
    "fdtd_mode_overlap_plane_noalloc": (i, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, i, i, i, i, i,
                                            C.c_void_p, i, i, d, i, d, C.c_void_p, C.c_void_p]),
}


class FdtdError(RuntimeError):
    pass


def load_library(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built: run `python 3d_fdtd_b200/build.py` "
                          f"(the engine has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load_library()
libc = C.CDLL(None)
libc.free.argtypes = [C.c_void_p]


def check(what: str = "") -> None:
    """Raise FdtdError if the library recorded an error (then clear it)."""
    code = lib.fdtd_last_error()
    if code != FDTD_OK:
        msg = lib.fdtd_last_error_message().decode()
        lib.fdtd_clear_error()
        raise FdtdError(f"{what}: {lib.fdtd_error_string(code).decode()} ({code}): {msg}")


def call(name: str, *args):
    """Call entry point `name` and raise on a recorded error."""
    r = getattr(lib, name)(*args)
    check(name)
    return r


# ---------------------------------------------------------------------------
# modes in the reference's text format (mode.c:843-1038)
# ---------------------------------------------------------------------------
class HostMode:
    """A reference `mode` whose arrays live in numpy (kept alive by this object)."""

    def __init__(self, fields: np.ndarray, disc: float, ep: np.ndarray | None = None,
                 mu: np.ndarray | None = None):
        mj, mi, six = fields.shape
        assert six == 6
        self.fields = np.ascontiguousarray(fields, dtype=np.complex128)
        self.ep = np.ascontiguousarray(ep if ep is not None else np.ones((mj, mi, 3)), dtype=np.complex128)
        self.mu = np.ascontiguousarray(mu if mu is not None else np.ones((mj, mi, 3)), dtype=np.complex128)
        self.pml = np.ones((mj, mi, 2), dtype=np.complex128)
        self.disc = float(disc)
        cptr = lambda a: a.ctypes.data_as(C.POINTER(Complex))
        self.struct = Mode(mi, mj, self.disc, Matrix(2 * mi * mj, 1, cptr(self.pml)),
                           Matrix(3 * mi * mj, 1, cptr(self.ep)), Matrix(3 * mi * mj, 1, cptr(self.mu)),
                           Matrix(6 * mi * mj, 1, cptr(self.fields)))
        # the library writes through these pointers (power normalisation in
        # place, as the reference does): the struct keeps its arrays alive even
        # when only `HostMode(...).struct` is held
        self.struct._owner = self

    @property
    def mi(self):
        return self.struct.i

    @property
    def mj(self):
        return self.struct.j

    def copy(self) -> "HostMode":
        return HostMode(self.fields.copy(), self.disc, self.ep.copy(), self.mu.copy())


def read_mode_file(path: str) -> HostMode:
    """Parse a mode written by mode_file_print (.txt or .txt.gz)."""
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rt") as fh:
        tok = fh.read().split()
    mi, mj, disc, dim = int(tok[0]), int(tok[1]), float(tok[2]), int(tok[3])
    vals = np.array(tok[4:], dtype=np.float64)
    if dim == 2:
        rec = vals.reshape(mi, mj, 24)                  # file order: i outer, j inner
        rec = rec.transpose(1, 0, 2)                    # -> [j][i]
    elif dim == 1:
        rec = np.broadcast_to(vals.reshape(mj, 1, 24), (mj, mi, 24))
    else:
        raise ValueError(f"mode file dimension {dim}")
    cplx = rec[..., 0::2] + 1j * rec[..., 1::2]         # 12 complex per cell
    return HostMode(cplx[..., 6:12], disc, cplx[..., 0:3], cplx[..., 3:6])


# ---------------------------------------------------------------------------
# convenience wrapper around a timefield3d
# ---------------------------------------------------------------------------
class Grid:
    """Owns one `timefield3d` created by the library."""

    def __init__(self, nx: int, ny: int, nz: int, disc: float, precision: int = F64):
        self.t = call("timefield3d_new", nx, ny, nz, disc)
        self.nx, self.ny, self.nz, self.disc = nx, ny, nz, disc
        if precision != F64:
            call("timefield3d_set_precision", self.t, precision)

    def close(self):
        if self.t is not None:
            lib.timefield3d_free(self.t)
            self.t = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # host mirrors, (nz, ny, nx, c) like the reference's AoS index order
    def _view(self, ptr, comps, dtype):
        n = self.nx * self.ny * self.nz * comps
        return np.ctypeslib.as_array(ptr, shape=(n,)).view(dtype).reshape(self.nz, self.ny, self.nx, comps)

    @property
    def ep(self):
        return self._view(self.t.ep, 3, np.float32)

    @property
    def mu(self):
        return self._view(self.t.mu, 3, np.float32)

    @property
    def sig(self):
        return self._view(self.t.sig, 6, np.float32)

    def fields(self) -> np.ndarray:
        """Device fields copied to the host mirror, (nz, ny, nx, 6) float64."""
        call("timefield3d_sync_host", self.t)
        return self._view(self.t.fields, 6, np.float64).copy()

    def fourier(self) -> np.ndarray:
        call("timefield3d_sync_host", self.t)
        n = self.nx * self.ny * self.nz * 6
        a = np.ctypeslib.as_array(C.cast(self.t.fourier_fields, dp), shape=(2 * n,))
        return a.view(np.complex128).reshape(self.nz, self.ny, self.nx, 6).copy()

    def __getattr__(self, name):
        # grid.apply_timestep_omp_full(dt) -> timefield3d_apply_timestep_omp_full(t, dt)
        fn = "timefield3d_" + name
        if fn not in SIGNATURES:
            raise AttributeError(name)
        return lambda *a: call(fn, self.t, *a)
