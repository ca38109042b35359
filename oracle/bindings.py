"""ctypes bindings for the two CPU checkers of the FDTD hot path.

TEST INFRASTRUCTURE.  Imported only by tests/, by the smoke check and by the
CPU-baseline legs of bench.py -- never by the engine itself.

* ``Reference`` wraps ``oracle/_ref/libref.so``: the reference's own C sources
  (timefield3d.c, mode.c, matrix.c, complex.c, adjoint3d.c) compiled unchanged by
  ``oracle/Makefile``.  Only compute functions are called; the gnuplot plot
  functions never are.
* ``Oracle`` wraps ``oracle/liboracle.so``: our SoA restatement in
  ``fdtd_oracle.c`` (which also defines CPML and multi-wavelength monitors).

Struct layouts follow timefield3d.h:15-27, mode.h:13-22, matrix.h:11-16,
complex.h:11-15 and adjoint3d.h:37-58.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libref.so")
ORACLE_SO = os.path.join(HERE, "liboracle.so")


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


def _arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).view(dtype) if n else np.zeros(0, dtype)


# ---------------------------------------------------------------------------
# the reference itself
# ---------------------------------------------------------------------------
class Reference:
    """The reference's compiled C (oracle/_ref/libref.so), called through its own API."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources exist")
        lib = C.CDLL(path)
        self.lib = lib
        T, M, P = Timefield3d, Mode, Taper
        d, i, f = C.c_double, C.c_int, C.c_float
        sig = {
            "timefield3d_new": (T, [i, i, i, d]),
            "timefield3d_free": (None, [T]),
            "timefield3d_zero_fields": (None, [T]),
            "timefield3d_set_background": (None, [T, f, f]),
            "timefield3d_set_top_half_plane": (None, [T, f, f, i]),
            "timefield3d_set_prism_permittivity": (None, [T, f, i, i, i, i, i, i]),
            "timefield3d_set_prism_electric_conductivity": (None, [T, f, i, i, i, i, i, i]),
            "timefield3d_set_background_magnetic_conductivity": (None, [T, f]),
            "timefield3d_set_waveguide": (None, [T, f, i, i, i, i, i, i]),
            "timefield3d_set_taper": (None, [T, d, d, i, i, i, i, i, i, i, i]),
            "timefield3d_apply_timestep_omp_full": (None, [T, d]),
            "timefield3d_update_fourier_fields_y_slice_omp": (None, [T, d, i]),
            "timefield3d_mode_source": (None, [T, i, i, i, M, d, d, i]),
            "timefield3d_mode_source_adjoint": (None, [T, i, i, i, M, d, i]),
            "timefield3d_mode_overlap": (Complex, [T, i, i, i, M, d, i, C.POINTER(Complex)]),
            "timefield3d_file_write_permittivity_y_slice": (None, [T, C.c_char_p, i, i, i, i, i, d, d]),
            "mode_file_load": (M, [C.c_void_p]),
            "mode_new": (M, [i, i, d]),
            "mode_free": (None, [M]),
            "mode_smul": (None, [Complex, M]),
            "mode_power_normalize": (None, [M]),
            "mode_power_norm": (d, [M]),
            "mode_set_background": (None, [M, Complex, Complex]),
            "mode_make_rectangle": (None, [M, Complex, Complex, i, i, i, i]),
            "mode_set_pml": (None, [M, d, i, i]),
            "mode_apply_beta_squared_operator": (M, [M, d]),
            "mode_solve_beta_squared": (Complex, [C.POINTER(M), d, d, C.POINTER(M), i, i, i, i]),
            "complex_exp": (Complex, [Complex]),
            "adjoint3d_taper_new": (P, [d, d, i, i, i, C.POINTER(i), C.POINTER(i), i, i, i]),
            "adjoint3d_taper_insert": (None, [T, P]),
            "adjoint3d_taper_store_forward_fields": (None, [P, T, i]),
            "adjoint3d_taper_store_adjoint_fields": (None, [P, T, i]),
            "adjoint3d_taper_calculate_ep_gradient": (None, [P]),
            "adjoint3d_taper_calculate_gradients_from_ep_gradient": (None, [P, d]),
            "adjoint3d_taper_update_asymmetric": (i, [P, d, d, i]),
            "adjoint3d_taper_update_symmetric": (i, [P, d, d, i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.gomp = C.CDLL("libgomp.so.1")
        self.gomp.omp_set_num_threads.argtypes = [C.c_int]
        self.gomp.omp_get_max_threads.restype = C.c_int
        libc = C.CDLL(None)
        libc.fopen.restype = C.c_void_p
        libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
        libc.fclose.argtypes = [C.c_void_p]
        self.libc = libc

    def __getattr__(self, name):
        return getattr(self.lib, name)

    def set_threads(self, n: int) -> None:
        """OpenMP threads of the reference's step (calling thread's default).

        The reference splits z into one slab per thread and runs the Mur faces
        of each slab independently (timefield3d.c:2794-2848); the z=0 / z=end
        faces read plane 1 / nz-2, which belong to the same slab only while
        every slab holds at least 2 planes.  Keep n <= nz/2 for a deterministic
        reference result."""
        self.gomp.omp_set_num_threads(int(n))

    # convenience views -------------------------------------------------------
    @staticmethod
    def fields(tf: Timefield3d) -> np.ndarray:
        """(k, j, i, 6) view of the AoS field array (timefield3d.c:1553 index order)."""
        n = tf.i * tf.j * tf.k
        return _arr(tf.fields, 6 * n, np.float64).reshape(tf.k, tf.j, tf.i, 6)

    @staticmethod
    def eps(tf: Timefield3d) -> np.ndarray:
        n = tf.i * tf.j * tf.k
        return _arr(tf.ep, 3 * n, np.float32).reshape(tf.k, tf.j, tf.i, 3)

    @staticmethod
    def mus(tf: Timefield3d) -> np.ndarray:
        n = tf.i * tf.j * tf.k
        return _arr(tf.mu, 3 * n, np.float32).reshape(tf.k, tf.j, tf.i, 3)

    @staticmethod
    def sources(tf: Timefield3d) -> np.ndarray:
        n = tf.i * tf.j * tf.k
        return _arr(tf.sources, 6 * n, np.float32).reshape(tf.k, tf.j, tf.i, 6)

    @staticmethod
    def sig(tf: Timefield3d) -> np.ndarray:
        n = tf.i * tf.j * tf.k
        return _arr(tf.sig, 6 * n, np.float32).reshape(tf.k, tf.j, tf.i, 6)

    def load_mode(self, path: str) -> Mode:
        fp = self.libc.fopen(path.encode(), b"r")
        if not fp:
            raise FileNotFoundError(path)
        m = self.lib.mode_file_load(fp)
        self.libc.fclose(fp)
        return m

    @staticmethod
    def mode_array(m: Mode) -> np.ndarray:
        """(mj, mi, 6) complex128 view of a mode's fields (mode.c:843 index order)."""
        n = m.i * m.j
        p = C.cast(m.fields.m, C.POINTER(C.c_double))
        return _arr(p, 12 * n, np.float64).view(np.complex128).reshape(m.j, m.i, 6)


# ---------------------------------------------------------------------------
# the restatement
# ---------------------------------------------------------------------------
class Oracle:
    """Our CPU restatement (oracle/liboracle.so) in SoA double precision."""

    PEC, MUR, CPML = 0, 1, 2

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle liboracle.so`")
        lib = C.CDLL(path)
        self.lib = lib
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        sig = {
            "orc_new": (vp, [i, i, i, d]), "orc_free": (None, [vp]), "orc_zero": (None, [vp]),
            "orc_field": (dp, [vp, i]), "orc_ep": (C.POINTER(C.c_float), [vp, i]),
            "orc_mu": (C.POINTER(C.c_float), [vp, i]), "orc_sig": (C.POINTER(C.c_float), [vp, i]),
            "orc_src": (C.POINTER(C.c_float), [vp, i]), "orc_set_boundary": (None, [vp, i]),
            "orc_set_cpml": (None, [vp, i, i, d, d, d, d]), "orc_cpml_profile": (dp, [vp, i, i]),
            "orc_step": (None, [vp, d]), "orc_step_threads": (None, [i]),
            "orc_mode_power_norm": (d, [dp, i, i, d]), "orc_mode_power_normalize": (None, [dp, i, i, d]),
            "orc_mode_source": (None, [vp, i, i, i, dp, i, i, d, d, d, i]),
            "orc_mode_source_adjoint": (None, [vp, i, i, i, dp, i, i, d, d, i]),
            "orc_mode_overlap": (None, [vp, i, i, i, dp, i, i, d, d, i, dp, dp]),
            "orc_overlap_instant": (None, [vp, i, i, i, dp, i, i, d, i, dp]),
            "orc_cexp_series": (None, [d, dp, dp]), "orc_reduce_phase": (d, [d]),
            "orc_dft_y_slice": (None, [vp, d, i, dp]),
            "orc_taper_store": (None, [vp, i, i, i, i, i, ip, ip, i, dp]),
            "orc_taper_ep_gradient": (None, [i, i, i, dp, dp, dp]),
            "orc_taper_vertex_gradient": (None, [i, i, i, dp, d, dp, dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args

    def __getattr__(self, name):
        return getattr(self.lib, name)

    @staticmethod
    def ptr(a: np.ndarray, ctype=C.c_double):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data_as(C.POINTER(ctype))

    def cexp(self, x: float) -> complex:
        re, im = C.c_double(), C.c_double()
        self.lib.orc_cexp_series(x, C.byref(re), C.byref(im))
        return complex(re.value, im.value)


class OracleGrid:
    """A grid in the restatement with numpy views of its SoA arrays, shape (nz, ny, nx)."""

    def __init__(self, orc: Oracle, nx: int, ny: int, nz: int, dx: float):
        self.orc, self.nx, self.ny, self.nz, self.dx = orc, nx, ny, nz, dx
        self.h = orc.orc_new(nx, ny, nz, dx)
        shape = (nz, ny, nx)
        n = nx * ny * nz
        self.f = [_arr(orc.orc_field(self.h, m), n, np.float64).reshape(shape) for m in range(6)]
        self.ep = [_arr(orc.orc_ep(self.h, c), n, np.float32).reshape(shape) for c in range(3)]
        self.mu = [_arr(orc.orc_mu(self.h, c), n, np.float32).reshape(shape) for c in range(3)]
        self.sig = [_arr(orc.orc_sig(self.h, m), n, np.float32).reshape(shape) for m in range(6)]
        self.src = [_arr(orc.orc_src(self.h, m), n, np.float32).reshape(shape) for m in range(6)]

    def close(self):
        if self.h:
            self.orc.orc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_boundary(self, b: int):
        self.orc.orc_set_boundary(self.h, b)

    def set_cpml(self, npml, order=3, sigma_max=-1.0, kappa_max=1.0, alpha_max=0.0, dt=None):
        self.orc.orc_set_cpml(self.h, npml, order, sigma_max, kappa_max, alpha_max, dt)

    def step(self, dt: float):
        self.orc.orc_step(self.h, dt)

    def zero(self):
        self.orc.orc_zero(self.h)

    def fields(self) -> np.ndarray:
        """(nz, ny, nx, 6) copy, same index order as Reference.fields."""
        return np.stack([a.copy() for a in self.f], axis=-1)
