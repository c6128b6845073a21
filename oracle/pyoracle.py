"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
import this module; it is the checker, never the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

# state array ids (include/diablo_b200.h enum db_field) and oracle work arrays
CU1, CU2, CU3, CP, CTH, CF1, CF2, CF3, CFTH, NU_T, KAPPA_T = range(11)
R1, R2, R3, RTH, S1 = 100, 101, 102, 103, 104


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc (oracle/Makefile)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp, dp]
        L.orc_destroy.argtypes = [vp]
        L.orc_error.restype = ctypes.c_char_p
        L.orc_array_len.restype = ctypes.c_long
        L.orc_array_len.argtypes = [vp]
        L.orc_array.restype = dp
        L.orc_array.argtypes = [vp, ip]
        L.orc_metric.restype = dp
        L.orc_metric.argtypes = [vp, ip]
        L.orc_fft_xz_to_fourier.argtypes = [vp, dp]
        L.orc_fft_xz_to_physical.argtypes = [vp, dp]
        L.orc_rk_chan_1.argtypes = [vp, ip]
        L.orc_rk_chan_1.restype = ip
        L.orc_step.argtypes = [vp]
        L.orc_step.restype = ip
        L.orc_rem_div_chan.argtypes = [vp]
        L.orc_poisson_p_chan.argtypes = [vp]
        L.orc_apply_bc_vel_post.argtypes = [vp]
        L.orc_courant_physical.argtypes = [vp]
        L.orc_courant_physical.restype = ctypes.c_double
        L.orc_set_clock.argtypes = [vp, ctypes.c_double, ip, ctypes.c_double, ctypes.c_double]
        L.orc_get_clock.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int), dp]
        L.orc_fft_c2c.argtypes = [dp, ip, ip]
        L.orc_fft_c2c.restype = ip
        L.orc_dft_c2c_ld.argtypes = [dp, ip, ip]
        L.orc_thomas_real.argtypes = [dp, dp, dp, dp, ip, ip]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fft_c2c(x: np.ndarray, sign: int = -1) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).view(np.float64).copy()
    if lib().orc_fft_c2c(_dptr(a), len(a) // 2, sign):
        raise ValueError("length must be a power of two")
    return a.view(np.complex128)


def dft_c2c_ld(x: np.ndarray, sign: int = -1) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).view(np.float64).copy()
    lib().orc_dft_c2c_ld(_dptr(a), len(a) // 2, sign)
    return a.view(np.complex128)


def thomas_real(a, b, c, g, ny: int, inx: int) -> np.ndarray:
    a, b, c, g = (np.ascontiguousarray(v, dtype=np.float64).copy() for v in (a, b, c, g))
    lib().orc_thomas_real(_dptr(a), _dptr(b), _dptr(c), _dptr(g), ny, inx)
    return g


class Oracle:
    """One reference-layout channel state on the CPU."""

    def __init__(self, params, gy):
        self.p = params
        self.gy = np.ascontiguousarray(gy, dtype=np.float64)
        self._h = lib().orc_create(ctypes.byref(params), _dptr(self.gy))
        if not self._h:
            raise ValueError(lib().orc_error().decode())
        self.n = lib().orc_array_len(self._h)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # --- arrays -----------------------------------------------------------
    def real(self, fid: int) -> np.ndarray:
        """Live real view (Nyp+2, Nz+2, Nx+2) of a state array."""
        ptr = lib().orc_array(self._h, fid)
        a = np.ctypeslib.as_array(ptr, shape=(self.n,))
        p = self.p
        return a.reshape(p.ny + 2, p.nz + 2, p.nx + 2)

    def cplx(self, fid: int) -> np.ndarray:
        """Live complex view (Nyp+2, Nz+2, Nxp+1)."""
        p = self.p
        return self.real(fid).reshape(-1).view(np.complex128).reshape(p.ny + 2, p.nz + 2, p.nxp + 1)

    def set(self, fid: int, values: np.ndarray):
        self.real(fid).reshape(-1)[:] = np.asarray(values, dtype=np.float64).reshape(-1)

    def get(self, fid: int) -> np.ndarray:
        return self.real(fid).copy()

    def metric(self, which: int, n: int) -> np.ndarray:
        ptr = lib().orc_metric(self._h, which)
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

    # --- operations -------------------------------------------------------
    def fft_to_fourier(self, buf: np.ndarray):
        lib().orc_fft_xz_to_fourier(self._h, _dptr(buf))

    def fft_to_physical(self, buf: np.ndarray):
        lib().orc_fft_xz_to_physical(self._h, _dptr(buf))

    def rk_substep(self, rk: int):
        if lib().orc_rk_chan_1(self._h, rk):
            raise RuntimeError(lib().orc_error().decode())

    def step(self):
        if lib().orc_step(self._h):
            raise RuntimeError(lib().orc_error().decode())

    def rem_div(self):
        lib().orc_rem_div_chan(self._h)

    def poisson_p(self):
        lib().orc_poisson_p_chan(self._h)

    def apply_bc_vel_post(self):
        lib().orc_apply_bc_vel_post(self._h)

    def courant_physical(self) -> float:
        return lib().orc_courant_physical(self._h)

    def set_clock(self, time=0.0, time_step=0, save_stats_time=1e300, save_flow_time=1e300):
        lib().orc_set_clock(self._h, time, time_step, save_stats_time, save_flow_time)

    def clock(self):
        t = ctypes.c_double()
        s = ctypes.c_int()
        d = ctypes.c_double()
        lib().orc_get_clock(self._h, ctypes.byref(t), ctypes.byref(s), ctypes.byref(d))
        return t.value, s.value, d.value

    def init_from_physical(self, u1, u2, u3, th):
        """create_flow_chan's tail: FFT, BCs, divergence removal
        (for/flow.f90:429-488); cp from the (zero) pressure."""
        for fid, v in ((CU1, u1), (CU2, u2), (CU3, u3), (CTH, th)):
            self.set(fid, v)
            self.fft_to_fourier(self.real(fid).reshape(-1))
        self.set(CP, np.zeros(self.n))
        self.apply_bc_vel_post()
        self.rem_div()
