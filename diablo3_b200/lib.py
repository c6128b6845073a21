"""ctypes binding of libdiablo_b200.so (include/diablo_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import DbParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdiablo_b200.so")

# enum db_field
CU1, CU2, CU3, CP, CTH, CF1, CF2, CF3, CFTH, NU_T, KAPPA_T = range(11)
DB_ZS_FIELD, DB_ZS_KE = 0, 1   # db_bin_ystar kinds
LES_ROWS = ("nu_sgs", "kappa_sgs", "eps_sgs2")   # db_les_stats rows
# rows of db_stats (include/diablo_b200.h order)
NTUNE = 6   # DB_NTUNE
STAT_ROWS = ("ume", "vme", "wme", "thme", "urms", "vrms", "wrms", "thrms", "uv", "wv", "uw", "thv", "epsilon", "chi")
# rows of db_budget
BUDGET_ROWS = ("tke", "uu_dudx", "wu_dwdx", "vu_dvdx", "vv_dvdy", "uv_dudy", "wv_dwdy", "epsilon_m",
               "omega_x", "omega_y", "omega_z")
STATE_FIELDS = (CU1, CU2, CU3, CP, CTH, CF1, CF2, CF3, CFTH)
# what a full RK step reads and writes: the CF history is rebuilt in its
# first substep before any read (for/solver.f90:413, 487)
STEP_FIELDS = (CU1, CU2, CU3, CP, CTH)

# exported symbols, in header order
EXPORTS = (
    "db_abi_version", "db_last_error", "db_init", "db_finalize",
    "db_upload_state", "db_download_state", "db_upload_field", "db_download_field",
    "db_set_clock", "db_get_status", "db_clear_status",
    "db_fft_xz_to_fourier", "db_fft_xz_to_physical", "db_fft_xz_to_fourier_dev", "db_fft_xz_to_physical_dev",
    "db_rk_substep", "db_rk_steps", "db_rem_div", "db_apply_bc_vel_post",
    "db_courant", "db_divergence", "db_stats", "db_budget", "db_bpe", "db_bin_ystar", "db_les_stats", "db_poisson_p",
    "db_autotune", "db_get_tuning", "db_set_tuning", "db_set_timing", "db_stage_times", "db_kernel_launches",
    "db_rem_div_static",
    "db_sgs_create", "db_sgs_destroy", "db_sgs_set", "db_sgs_get", "db_sgs_set_range", "db_sgs_forward",
    "db_sgs_gradient", "db_sgs_train_step", "db_sgs_gemm_check", "db_set_sgs_net", "db_les_eval",
    "db_sgs_targets",
    "db_ensemble_create", "db_ensemble_steps", "db_ensemble_destroy", "db_ensemble_error",
    "db_ensemble_set_batched", "db_ensemble_info",
    "db_set_wait_limit",
)
STAGES = ("inv_z", "inv_x", "products", "zpass_rhs", "inv_x_r", "thomas", "courant",
          "fwd_x", "fwd_z", "rem_div")


class DbStatus(ctypes.Structure):
    _fields_ = [
        ("flags", ctypes.c_int32), ("time_step", ctypes.c_int32),
        ("time", ctypes.c_double), ("delta_t", ctypes.c_double), ("max_div", ctypes.c_double),
    ]


class DiabloError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[db error {code}] {msg}")
        self.code = code


_lib = None


def load(path: str | None = None):
    """Load the library (it must have been built: diablo3_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("DIABLO_B200_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run `python -m diablo3_b200.build` (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    vp, dp, i32 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int32
    L.db_abi_version.restype = ctypes.c_int
    L.db_last_error.restype = ctypes.c_char_p
    L.db_last_error.argtypes = [vp]
    L.db_init.argtypes = [ctypes.POINTER(DbParams), dp, vp, ctypes.POINTER(vp)]
    L.db_finalize.argtypes = [vp]
    L.db_upload_state.argtypes = [vp] + [dp] * 9
    L.db_download_state.argtypes = [vp] + [dp] * 9
    L.db_upload_field.argtypes = [vp, ctypes.c_int, dp]
    L.db_download_field.argtypes = [vp, ctypes.c_int, dp]
    L.db_set_clock.argtypes = [vp, ctypes.c_double, i32, ctypes.c_double, ctypes.c_double]
    L.db_get_status.argtypes = [vp, ctypes.POINTER(DbStatus)]
    L.db_clear_status.argtypes = [vp]
    L.db_fft_xz_to_fourier.argtypes = [vp, dp]
    L.db_fft_xz_to_physical.argtypes = [vp, dp]
    L.db_fft_xz_to_fourier_dev.argtypes = [vp, vp]
    L.db_fft_xz_to_physical_dev.argtypes = [vp, vp]
    L.db_rk_substep.argtypes = [vp, ctypes.c_int]
    L.db_rk_steps.argtypes = [vp, ctypes.c_int]
    L.db_rem_div.argtypes = [vp]
    L.db_apply_bc_vel_post.argtypes = [vp]
    L.db_courant.argtypes = [vp, dp]
    L.db_divergence.argtypes = [vp, dp]
    L.db_stats.argtypes = [vp, dp]
    L.db_budget.argtypes = [vp, dp]
    L.db_poisson_p.argtypes = [vp]
    L.db_bpe.argtypes = [vp, ctypes.c_int, dp, dp, dp]
    L.db_bin_ystar.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int, dp, dp]
    L.db_les_stats.argtypes = [vp, dp]
    L.db_autotune.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    L.db_get_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    L.db_set_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    L.db_set_timing.argtypes = [vp, ctypes.c_int]
    L.db_stage_times.argtypes = [vp, dp, ctypes.c_int]
    L.db_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.db_set_wait_limit.argtypes = [vp, ctypes.c_uint32]
    L.db_rem_div_static.argtypes = [ctypes.POINTER(DbParams), dp, vp, vp, vp, vp]
    fp, ll = ctypes.POINTER(ctypes.c_float), ctypes.c_longlong
    L.db_sgs_create.argtypes = [vp, ctypes.POINTER(vp)]
    L.db_sgs_destroy.argtypes = [vp]
    L.db_sgs_set.argtypes = [vp, fp, fp, fp, fp]
    L.db_sgs_get.argtypes = [vp, fp]
    L.db_sgs_set_range.argtypes = [vp, fp, fp]
    L.db_sgs_forward.argtypes = [vp, vp, vp, ll]
    L.db_sgs_gradient.argtypes = [vp, vp, vp, ll, fp, dp]
    L.db_sgs_train_step.argtypes = [vp, vp, vp, ll, ctypes.c_float, dp]
    L.db_sgs_gemm_check.argtypes = [vp, vp, fp, ctypes.c_int, ctypes.c_int]
    L.db_set_sgs_net.argtypes = [vp, vp]
    L.db_les_eval.argtypes = [vp, ctypes.c_int, dp, dp, fp]
    L.db_ensemble_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp, ctypes.POINTER(vp)]
    L.db_ensemble_steps.argtypes = [vp, ctypes.c_int]
    L.db_ensemble_destroy.argtypes = [vp]
    L.db_ensemble_error.argtypes = [vp]
    L.db_ensemble_error.restype = ctypes.c_char_p
    L.db_ensemble_set_batched.argtypes = [vp, ctypes.c_int]
    L.db_ensemble_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]
    L.db_sgs_targets.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, vp, vp,
                                 ctypes.POINTER(ctypes.c_longlong)]
    for name in EXPORTS:
        if name not in ("db_abi_version", "db_last_error", "db_ensemble_error"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous float32")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def check(rc: int, handle=None):
    if rc != 0:
        raise DiabloError(rc, load().db_last_error(handle).decode())
