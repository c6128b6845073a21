"""Ensembles of independent channels advanced by one CUDA graph per step
(include/diablo_b200.h, db_ensemble_*): the data-generation runs of the
learned closure (many small channels with different seeds and Ri).  Members
of one size without LES at a fixed dt are batched: each kernel of the step
is launched once for all of them."""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import lib as _L
from .channel import Channel


def config4_members(n: int = 64, nx: int = 128, ny: int = 65, nz: int = 128, re: float = 2000.0,
                    precision: int = 1, seed: int = 1000):
    """Parameters of the closure-data ensemble: member i has seed i and
    Ri_i ~ U[0.5, 2] (numpy PCG64(seed)), f = 1, N^2 = 1 and the horizontal
    buoyancy gradient M^2 = sqrt(N^2 f^2 / Ri)."""
    from .params import make_params
    rng = np.random.Generator(np.random.PCG64(seed))
    ri = rng.uniform(0.5, 2.0, n)
    out = []
    for i in range(n):
        m2 = math.sqrt(1.0 / ri[i])
        out.append(make_params(
            nx=nx, ny=ny, nz=nz, lx=2 * math.pi, lz=2 * math.pi, ly=2.0, re=re, pr=1.0, ri=1.0, ro=1.0,
            delta=1.0, grav_y=1.0, ic_type=4, kick=1e-3, delta_t=1e-3, variable_dt=0,
            u_bc_ymin=0, w_bc_ymin=0, v_bc_ymin=0, th_bc_ymin=1, u_bc_ymax=1, w_bc_ymax=1, v_bc_ymax=0,
            th_bc_ymax=1, th_bc_ymin_c1=1.0, th_bc_ymax_c1=1.0, dthdx_override=m2, precision=precision))
    return out, ri


class Ensemble:
    """Channels (one context and stream each) stepped together."""

    def __init__(self, params_list, gy, seeds=None, init: bool = True, stream: int | None = None):
        self.L = _L.load()
        self.members = [Channel(p, gy) for p in params_list]
        if init:
            for i, ch in enumerate(self.members):
                ch.init_flow(seed=seeds[i] if seeds is not None else i)
        arr = (ctypes.c_void_p * len(self.members))(*[ch.h for ch in self.members])
        h = ctypes.c_void_p()
        rc = self.L.db_ensemble_create(arr, len(self.members), ctypes.c_void_p(stream) if stream else None,
                                       ctypes.byref(h))
        if rc != 0:
            raise _L.DiabloError(rc, self.L.db_ensemble_error(None).decode())
        self.h = h
        self._groups0 = self.groups   # the default grouping of the batched form (0: not batched)

    def step(self, nsteps: int = 1):
        rc = self.L.db_ensemble_steps(self.h, nsteps)
        if rc != 0:
            raise _L.DiabloError(rc, self.L.db_ensemble_error(self.h).decode())

    @property
    def groups(self) -> int:
        """Groups of the batched form (each kernel of a step launched once per
        group of members), 0 for the per-member graph branches."""
        b = ctypes.c_int()
        self.L.db_ensemble_info(self.h, ctypes.byref(b), None)
        return b.value

    @groups.setter
    def groups(self, n: int):
        rc = self.L.db_ensemble_set_batched(self.h, int(n))
        if rc != 0:
            raise _L.DiabloError(rc, "members do not qualify for the batched form")

    @property
    def batched(self) -> bool:
        return self.groups > 0

    @batched.setter
    def batched(self, on: bool):
        self.groups = (self._groups0 or 1) if on else 0

    def kernels_per_step(self) -> int:
        k = ctypes.c_longlong()
        self.L.db_ensemble_info(self.h, None, ctypes.byref(k))
        return int(k.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.db_ensemble_destroy(self.h)
            self.h = None
        for ch in getattr(self, "members", []):
            ch.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
