"""The benchmark workloads (seeded synthetic initial conditions, no data
set): their parameters and one-line descriptions, shared by bench.py and
the accuracy tests of the timed configurations.

  config0  64x65x64 plain FP64 DNS, fixed dt (parity/latency case)
  config1  512x257x512 plain FP64 DNS, infinite front, Re 5000, CFL 0.5
  slab     config1 with 65 wall-normal points (profiling case)
  config2  256x129x256 AMD LES of a finite front (IC 6), Re 1e5
  config3  128x65x128 LES of a finite front (IC 6), Re 1e4
"""
from __future__ import annotations

import math


def workload_params(name: str):
    from .params import make_params
    if name == "config1":
        return make_params(
            nx=512, ny=257, nz=512, lx=2 * math.pi, lz=2 * math.pi, ly=2.0,
            re=5000.0, pr=1.0, ri=1.0, ro=1.0, delta=1.0, grav_y=1.0, ic_type=4, kick=1e-3,
            delta_t=1e-3, variable_dt=1, cfl=0.5, update_dt=1, time_limit=1e9,
            u_bc_ymin=0, w_bc_ymin=0, v_bc_ymin=0, th_bc_ymin=1,
            u_bc_ymax=1, w_bc_ymax=1, v_bc_ymax=0, th_bc_ymax=1,
            th_bc_ymin_c1=1.0, th_bc_ymax_c1=1.0)
    if name == "slab":
        p = workload_params("config1")
        p.ny = 65  # 512x65x512: same planes, fields still > L2, for ncu captures
        return p
    if name == "config0":
        p = workload_params("config1")
        p.nx, p.ny, p.nz, p.re, p.variable_dt = 64, 65, 64, 1000.0, 0
        return p
    if name in ("config2", "config3"):
        # finite front (IC_type 6, front width 0.5), AMD LES, CFL-limited dt
        p = workload_params("config1")
        p.ic_type, p.delta = 6, 0.5
        p.use_les, p.les_model_type, p.create_new_flow = 1, 5, 0
        if name == "config2":
            p.nx, p.ny, p.nz, p.re = 256, 129, 256, 1e5
        else:
            p.nx, p.ny, p.nz, p.re = 128, 65, 128, 1e4
        return p
    raise ValueError(name)


WORKLOAD_DESC = {
    "config1": "plain FP64 DNS, infinite front, 512x257x512 (x,y,z), Re 5000, Ri 1 (M2=N2=f=1), CFL 0.5",
    "config0": "plain FP64 DNS, infinite front, 64x65x64, Re 1000, fixed dt 1e-3",
    "slab": "plain FP64 DNS, infinite front, 512x65x512 (profiling case), Re 5000, Ri 1, CFL 0.5",
    "config2": "LES, finite front (IC 6, width 0.5), 256x129x256, Re 1e5, AMD closure, CFL 0.5",
    "config3": "LES, finite front (IC 6, width 0.5), 128x65x128, Re 1e4, CFL 0.5",
}
