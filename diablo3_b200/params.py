"""Run parameters: the ``db_params`` struct of include/diablo_b200.h.

The fields are the contents of DIABLO's ``input.dat`` / ``input_chan.dat``
(version 3.4) and ``grid_def.all``, as the Fortran reads them in
``init_parameters`` / ``input_chan`` (for/parameters.f90:84-121, 202-250).
Coordinates follow the Fortran code: y is wall-normal.  The input files are
written with z vertical, so this parser applies the same swaps the reference
does (for/make_headers:17-21, for/parameters.f90:101, 227, 232-242).
"""
from __future__ import annotations

import ctypes
import math
import os
import re

_FIELDS = [
    ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("n_th", ctypes.c_int32),
    ("re", ctypes.c_double), ("beta", ctypes.c_double), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
    ("lz", ctypes.c_double), ("nu_v_scale", ctypes.c_double),
    ("delta_t", ctypes.c_double), ("cfl", ctypes.c_double),
    ("variable_dt", ctypes.c_int32), ("update_dt", ctypes.c_int32),
    ("ri", ctypes.c_double), ("pr", ctypes.c_double),
    ("use_les", ctypes.c_int32), ("create_new_flow", ctypes.c_int32),
    ("time_ad_meth", ctypes.c_int32), ("les_model_type", ctypes.c_int32),
    ("ic_type", ctypes.c_int32), ("physical_noise", ctypes.c_int32),
    ("kick", ctypes.c_double), ("ro", ctypes.c_double), ("delta", ctypes.c_double),
    ("grav_x", ctypes.c_double), ("grav_y", ctypes.c_double), ("grav_z", ctypes.c_double),
    ("f_type", ctypes.c_int32), ("flavor_front", ctypes.c_int32),
    ("ubulk0", ctypes.c_double), ("px0", ctypes.c_double), ("omega0", ctypes.c_double),
    ("amp_omega0", ctypes.c_double), ("force_start", ctypes.c_double),
    ("u_bc_ymin", ctypes.c_int32), ("v_bc_ymin", ctypes.c_int32), ("w_bc_ymin", ctypes.c_int32),
    ("th_bc_ymin", ctypes.c_int32),
    ("u_bc_ymax", ctypes.c_int32), ("v_bc_ymax", ctypes.c_int32), ("w_bc_ymax", ctypes.c_int32),
    ("th_bc_ymax", ctypes.c_int32),
    ("u_bc_ymin_c1", ctypes.c_double), ("v_bc_ymin_c1", ctypes.c_double),
    ("w_bc_ymin_c1", ctypes.c_double), ("th_bc_ymin_c1", ctypes.c_double),
    ("u_bc_ymax_c1", ctypes.c_double), ("v_bc_ymax_c1", ctypes.c_double),
    ("w_bc_ymax_c1", ctypes.c_double), ("th_bc_ymax_c1", ctypes.c_double),
    ("dthdx_override", ctypes.c_double),
    ("time_limit", ctypes.c_double), ("save_stats_dt", ctypes.c_double), ("save_flow_dt", ctypes.c_double),
    ("precision", ctypes.c_int32), ("reserved_i", ctypes.c_int32 * 7),
]


class DbParams(ctypes.Structure):
    """ctypes mirror of ``db_params`` (include/diablo_b200.h)."""

    _fields_ = _FIELDS

    def copy(self) -> "DbParams":
        out = DbParams()
        ctypes.memmove(ctypes.byref(out), ctypes.byref(self), ctypes.sizeof(DbParams))
        return out

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in _FIELDS if name != "reserved_i"}

    # derived sizes of the reference layout (for/domain.f90:22-32)
    @property
    def nxp(self) -> int:
        return self.nx // 2

    @property
    def nkx(self) -> int:
        return self.nx // 3

    @property
    def nkz(self) -> int:
        return self.nz // 3

    @property
    def ref_array_len(self) -> int:
        """Doubles in one reference-layout array (0:Nx+1, 0:Nz+1, 0:Nyp+1)."""
        return (self.nx + 2) * (self.nz + 2) * (self.ny + 2)


def make_params(**kw) -> DbParams:
    """Parameters with the reference's defaults for an infinite-front DNS
    (IC 4, rotating, stratified, one scalar), overridden by ``kw``."""
    p = DbParams()
    defaults = dict(
        nx=64, ny=65, nz=64, n_th=1,
        re=1000.0, beta=1.0, lx=2 * math.pi, ly=2.0, lz=2 * math.pi, nu_v_scale=1.0,
        delta_t=1e-3, cfl=0.5, variable_dt=0, update_dt=1,
        ri=1.0, pr=1.0, use_les=0, create_new_flow=1,
        time_ad_meth=1, les_model_type=5, ic_type=4, physical_noise=1,
        kick=1e-3, ro=1.0, delta=1.0, grav_x=0.0, grav_y=1.0, grav_z=0.0,
        f_type=3, flavor_front=1,
        ubulk0=0.0, px0=0.0, omega0=0.0, amp_omega0=0.0, force_start=0.0,
        u_bc_ymin=0, v_bc_ymin=0, w_bc_ymin=0, th_bc_ymin=1,
        u_bc_ymax=1, v_bc_ymax=0, w_bc_ymax=1, th_bc_ymax=1,
        u_bc_ymin_c1=0.0, v_bc_ymin_c1=0.0, w_bc_ymin_c1=0.0, th_bc_ymin_c1=1.0,
        u_bc_ymax_c1=0.0, v_bc_ymax_c1=0.0, w_bc_ymax_c1=0.0, th_bc_ymax_c1=1.0,
        dthdx_override=float("nan"),
        time_limit=1e30, save_stats_dt=1e30, save_flow_dt=1e30,
        precision=0,
    )
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(p, k, v)
    return p


# ---------------------------------------------------------------------------
# reference input files

def _data_lines(path: str) -> list[str]:
    with open(path) as f:
        return f.read().splitlines()


def _tokens(line: str) -> list[str]:
    # Fortran list-directed read: blanks/commas separate, quotes delimit strings
    return [t for t in re.findall(r"'[^']*'|\"[^\"]*\"|[^\s,]+", line)]


def _num(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def _logical(tok: str) -> int:
    t = tok.strip(".").upper()
    if t in ("TRUE", "T"):
        return 1
    if t in ("FALSE", "F"):
        return 0
    raise ValueError(f"not a Fortran logical: {tok}")


class InputError(ValueError):
    pass


def read_grid_def(path: str) -> tuple[int, int, int, int]:
    """grid_def.all -> code (Nx, NY, Nz, N_th).  The file writes the
    wall-normal size as "Nz"; make_headers swaps it to code NY
    (for/make_headers:11-21)."""
    vals = {}
    for line in _data_lines(path):
        m = re.match(r"\s*(\w+)\s*=\s*(\d+)", line)
        if m:
            vals[m.group(1).lower()] = int(m.group(2))
    try:
        return vals["nx"], vals["nz"], vals["ny"], vals["nth"]
    except KeyError as e:
        raise InputError(f"{path}: missing {e}") from None


def read_inputs(run_dir: str, version_check: bool = True) -> DbParams:
    """Parse ``input.dat``, ``input_chan.dat`` and ``grid_def.all`` of a run
    directory exactly as init_parameters/input_chan do (comment lines are
    skipped by position; version 3.4 is required, for/parameters.f90:96,211).
    A missing file, a file that ends early or a value that does not read as
    its type raises InputError (the reference stops there too).
    """
    try:
        return _read_inputs(run_dir, version_check)
    except InputError:
        raise
    except FileNotFoundError as e:
        raise InputError(f"{run_dir}: missing {os.path.basename(e.filename or '?')}") from None
    except StopIteration:
        raise InputError(f"{run_dir}: an input file ends before all its entries") from None
    except (ValueError, IndexError) as e:
        raise InputError(f"{run_dir}: unreadable entry ({e})") from None


def _read_inputs(run_dir: str, version_check: bool) -> DbParams:
    nx, ny, nz, nth = read_grid_def(os.path.join(run_dir, "grid_def.all"))
    L = _data_lines(os.path.join(run_dir, "input.dat"))
    # for/parameters.f90:91-121: 4 comment lines, then data/comment pairs
    it = iter(L)
    for _ in range(4):
        next(it)
    flavor, version = _tokens(next(it))[:2]
    if version_check and abs(_num(version) - 3.4) > 1e-6:
        raise InputError("Wrong input data format.")
    next(it)
    use_mpi, use_les = map(_logical, _tokens(next(it))[:2])
    next(it)
    re_, beta, lx, lz, ly = map(_num, _tokens(next(it))[:5])  # LX LY LZ -> Lx, Lz, Ly
    next(it)
    nu_v_scale = _num(_tokens(next(it))[0])
    next(it)
    t = _tokens(next(it))
    num_per_dir, create_new_flow = int(_num(t[0])), _logical(t[1])
    next(it)
    t = _tokens(next(it))
    wall_time_limit, time_limit, delta_t = map(_num, t[:3])
    reset_time, variable_dt = _logical(t[3]), _logical(t[4])
    cfl, update_dt = _num(t[5]), int(_num(t[6]))
    next(it)
    t = _tokens(next(it))
    save_flow_dt, save_stats_dt = _num(t[1]), _num(t[2])
    next(it)
    ri, pr = 0.0, 1.0
    for _n in range(nth):
        next(it)
        next(it)
        next(it)
        next(it)
        next(it)
        ri, pr = map(_num, _tokens(next(it))[:2])
    if num_per_dir != 2:
        raise InputError("only the channel (NUM_PER_DIR = 2) exists in diablo3")

    C = iter(_data_lines(os.path.join(run_dir, "input_chan.dat")))
    for _ in range(4):
        next(C)
    cversion = _num(_tokens(next(C))[0])
    if version_check and abs(cversion - 3.4) > 1e-6:
        raise InputError("Wrong input data format input_chan")
    next(C)
    time_ad_meth = int(_num(_tokens(next(C))[0]))
    next(C)
    les_model_type = int(_num(_tokens(next(C))[0]))
    next(C)
    t = _tokens(next(C))
    ic_type, kick, physical_noise = int(_num(t[0])), _num(t[1]), _logical(t[2])
    next(C)
    ro = _num(_tokens(next(C))[0])
    next(C)
    delta = _num(_tokens(next(C))[0])
    next(C)
    gx, gz, gy = map(_num, _tokens(next(C))[:3])  # GRAV_X, GRAV_Y, GRAV_Z -> x, z, y
    next(C)
    t = _tokens(next(C))
    f_type = int(_num(t[0]))
    ubulk0, px0, omega0, amp_omega0 = map(_num, t[1:5])
    force_start = _num(t[5]) if len(t) > 5 else 0.0
    next(C)

    def bc_pair():
        next(C)
        tt = _tokens(next(C))
        return int(_num(tt[0])), _num(tt[1])

    u_min = bc_pair(); w_min = bc_pair(); v_min = bc_pair()   # u, w, v order (parameters.f90:232-242)
    u_max = bc_pair(); w_max = bc_pair(); v_max = bc_pair()
    next(C)
    th_min = th_max = (1, 0.0)
    for _n in range(nth):
        th_min = bc_pair()
        th_max = bc_pair()

    return make_params(
        nx=nx, ny=ny, nz=nz, n_th=nth, re=re_, beta=beta, lx=lx, ly=ly, lz=lz,
        nu_v_scale=nu_v_scale, delta_t=delta_t, cfl=cfl, variable_dt=variable_dt,
        update_dt=update_dt, ri=ri, pr=pr, use_les=use_les, create_new_flow=create_new_flow,
        time_ad_meth=time_ad_meth, les_model_type=les_model_type, ic_type=ic_type,
        physical_noise=physical_noise, kick=kick, ro=ro, delta=delta,
        grav_x=gx, grav_y=gy, grav_z=gz, f_type=f_type,
        flavor_front=1 if flavor.strip("'\"").strip() == "Front" else 0,
        ubulk0=ubulk0, px0=px0, omega0=omega0, amp_omega0=amp_omega0, force_start=force_start,
        u_bc_ymin=u_min[0], u_bc_ymin_c1=u_min[1], w_bc_ymin=w_min[0], w_bc_ymin_c1=w_min[1],
        v_bc_ymin=v_min[0], v_bc_ymin_c1=v_min[1],
        u_bc_ymax=u_max[0], u_bc_ymax_c1=u_max[1], w_bc_ymax=w_max[0], w_bc_ymax_c1=w_max[1],
        v_bc_ymax=v_max[0], v_bc_ymax_c1=v_max[1],
        th_bc_ymin=th_min[0], th_bc_ymin_c1=th_min[1], th_bc_ymax=th_max[0], th_bc_ymax_c1=th_max[1],
        time_limit=time_limit, save_stats_dt=save_stats_dt, save_flow_dt=save_flow_dt,
    )
