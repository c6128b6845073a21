"""Shared helpers for the parity tests (CPU oracle vs CUDA path)."""
from __future__ import annotations

import math

import numpy as np

from diablo3_b200.grid import create_grid
from diablo3_b200.params import make_params

STATE = (0, 1, 2, 3, 4, 5, 6, 7, 8)   # cu1 cu2 cu3 cp cth cf1 cf2 cf3 cfth
NAMES = ("cu1", "cu2", "cu3", "cp", "cth", "cf1", "cf2", "cf3", "cfth")


def config0_params(**kw):
    """Config 0: infinite-front DNS, 64x65x64, y in [-1, 1] (GRID_TYPE 1),
    Re 1000, Pr 1, N^2 = 1, f = 1, bottom no-slip, top stress-free."""
    base = dict(nx=64, ny=65, nz=64, lx=2 * math.pi, lz=2 * math.pi, ly=2.0,
                re=1000.0, pr=1.0, ri=1.0, ro=1.0, delta=1.0, grav_y=1.0,
                ic_type=4, kick=1e-3, delta_t=1e-3, variable_dt=0,
                u_bc_ymin=0, w_bc_ymin=0, v_bc_ymin=0, th_bc_ymin=1,
                u_bc_ymax=1, w_bc_ymax=1, v_bc_ymax=0, th_bc_ymax=1,
                th_bc_ymin_c1=1.0, th_bc_ymax_c1=1.0)
    base.update(kw)
    return make_params(**base)


def grid_for(p, grid_type: int = 1, cs: float = 1.5):
    return create_grid(p.ny, lz=p.ly, cs=cs, grid_type=grid_type)


def significant(p, a: np.ndarray) -> np.ndarray:
    """Significant spectral entries of a reference complex array
    (kx <= Nkx, packed kz rows 0..2Nkz)."""
    return a[:, : 2 * p.nkz + 1, : p.nkx + 1]


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    na = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return float(d / na) if na > 0 else float(d)


def oracle_state(o, p) -> dict:
    return {fid: significant(p, o.cplx(fid)).copy() for fid in STATE}


def channel_state(ch, p) -> dict:
    st = ch.download_state()
    return {fid: significant(p, st[fid]) for fid in STATE}


def seed_pair(oracle_cls, channel_cls, p, gy, seed=7, noise="gaussian"):
    """Oracle and GPU channel starting from the same spectral state: the IC
    is built once on the CPU (create_flow_chan restatement) and uploaded."""
    from diablo3_b200.ic import initial_fields
    o = oracle_cls(p, gy)
    u1, u2, u3, th = initial_fields(p, gy, seed=seed, noise=noise)
    o.init_from_physical(u1, u2, u3, th)
    ch = channel_cls(p, gy)
    ch.upload_state({fid: o.cplx(fid).copy() for fid in STATE})
    return o, ch


def to_phys(p, c):
    """Packed dealiased spectral planes -> physical planes (numpy irfft2)."""
    nkx, nkz = p.nkx, p.nkz
    full = np.zeros((c.shape[0], p.nz, p.nx // 2 + 1), complex)
    full[:, : nkz + 1, : nkx + 1] = c[:, : nkz + 1, : nkx + 1]
    full[:, p.nz - nkz:, : nkx + 1] = c[:, nkz + 1: 2 * nkz + 1, : nkx + 1]
    return np.fft.irfft2(full, s=(p.nz, p.nx), axes=(1, 2)) * (p.nx * p.nz)


def gradients_at_gy(p, c, met, kx, kz, fid_list=(0, 1, 2)):
    """Velocity gradient G[i][k] = d u_i / d x_k and scalar gradient g[k],
    physical, at GY rows (x/z derivatives and d u2/dy live at GYF rows and
    are interpolated to GY with the dyf weights)."""
    dy, dyf = met["dy"], met["dyf"]
    ny = p.ny
    sl = (slice(None), slice(0, 2 * p.nkz + 1), slice(0, p.nkx + 1))
    ikx = 1j * kx[None, None, :]
    ikz = 1j * kz[None, :, None]
    u = [c[f][sl] for f in (0, 1, 2)]
    th = c[4][sl]

    def ph(a):
        return to_phys(p, a)

    def gyf_to_gy(x):  # rows j of result = GY row j, j = 1..ny
        out = np.zeros_like(x)
        for j in range(1, ny + 1):
            out[j] = (x[j] * dyf[j - 1] + x[j - 1] * dyf[j]) / (2 * dy[j])
        return out

    def ddy_gy(a):  # (a(j) - a(j-1)) / dy(j), GYF field -> GY
        out = np.zeros_like(a)
        out[1:] = (a[1:] - a[:-1]) / dy[1:, None, None]
        return out

    d2dy = np.zeros_like(u[1])
    d2dy[:-1] = (u[1][1:] - u[1][:-1]) / dyf[:-1, None, None]
    G = [[None] * 3 for _ in range(3)]
    G[0][0] = gyf_to_gy(ph(ikx * u[0]))
    G[0][1] = ph(ddy_gy(u[0]))
    G[0][2] = gyf_to_gy(ph(ikz * u[0]))
    G[1][0] = ph(ikx * u[1])
    G[1][1] = gyf_to_gy(ph(d2dy))
    G[1][2] = ph(ikz * u[1])
    G[2][0] = gyf_to_gy(ph(ikx * u[2]))
    G[2][1] = ph(ddy_gy(u[2]))
    G[2][2] = gyf_to_gy(ph(ikz * u[2]))
    g = [gyf_to_gy(ph(ikx * th)), ph(ddy_gy(th)), gyf_to_gy(ph(ikz * th))]
    return np.array(G), np.array(g)
