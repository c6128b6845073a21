"""Initial conditions in physical space, reference layout.

Restates create_flow_chan (for/flow.f90:260-499) and create_th_chan
(for/flow.f90:562-659): velocity and buoyancy for IC types 0-8, then a
seeded perturbation.  The reference draws its noise from Fortran's
``random_number`` with rank-dependent seeds (flow.f90:269-274), which cannot
be reproduced outside that compiler; here the noise comes from numpy's
PCG64 with an explicit seed, either uniform ``kick*(r-0.5)`` like the
reference or Gaussian of standard deviation ``kick`` band-limited to
|kx| < Nx/6, |kz| < Nz/6 (a third of the largest wavenumber).

Arrays are numpy views of the reference layout: real (Nyp+2, Nz+2, Nx+2),
i.e. Fortran u(0:Nx+1, 0:Nz+1, 0:Nyp+1) in memory order.
"""
from __future__ import annotations

import math

import numpy as np

from .grid import metrics
from .params import DbParams


def ref_shape(p: DbParams) -> tuple[int, int, int]:
    return (p.ny + 2, p.nz + 2, p.nx + 2)


def ref_cshape(p: DbParams) -> tuple[int, int, int]:
    return (p.ny + 2, p.nz + 2, p.nxp + 1)


def _noise(p: DbParams, rng: np.random.Generator, kind: str) -> np.ndarray:
    nx, nz, nplanes = p.nx, p.nz, p.ny + 2
    if kind == "uniform":
        return p.kick * (rng.random((nplanes, nz, nx)) - 0.5)
    if kind != "gaussian":
        raise ValueError(kind)
    w = rng.standard_normal((nplanes, nz, nx))
    wh = np.fft.rfft2(w, axes=(1, 2))
    kxi = np.arange(wh.shape[2])
    kzi = np.fft.fftfreq(nz, 1.0 / nz)
    mask = (kxi[None, :] < nx / 6.0) & (np.abs(kzi)[:, None] < nz / 6.0)
    wh *= mask[None, :, :]
    f = np.fft.irfft2(wh, s=(nz, nx), axes=(1, 2))
    std = f.std()
    return p.kick * f / (std if std > 0 else 1.0)


def initial_fields(p: DbParams, gy: np.ndarray, seed: int = 0, noise: str = "gaussian"):
    """Physical u1, u2, u3, th (reference layout, float64) for p.ic_type.

    Planes the reference leaves unset are zero (fresh fftw_alloc memory).
    """
    shp = ref_shape(p)
    u1 = np.zeros(shp)
    u2 = np.zeros(shp)
    u3 = np.zeros(shp)
    th = np.zeros(shp)
    nx, nz, nyp = p.nx, p.nz, p.ny
    m = metrics(np.asarray(gy, dtype=np.float64))
    gyf = m["gyf"]
    gx = (np.arange(nx) * p.lx) / nx
    ic, Ly, Lx, delta = p.ic_type, p.ly, p.lx, p.delta
    ro_inv = 1.0 / p.ro
    ri = p.ri
    X = gx[None, :]

    def setv(arr, j0, j1, val):
        for j in range(j0, j1 + 1):
            v = val(j)
            arr[j, :nz, :nx] = v

    # velocity, for/flow.f90:283-404
    if ic == 0:
        setv(u1, 0, nyp, lambda j: 1.5 * p.ubulk0 * (1.0 - gyf[j] ** 2))
    elif ic == 1:
        setv(u1, 1, nyp, lambda j: -1.5 * p.ubulk0 * gyf[j] ** 2 + 3.0 * p.ubulk0 * gyf[j])
    elif ic == 2:
        setv(u1, 0, nyp, lambda j: gyf[j])
    elif ic == 3:
        setv(u1, 0, nyp, lambda j: math.tanh(gyf[j]))
    elif ic == 4:
        pass
    elif ic == 5:
        t = (math.tanh(0.5 * Lx / delta) - math.tanh(-0.5 * Lx / delta))
        prof = (np.tanh((gx - 0.5 * Lx) / delta) - t / Lx * (gx - 0.5 * Lx)) / (delta * (1.0 / delta - t / Lx))
        setv(u3, 0, nyp, lambda j: np.broadcast_to(prof[None, :], (nz, nx)))
    elif ic == 6:
        def f6(j):
            y = gyf[j] - 0.5 * Ly
            if ri == 0:
                v = y / np.cosh((X - 0.5 * Lx) / delta) ** 2 / math.tanh(0.5 * Lx / delta) - 2.0 * delta / Lx * y
            else:
                s = math.sqrt(ri ** 2 + ro_inv ** 2)
                v = delta * s / ri * np.tanh(((X - 0.5 * Lx) * ro_inv + y * ri) / (delta * s)) - 2.0 * delta / Lx * y
            return np.broadcast_to(v, (nz, nx))
        setv(u3, 0, nyp, f6)
    elif ic == 7:
        def f7(j):
            v = gyf[j] / np.cosh((X - 0.5 * Lx) / delta) ** 2 / math.tanh(0.5 * Lx / delta) - 2.0 * delta / Lx * gyf[j]
            return np.broadcast_to(v, (nz, nx))
        setv(u3, 0, nyp, f7)
    elif ic == 8:
        setv(u3, 0, nyp, lambda j: -2.0 * delta / Lx * (gyf[j] - 0.5 * Ly))
    else:
        raise ValueError(f"unsupported IC_type {ic}")

    # scalar, for/flow.f90:574-651
    if ic == 0:
        setv(th, 1, nyp, lambda j: np.broadcast_to(ri * np.sin(2.0 * math.pi * X / Lx) / (4.0 * math.pi ** 2), (nz, nx)))
    elif ic in (1, 2):
        if p.th_bc_ymin == 0 and p.th_bc_ymax == 0:
            setv(th, 1, nyp, lambda j: ((p.th_bc_ymax_c1 - p.th_bc_ymin_c1) * (gyf[j] + 1.0) / 2.0 + p.th_bc_ymin_c1)
                 if gyf[j] <= 2.0 else p.th_bc_ymax_c1)
        elif p.th_bc_ymin == 1 and p.th_bc_ymax == 1:
            setv(th, 1, nyp, lambda j: p.th_bc_ymin_c1 * gyf[j])
    elif ic == 3:
        setv(th, 1, nyp, lambda j: ri * math.tanh(gyf[j]))
    elif ic in (4, 5):
        th[0, :nz, :nx] = 0.0
        setv(th, 1, nyp, lambda j: ri * (gyf[j] - 0.5 * Ly))
    elif ic in (6, 7, 8):
        def ft(j):
            if ri == 0:
                v = ro_inv * np.tanh((X - 0.5 * Lx) / delta) / math.tanh(0.5 * Lx / delta) + ro_inv * (1.0 - 2.0 / Lx * X)
            else:
                s = math.sqrt(ri ** 2 + ro_inv ** 2)
                v = s * np.tanh(((X - 0.5 * Lx) * ro_inv + (gyf[j] - 0.5 * Ly) * ri) / (delta * s)) \
                    + ro_inv * (1.0 - 2.0 / Lx * X)
            return np.broadcast_to(v, (nz, nx))
        setv(th, 1, nyp, ft)

    # perturbation, for/flow.f90:410-426 (physical-space noise, all planes)
    if p.kick != 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        u1[:, :nz, :nx] += _noise(p, rng, noise)
        u2[:, :nz, :nx] += _noise(p, rng, noise)
        u3[:, :nz, :nx] += _noise(p, rng, noise)
    return u1, u2, u3, th
