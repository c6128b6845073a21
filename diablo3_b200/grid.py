"""Wall-normal grid: the contents of ``grid.h5:/grids/y``.

Restates proc/init/create_grid.m:29-87 (MATLAB, not runnable here): a
stretched G grid of N+1 points is built, the half-points GF are scaled and
shifted so that GF(2) and GF(N+1) sit on the walls, and G(2:N+2) is what the
Fortran reads into GY(1:Nyp+1) (for/domain.f90:466-520).
"""
from __future__ import annotations

import numpy as np


def create_grid(n: int, lz: float = 1.0, cs: float = 1.5, grid_type: int = 3) -> np.ndarray:
    """Return GY(1:n+1) (n = code NY) for the given stretching.

    grid_type 1: tanh, fine at both walls, centred on 0 (closed channel);
    2: cubic, fine in the centre; 3: tanh, fine at both walls, on [0, lz];
    4: tanh, fine at the top (surface boundary layer).
    """
    if n < 2:
        raise ValueError("n must be >= 2")
    # MATLAB arrays are 1-based; index J+1 of G holds point J (J = 1..N+1)
    J = np.arange(1, n + 2, dtype=np.float64)
    if grid_type == 1:
        g = (lz / 2.0) * np.tanh(cs * ((2.0 * (J - 1)) / n - 1.0)) / np.tanh(cs)
    elif grid_type == 2:
        s = (2.0 * (J - 1)) / n - 1.0
        g = (lz / 2.0) * (cs * s ** 3 + s) / (cs + 1)
    elif grid_type == 3:
        g = (lz / 2.0) * np.tanh(cs * ((2.0 * (J - 1)) / n - 1.0)) / np.tanh(cs) + lz / 2.0
    elif grid_type == 4:
        g = lz * np.tanh(cs * ((n - (J - 1)) / n - 1.0)) / np.tanh(cs) + lz
        g = -g
    else:
        raise ValueError("unknown grid type")
    # G(2..N+2) -> g[0..N]; GF(J+1) = (G(J+1)+G(J+2))/2, J = 1..N -> gf[0..N-1]
    gf = (g[:-1] + g[1:]) / 2.0
    gf_lower, gf_upper = gf[0], gf[n - 1]
    g_lower, g_upper = g[0], g[n]
    scale = (g_upper - g_lower) / (gf_upper - gf_lower)
    gf = gf * scale
    g = g * scale
    shift = g_lower - gf[0]
    g = g + shift
    return np.ascontiguousarray(g)


def metrics(gy: np.ndarray) -> dict:
    """GY, GYF, DY, DYF on 0..Nyp+1 as create_grid_chan/ReadGridHDF5 build
    them (for/domain.f90:276-300, 538-565); index 0 of GY is never set by
    the reference and is left 0."""
    nyp = len(gy) - 1
    out_gy = np.zeros(nyp + 2)
    out_gy[1:] = gy
    gyf = np.zeros(nyp + 2)
    gyf[1:nyp + 1] = 0.5 * (out_gy[1:nyp + 1] + out_gy[2:nyp + 2])
    gyf[0] = 2.0 * gyf[1] - gyf[2]
    gyf[nyp + 1] = 2.0 * gyf[nyp] - gyf[nyp - 1]
    dy = np.zeros(nyp + 2)
    dy[1:] = gyf[1:] - gyf[:-1]
    dyf = np.zeros(nyp + 2)
    dyf[1:nyp + 1] = out_gy[2:nyp + 2] - out_gy[1:nyp + 1]
    dyf[0] = dyf[1]
    dyf[nyp + 1] = dyf[nyp]
    return {"gy": out_gy, "gyf": gyf, "dy": dy, "dyf": dyf}
