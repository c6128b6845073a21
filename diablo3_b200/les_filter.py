"""Resolved (DNS) state -> LES grid, and the horizontal-mean profiles the
learned closure is judged on.

The LES grid has Nx/f, Nz/f points and the same y-stretching with fewer
cells.  Horizontally a field is box-filtered over f x f points (uniform
spacing; box averages of f consecutive points).  In y, a cell-centred
field (u1, u3, th at GYF) on LES cell k is the dyf-weighted mean of the
fine cells whose centres lie between the LES faces GY(k), GY(k+1); the
face field u2 (at GY) is interpolated linearly to the LES faces.  A
horizontal mean is unchanged by the horizontal box filter, so the filtered
DNS mean profile is the same y-filter applied to the fine horizontal means
(the kx = kz = 0 Fourier mode of the state).
"""
from __future__ import annotations

import numpy as np

from . import lib as _L
from .grid import metrics


def _cell_weights(gy_f: np.ndarray, gy_c: np.ndarray) -> np.ndarray:
    """W[kc, jf]: weight of fine cell jf (GYF) in LES cell kc, rows summing
    to 1 for every LES cell that holds a fine cell centre."""
    mf, mc = metrics(np.asarray(gy_f, np.float64)), metrics(np.asarray(gy_c, np.float64))
    nf, nc = len(mf["gyf"]), len(mc["gyf"])
    W = np.zeros((nc, nf))
    nyp_f, nyp_c = nf - 2, nc - 2
    for kc in range(1, nyp_c + 1):
        lo, hi = mc["gy"][kc], mc["gy"][kc + 1]
        for jf in range(1, nyp_f + 1):
            if lo <= mf["gyf"][jf] < hi or (kc == nyp_c and mf["gyf"][jf] == hi):
                W[kc, jf] = mf["dyf"][jf]
    # ghost cells: the nearest interior fine cell
    W[0, 1] = 1.0
    W[nyp_c + 1, nyp_f] = 1.0
    s = W.sum(axis=1, keepdims=True)
    return W / np.where(s > 0, s, 1.0)


def _face_interp(gy_f: np.ndarray, gy_c: np.ndarray) -> np.ndarray:
    """I[kc, jf]: linear interpolation of a GY-face field to the LES faces."""
    mf, mc = metrics(np.asarray(gy_f, np.float64)), metrics(np.asarray(gy_c, np.float64))
    nf, nc = len(mf["gy"]), len(mc["gy"])
    I = np.zeros((nc, nf))
    yf = mf["gy"][1:]
    for kc in range(1, nc):
        y = mc["gy"][kc]
        i = int(np.clip(np.searchsorted(yf, y) - 1, 0, len(yf) - 2))
        t = (y - yf[i]) / (yf[i + 1] - yf[i])
        I[kc, i + 1] = 1.0 - t
        I[kc, i + 2] = t
    I[0, 1] = 1.0
    return I


def _hbox(a: np.ndarray, nz: int, nx: int, f: int) -> np.ndarray:
    """Box average over f x f points of the [j][z][x] planes (physical part
    of a reference-layout array)."""
    b = a[:, :nz, :nx]
    return b.reshape(b.shape[0], nz // f, f, nx // f, f).mean(axis=(2, 4))


def filter_state_to_les(ch_fine, p_les, gy_les, f: int = 4):
    """Physical u1, u2, u3, th on the LES grid (reference layout arrays of
    the LES shape) from the state of a resolved channel."""
    pf = ch_fine.p
    st = ch_fine.download_state()
    W = _cell_weights(ch_fine.gy, gy_les)
    I = _face_interp(ch_fine.gy, gy_les)
    out = []
    for fid in (_L.CU1, _L.CU2, _L.CU3, _L.CTH):
        phys = ch_fine.fft_xz_to_physical(st[fid].copy())
        box = _hbox(phys, pf.nz, pf.nx, f)                       # [jf][zc][xc]
        M = I if fid == _L.CU2 else W
        coarse = np.tensordot(M, box, axes=(1, 0))              # [jc][zc][xc]
        arr = np.zeros((p_les.ny + 2, p_les.nz + 2, p_les.nx + 2))
        arr[:, : p_les.nz, : p_les.nx] = coarse
        out.append(arr)
    return tuple(out)


def mean_profiles(ch) -> dict:
    """Horizontal means of u1, u3, th at the GYF rows 0..Nyp+1 of a channel
    (the kx = kz = 0 mode of its spectral state)."""
    st = ch.download_state()
    return {name: st[fid][:, 0, 0].real.copy() for name, fid in (("u1", _L.CU1), ("u3", _L.CU3), ("th", _L.CTH))}


def filtered_mean_profiles(ch_fine, gy_les) -> dict:
    """Mean profiles of the resolved state filtered onto the LES grid."""
    W = _cell_weights(ch_fine.gy, gy_les)
    return {k: W @ v for k, v in mean_profiles(ch_fine).items()}


def profile_errors(les: dict, ref: dict, rows: slice) -> dict:
    """Relative L2 error of each mean profile over the given LES rows."""
    return {k: float(np.linalg.norm(les[k][rows] - ref[k][rows]) / max(np.linalg.norm(ref[k][rows]), 1e-300))
            for k in ref}


def evolution_errors(les: dict, les0: dict, ref: dict, ref0: dict, rows: slice) -> dict:
    """Relative L2 error of the change of each mean profile since a common
    start (les0, ref0): what the closure and the resolved dynamics did to
    the profile, without the part both inherit from the initial state."""
    out = {}
    for k in ref:
        d_ref = ref[k][rows] - ref0[k][rows]
        d_les = les[k][rows] - les0[k][rows]
        out[k] = float(np.linalg.norm(d_les - d_ref) / max(np.linalg.norm(d_ref), 1e-300))
    return out


__all__ = ["filter_state_to_les", "mean_profiles", "filtered_mean_profiles", "profile_errors", "evolution_errors"]
