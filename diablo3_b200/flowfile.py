"""Flow files in the reference's restart layout (WriteHDF5 / ReadHDF5,
for/phdf5.f90:918-1197, 1204-1456), for exchanging state with a run of the
reference.

A file holds what the reference's ``out.NNNNNN.h5`` / ``end.h5`` hold:
  attributes  Resolution = [Nx, Nyp, Nz], Date (text)
  /Timestep   attributes Time, Save_Flow_Time, Save_Stats_Time,
              Save_Movie_Time, Time_Step; datasets
                U    u1 at the GYF points 1..Nyp
                W    u2 moved to the GYF points (g2gf, for/tools.f90:299-318)
                V    u3
                TH1  the buoyancy
                P    the pressure (when saved)
              each (Nx, Nyp, Nz) in Fortran order (swapzy, tools.f90:216-233),
              i.e. a C array [Nz][Nyp][Nx] of float64.
There is no HDF5 library here, so the container is this library's own: the
8-byte magic ``DIABLOF1``, a little-endian uint64 header length, a JSON
header with the attributes and the dataset list (name, shape, CRC-32), then
the datasets back to back (little-endian float64).  Each dataset maps one
to one onto the HDF5 dataset of the same path.

Reading follows ReadHDF5: the resolution must match (phdf5.f90:1293-1303),
each dataset lands on the planes 1..Nyp of a zeroed array (swapyz), W goes
back to the GY points (gf2g, tools.f90:255-297), the fields go to Fourier
space, and without P the pressure comes from poisson_p_chan
(phdf5.f90:1452-1454).  The RK history cf is not in the file (zero; the
first substep does not read it).  The transforms here are numpy FP64 FFTs
with the reference's normalisation (forward / (Nx Nz), unnormalised inverse)
and 2/3 truncation, whatever the channel's precision.

The reference's writer leaves u2's wall rows at -u2(2), -u2(Nyp) in memory
(gf2g after g2gf); this writer does not change the channel's state.
"""
from __future__ import annotations

import json
import struct
import time as _time
import zlib

import numpy as np

from . import lib as _L

MAGIC = b"DIABLOF1"


class FlowFileError(ValueError):
    """A flow file that does not fit the run (or is not one)."""


# ---------------------------------------------------------------------------
# the reference's transforms and staggering on host arrays

def to_physical(p, c: np.ndarray) -> np.ndarray:
    """Reference-layout spectral array (planes, Nz+2, Nxp+1) -> physical
    planes (planes, Nz, Nx) (fft_xz_to_physical)."""
    nkx, nkz = p.nx // 3, p.nz // 3
    full = np.zeros((c.shape[0], p.nz, p.nx // 2 + 1), complex)
    full[:, : nkz + 1, : nkx + 1] = c[:, : nkz + 1, : nkx + 1]
    full[:, p.nz - nkz:, : nkx + 1] = c[:, nkz + 1: 2 * nkz + 1, : nkx + 1]
    return np.fft.irfft2(full, s=(p.nz, p.nx), axes=(1, 2)) * (p.nx * p.nz)


def to_fourier(p, u: np.ndarray) -> np.ndarray:
    """Physical planes (planes, Nz, Nx) -> reference-layout spectral array
    (planes, Nz+2, Nxp+1), retained modes only (fft_xz_to_fourier)."""
    nkx, nkz = p.nx // 3, p.nz // 3
    full = np.fft.rfft2(u, axes=(1, 2)) / (p.nx * p.nz)
    c = np.zeros((u.shape[0], p.nz + 2, p.nx // 2 + 1), complex)
    c[:, : nkz + 1, : nkx + 1] = full[:, : nkz + 1, : nkx + 1]
    c[:, nkz + 1: 2 * nkz + 1, : nkx + 1] = full[:, p.nz - nkz:, : nkx + 1]
    return c


def g2gf(v: np.ndarray, nyp: int) -> np.ndarray:
    """u2 at the GY points -> the GYF points 1..Nyp (tools.f90:299-318, one
    rank in y); v: planes 0..Nyp+1."""
    w = v.copy()
    w[1] = w[2]
    w[nyp + 1] = w[nyp]
    out = w.copy()
    out[1: nyp + 1] = 0.5 * (w[1: nyp + 1] + w[2: nyp + 2])
    return out


def gf2g(v: np.ndarray, nyp: int) -> np.ndarray:
    """The inverse move (tools.f90:255-297, one rank in y), then the wall
    rows that give zero mass flux."""
    w = v.copy()
    w[nyp + 1] = w[nyp]
    for y in range(nyp, 0, -1):
        w[y] = 2 * w[y] - w[y + 1]
    w[1] = -w[2]
    w[nyp + 1] = -w[nyp]
    return w


def _swapzy(u: np.ndarray, nyp: int) -> np.ndarray:
    # planes 1..Nyp of (planes, Nz, Nx) -> C array [Nz][Nyp][Nx]
    return np.ascontiguousarray(np.transpose(u[1: nyp + 1], (1, 0, 2)))


def _swapyz(a: np.ndarray, p) -> np.ndarray:
    u = np.zeros((p.ny + 2, p.nz, p.nx))
    u[1: p.ny + 1] = np.transpose(a, (1, 0, 2))
    return u


# ---------------------------------------------------------------------------

def write_flow(ch, path: str, save_pressure: bool = True, save_flow_time: float | None = None,
               save_stats_time: float | None = None, save_movie_time: float | None = None) -> None:
    """WriteHDF5's content of the channel's current state into `path`."""
    p = ch.p
    st = ch.status()
    state = ch.download_state()
    u1 = to_physical(p, state[_L.CU1])
    u2 = g2gf(to_physical(p, state[_L.CU2]), p.ny)
    u3 = to_physical(p, state[_L.CU3])
    th = to_physical(p, state[_L.CTH])
    sets = [("U", u1), ("W", u2), ("V", u3), ("TH1", th)]
    if save_pressure:
        sets.append(("P", to_physical(p, state[_L.CP])))
    t = st.time
    hdr = {
        "Resolution": [p.nx, p.ny, p.nz],
        "Date": _time.strftime("%Y-%m-%d %H:%M:%S"),
        "Timestep": {
            "Time": t,
            "Save_Flow_Time": t + p.save_flow_dt if save_flow_time is None else save_flow_time,
            "Save_Stats_Time": t + p.save_stats_dt if save_stats_time is None else save_stats_time,
            "Save_Movie_Time": t + p.save_stats_dt if save_movie_time is None else save_movie_time,
            "Time_Step": int(st.time_step),
        },
        "datasets": [],
    }
    blobs = []
    for name, u in sets:
        b = _swapzy(u, p.ny).astype("<f8").tobytes()
        hdr["datasets"].append({"name": name, "shape": [p.nz, p.ny, p.nx], "crc32": zlib.crc32(b)})
        blobs.append(b)
    h = json.dumps(hdr).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(h)))
        f.write(h)
        for b in blobs:
            f.write(b)


def read_file(path: str):
    """(header, {dataset: [Nz][Nyp][Nx] array}) of a flow file."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise FlowFileError(f"{path}: not a flow file")
        raw = f.read(8)
        if len(raw) != 8:
            raise FlowFileError(f"{path}: truncated in the header")
        (n,) = struct.unpack("<Q", raw)
        h = f.read(n)
        if len(h) != n:
            raise FlowFileError(f"{path}: truncated in the header")
        try:
            hdr = json.loads(h.decode())
            entries = hdr["datasets"]
            hdr["Resolution"], hdr["Timestep"]
        except (UnicodeDecodeError, json.JSONDecodeError, KeyError, TypeError) as e:
            raise FlowFileError(f"{path}: bad header ({e})") from None
        out = {}
        for e in entries:
            shape = [int(x) for x in e["shape"]]
            cnt = int(np.prod(shape)) * 8
            b = f.read(cnt)
            if len(b) != cnt:
                raise FlowFileError(f"{path}: truncated at {e['name']}")
            if zlib.crc32(b) != e.get("crc32"):
                raise FlowFileError(f"{path}: {e['name']} does not match its CRC-32")
            out[e["name"]] = np.frombuffer(b, dtype="<f8").reshape(shape).astype(np.float64)
    return hdr, out


def read_flow(path: str, p, gy, stream: int | None = None):
    """A Channel started from a flow file as ReadHDF5 starts the reference."""
    from .channel import Channel
    hdr, d = read_file(path)
    if list(hdr["Resolution"]) != [p.nx, p.ny, p.nz]:
        raise FlowFileError(f"{path}: resolution {hdr['Resolution']} does not match the run "
                            f"({p.nx}, {p.ny}, {p.nz})")
    for name in ("U", "W", "V", "TH1"):
        if name not in d:
            raise FlowFileError(f"{path}: no dataset {name}")
    u1 = _swapyz(d["U"], p)
    u2 = gf2g(_swapyz(d["W"], p), p.ny)
    u3 = _swapyz(d["V"], p)
    th = _swapyz(d["TH1"], p)
    ch = Channel(p, gy, stream=stream)
    spec = {_L.CU1: to_fourier(p, u1), _L.CU2: to_fourier(p, u2), _L.CU3: to_fourier(p, u3),
            _L.CTH: to_fourier(p, th)}
    if "P" in d:
        spec[_L.CP] = to_fourier(p, _swapyz(d["P"], p))
    ch.upload_state(spec)
    ts = hdr["Timestep"]
    ch.set_clock(float(ts["Time"]), int(ts["Time_Step"]), float(ts["Save_Stats_Time"]), float(ts["Save_Flow_Time"]))
    if p.variable_dt:   # ReadHDF5 calls courant before going back to Fourier space
        ch.courant()
    if "P" not in d:
        ch.poisson_p_chan()
    return ch


__all__ = ["write_flow", "read_flow", "read_file", "to_physical", "to_fourier", "g2gf", "gf2g",
           "FlowFileError", "MAGIC"]
