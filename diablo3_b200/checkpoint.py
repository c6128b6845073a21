"""Checkpoint / restart of a channel (the role of save_flow / read_flow,
for/phdf5.f90:918-1456, without an HDF5 library).

A checkpoint holds the exact device state, so a restarted run continues
bit-identically: the nine spectral fields of the reference layout
(cu1, cu2, cu3, cp, cth, cf1, cf2, cf3, cfth; complex128), nu_t and
kappa_t with LES, the run parameters with dt set to the current step, the
y-grid and the clock.  (The reference's restart file holds physical U, V,
W, TH with u2 interpolated to GYF, tools.f90:255-322, and rebuilds the
pressure with poisson_p_chan; keeping the spectral state and cf avoids
both approximations.)

File layout: 8-byte magic ``DIABLOB3``, little-endian uint64 length of a
UTF-8 JSON header, the header, then the arrays back to back in the order
the header's ``arrays`` list gives (dtype, shape and the CRC-32 of the
bytes per entry).  Reading checks all of it: a file that is not a
checkpoint, a header that does not parse or lacks an entry, an array that
is cut short or whose bytes changed raise CheckpointError, before any
state reaches a device.
"""
from __future__ import annotations

import json
import math
import struct
import zlib

import numpy as np

from . import lib as _L

MAGIC = b"DIABLOB3"
VERSION = 2          # 2: CRC-32 per array; version 1 files (no CRC) are still read


class CheckpointError(ValueError):
    """A checkpoint file that cannot be restarted from."""


def _clean(v):
    if isinstance(v, float) and math.isnan(v):
        return "nan"
    return v


def write(path: str, hdr: dict, arrays) -> None:
    """Write a header dict (without the array list) and [(name, array)]."""
    hdr = dict(hdr)
    hdr["version"] = VERSION
    hdr["arrays"] = []
    blobs = []
    for n, a in arrays:
        b = np.ascontiguousarray(a).tobytes()
        hdr["arrays"].append({"name": n, "dtype": str(a.dtype), "shape": list(a.shape), "crc32": zlib.crc32(b)})
        blobs.append(b)
    h = json.dumps(hdr).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(h)))
        f.write(h)
        for b in blobs:
            f.write(b)


def save(ch, path: str) -> None:
    """Write the state, clock and parameters of a Channel to `path`."""
    st = ch.status()
    state = ch.download_state()
    arrays = [(f"spec{fid}", state[fid]) for fid in _L.STATE_FIELDS]
    if ch.p.use_les:
        arrays += [("nu_t", ch.download_field(_L.NU_T)), ("kappa_t", ch.download_field(_L.KAPPA_T))]
    params = {k: _clean(v) for k, v in ch.p.as_dict().items()}
    params["delta_t"] = st.delta_t
    write(path, {"params": params, "gy": [float(x) for x in ch.gy], "time": st.time,
                 "time_step": int(st.time_step)}, arrays)


def read(path: str):
    """(header, {name: array}) of a checkpoint file; CheckpointError when it
    is not a complete, unchanged checkpoint of this library."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise CheckpointError(f"{path}: not a checkpoint of this library")
        raw = f.read(8)
        if len(raw) != 8:
            raise CheckpointError(f"{path}: truncated in the header")
        (n,) = struct.unpack("<Q", raw)
        h = f.read(n)
        if len(h) != n:
            raise CheckpointError(f"{path}: truncated in the header")
        try:
            hdr = json.loads(h.decode())
            version = hdr.get("version")
            entries = hdr["arrays"]
            for k in ("params", "gy", "time", "time_step"):
                hdr[k]
        except (UnicodeDecodeError, json.JSONDecodeError, KeyError, AttributeError, TypeError) as e:
            raise CheckpointError(f"{path}: bad header ({e})") from None
        if version not in (1, VERSION):
            raise CheckpointError(f"{path}: checkpoint version {version} (expected {VERSION})")
        arrays = {}
        for e in entries:
            try:
                dt = np.dtype(e["dtype"])
                shape = [int(x) for x in e["shape"]]
                name = e["name"]
            except (KeyError, TypeError, ValueError) as err:
                raise CheckpointError(f"{path}: bad array entry ({err})") from None
            cnt = int(np.prod(shape))
            buf = f.read(cnt * dt.itemsize)
            if len(buf) != cnt * dt.itemsize:
                raise CheckpointError(f"{path}: truncated at {name}")
            if version >= 2 and zlib.crc32(buf) != e.get("crc32"):
                raise CheckpointError(f"{path}: {name} does not match its CRC-32 (the file changed)")
            arrays[name] = np.frombuffer(buf, dtype=dt).reshape(shape).copy()
        if f.read(1):
            raise CheckpointError(f"{path}: bytes after the last array")
    return hdr, arrays


def load(path: str, stream: int | None = None, **overrides):
    """A new Channel continuing the checkpointed run (parameters from the
    file, optionally overridden, e.g. ``precision=1`` to continue an FP64
    run on the mixed path)."""
    from .channel import Channel
    from .params import make_params
    hdr, arrays = read(path)
    pd = {k: (float("nan") if v == "nan" else v) for k, v in hdr["params"].items()}
    pd.update(overrides)
    p = make_params(**pd)
    ch = Channel(p, np.asarray(hdr["gy"], np.float64), stream=stream)
    ch.upload_state({fid: arrays[f"spec{fid}"] for fid in _L.STATE_FIELDS})
    if p.use_les and "nu_t" in arrays:
        ch.upload_field(_L.NU_T, arrays["nu_t"])
        ch.upload_field(_L.KAPPA_T, arrays["kappa_t"])
    t = hdr["time"]
    ch.set_clock(t, hdr["time_step"], t + p.save_stats_dt, t + p.save_flow_dt)
    return ch


__all__ = ["save", "write", "read", "load", "MAGIC", "CheckpointError"]
