"""Algorithmic HBM bytes of the substep, per stage (one place).

Units per wall-normal plane set (Nyp+2 planes, ghosts included):
  P  = Nx * Nz * 8 B             one physical field (4 B on the mixed path)
  Xh = (Nkx+1) * Nz * 16 B       one x-transformed, not z-transformed field
                                 (8 B per complex on the mixed path)
  S  = (Nkx+1) * (2Nkz+1) * 16 B one dealiased packed spectral field (always FP64)
Each stage counts the bytes it must read and write once when everything
inside it is fused (neighbour planes in y are L2 hits).

Without eddy viscosity (no LES) the CN matrices are the same in every
column, so the implicit solves run on the retained Fourier modes and the
transforms of cr and of the new state drop out:
  inv_z      4 S  -> 4 Xh           cu1, cu2, cu3, cth to x-half
  inv_x      4 Xh -> 4 P            to physical u1, u2, u3, th
  products   4 P  -> 8 Xh           11 products + x-FFT, x-derivatives folded
  zpass_rhs  8 Xh -> 8 S            z-FFT of the 8 product fields (FP64:
                                    Z(N_e), Z(M_e); the mixed path writes
                                    the 4 terms NL_e = Z(N_e) + i kz Z(M_e):
                                    8 Xh -> 4 S)
  thomas     8 S + 9 S -> 8 S       spectral RHS joined with the CN solves:
                                    Z(N), Z(M) (mixed: NL, 4 S), cu1, cu2,
                                    cu3, cth, cp, cf_old in; cf and the new cu
                                    out (the forward sweep's y values are a
                                    round trip that is not counted)
  courant    (3 S + 6 Xh) / 3       u1..u3 inverse z, then their inverse x
                                    reducing the CFL terms (no physical
                                    store), on the third substep only
  rem_div    4 S  -> 4 S            cu1, cu2, cu3, cp in and out
At 512x257x512 this is ~46 P, i.e. ~369 B per grid point and substep for
FP64 (a z-pass fused with the RHS would save the 8 S of Z(N), Z(M): its
FP64 form spills and ran slower).

The reference's own sequence (cr to physical space, physical CN solves,
new state back to Fourier space; the LES substep still runs it) adds
  inv_x_r    4 Xh -> 4 P            r1, r2, r3, rth (after an inverse z of cr)
  thomas     8 P  -> 4 P            r and u in (CN explicit), u out
  fwd_x      4 P  -> 4 Xh
  fwd_z      4 Xh -> 4 S
for ~67 P (~540 B per point and substep): reference_substep_bytes.

With the LES model (les_model_type 5) the stages change to
  inv_z      4 S  -> 8 Xh           state and its z-derivatives
  inv_x      8 Xh -> 12 P           state, x- and z-derivatives
  products   12 P -> 13 P (AMD walk: nu_t, kappa_t and the 11 product +
             SGS-forcing sequences), then 11 P -> 8 Xh
  thomas     per equation r, u, nu in, u out: 16 P
"""
from __future__ import annotations

import os
import re


def units(p) -> dict:
    nplanes = p.ny + 2
    nkx, nkz = p.nx // 3, p.nz // 3
    w = 4 if getattr(p, "precision", 0) else 8
    return {
        "P": p.nx * p.nz * w * nplanes,
        "Xh": (nkx + 1) * p.nz * 2 * w * nplanes,
        "S": (nkx + 1) * (2 * nkz + 1) * 16 * nplanes,
    }


def _physical_path_bytes(p) -> dict:
    """The reference's stage sequence: CN solves in physical space."""
    u = units(p)
    P, X, S = u["P"], u["Xh"], u["S"]
    les = bool(getattr(p, "use_les", 0))
    return {
        "inv_z": 4 * S + (8 if les else 4) * X,
        "inv_x": (8 * X + 12 * P) if les else (4 * X + 4 * P),
        "products": (12 * P + 13 * P + 11 * P + 8 * X) if les else (4 * P + 8 * X),
        "zpass_rhs": 8 * X + 9 * S + 4 * S + 4 * X,
        "inv_x_r": 4 * X + 4 * P,
        "thomas": 16 * P if les else 12 * P,
        "courant": (3 * P / 3.0) if p.variable_dt else 0.0,
        "fwd_x": 4 * P + 4 * X,
        "fwd_z": 4 * X + 4 * S,
        "rem_div": 8 * S,
    }


def stage_bytes(p) -> dict:
    """Algorithmic bytes of each stage as the library runs it (spectral CN
    solves without LES, physical ones with it)."""
    if getattr(p, "use_les", 0):
        return _physical_path_bytes(p)
    u = units(p)
    P, X, S = u["P"], u["Xh"], u["S"]
    mixed = bool(getattr(p, "precision", 0))
    return {
        "inv_z": 4 * S + 4 * X,
        "inv_x": 4 * X + 4 * P,
        "products": 4 * P + 8 * X,
        "zpass_rhs": 8 * X + (4 if mixed else 8) * S,
        "inv_x_r": 0.0,
        "thomas": (21 if mixed else 25) * S,
        "courant": ((3 * S + 6 * X) / 3.0) if p.variable_dt else 0.0,
        "fwd_x": 0.0,
        "fwd_z": 0.0,
        "rem_div": 8 * S,
    }


def substep_bytes(p) -> float:
    return float(sum(stage_bytes(p).values()))


def reference_substep_bytes(p) -> float:
    """Bytes of the reference's stage sequence (transforms of cr and of the
    new state, physical CN solves), every stage fused as far as it goes."""
    return float(sum(_physical_path_bytes(p).values()))


def state_transfer_bytes(p, nfields: int = 9) -> tuple:
    """Bytes nfields db_upload_field and db_download_field calls move over
    PCIe (host to device, device to host): both ways the retained modes of
    each reference-layout array (kx <= Nkx of the first 2 Nkz + 1 rows of
    every plane); the download writes the zero padding on the host."""
    nplanes = p.ny + 2
    h2d = nfields * nplanes * (2 * (p.nz // 3) + 1) * (p.nx // 3 + 1) * 16
    return h2d, h2d


def profiled_traffic(stage: str, root: str, precision: str = "fp64"):
    """dram__bytes_read.sum + dram__bytes_write.sum per launch of a stage at
    the 512x257x512 size, from the ncu summaries committed under profiles/
    (a line ``traffic_per_launch <stage> <bytes> <fp64|mixed>``), or None."""
    d = os.path.join(root, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith((".md", ".txt")):
            continue
        with open(os.path.join(d, fn)) as f:
            for line in f:
                m = re.match(r"\s*traffic_per_launch\s+(\w+)\s+([0-9.eE+]+)\s+(\w+)", line)
                if m and m.group(1) == stage and m.group(3) == precision:
                    return float(m.group(2))
    return None
