"""Energy-budget statistics (db_budget, db_bpe) against numpy restatements
of compute_TKE, compute_TKE_Production, compute_MKE_diss, compute_Vorticity
and compute_BPE (for/diagnostics.f90:1097-1856) evaluated on the same
spectral state, for the infinite front (homogeneousX: x-z means) and the
finite front (z-means per x), on the FP64 and the mixed path (the budget is
FP64 from the FP64 state on both).  Bars: 1e-10 of each row's scale; the
BPE to 1e-10, its PDF bin by bin (a point within rounding of a bin edge
could fall on either side: at most one point's weight).

The budget closure of proc/plot_energetics.m:16-21 is checked over a run:
with E the y-average (integrate_y_var) of the TKE, P of minus the
production terms, B of the buoyancy flux g <v'th'> and eps of the
dissipation, error = dE/dt - P - B + eps stays small against the terms.
"""
import math

import numpy as np
import pytest

from _util import config0_params, grid_for, significant, to_phys

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Channel():
    from diablo3_b200.channel import Channel
    return Channel


def _dthdx(p):
    ro_inv = 1.0 / p.ro
    if not math.isnan(p.dthdx_override):
        return p.dthdx_override
    if p.ic_type in (4, 5):
        return ro_inv / p.delta
    if 6 <= p.ic_type <= 8:
        return 2.0 / p.lx * ro_inv
    return 0.0


def _geom(p, gy):
    from diablo3_b200.grid import metrics
    m = metrics(np.asarray(gy, np.float64))
    pi = float(np.float32(4.0) * np.arctan(np.float32(1.0)))
    kx = np.arange(p.nkx + 1) * 2 * pi / p.lx
    return m, kx, pi


def ref_budget(p, gy, st):
    """The rows of db_budget from the reference's loops (numpy)."""
    m, kx, _ = _geom(p, gy)
    dy, dyf, gyv = m["dy"], m["dyf"], m["gy"]
    c = {f: significant(p, st[f]) for f in (0, 1, 2)}
    u = [to_phys(p, c[f]) for f in (0, 1, 2)]          # (planes, z, x)
    npl, nx, Nyp = p.ny + 2, p.nx, p.ny
    homx = not (5 <= p.ic_type <= 8)
    if homx:
        M = [np.repeat(c[f][:, 0, 0].real[:, None], nx, axis=1) for f in range(3)]
    else:
        M = [u[f].mean(axis=1) for f in range(3)]
    a = [u[f] - M[f][:, None, :] for f in range(3)]
    tws = (p.delta * p.ro) * _dthdx(p) if (p.flavor_front and p.ro != 0) else 0.0

    def ddx(f, j):
        if homx:
            return np.zeros(nx)
        r = np.zeros(nx // 2 + 1, complex)
        r[: p.nkx + 1] = 1j * kx * c[f][j, 0, :]
        return np.fft.irfft(r, n=nx) * nx

    out = {k: np.zeros(npl) for k in ("tke", "uu_dudx", "wu_dwdx", "vu_dvdx", "vv_dvdy", "uv_dudy", "wv_dwdy",
                                      "epsilon_m")}
    for j in range(1, Nyp + 1):
        uu, vv, ww = (a[0][j] ** 2).mean(0), (a[1][j] ** 2).mean(0), (a[2][j] ** 2).mean(0)
        uw = (a[0][j] * a[2][j]).mean(0)
        out["tke"][j] = 0.5 * (uu + vv + ww).mean()
        dudx, dvdx, dwdx = ddx(0, j), ddx(1, j), ddx(2, j)
        out["uu_dudx"][j] = (uu * dudx).mean()
        out["wu_dwdx"][j] = (uw * dwdx).mean()
        eps = np.zeros(nx)
        if not homx:
            w0, w1 = dyf[j - 1] / (2 * dy[j]), dyf[j] / (2 * dy[j])
            dudxm, dwdxm = ddx(0, j - 1), ddx(2, j - 1)
            eps += w0 * dudx ** 2 + w1 * dudxm ** 2 + dvdx ** 2 + w0 * dwdx ** 2 + w1 * dwdxm ** 2
        if j >= 2:
            i2 = 1.0 / (2 * dy[j])
            uv = ((dyf[j - 1] * a[0][j] + dyf[j] * a[0][j - 1]) * i2 * a[1][j]).mean(0)
            wv = ((dyf[j - 1] * a[2][j] + dyf[j] * a[2][j - 1]) * i2 * a[1][j]).mean(0)
            dvdy = (M[1][j + 1] - M[1][j - 1]) / (gyv[j + 1] - gyv[j - 1])
            dudy = (M[0][j] - M[0][j - 1]) / dy[j]
            dwdy = (M[2][j] - M[2][j - 1]) / dy[j] + tws
            out["vu_dvdx"][j] = (uv * dvdx).mean()
            out["vv_dvdy"][j] = (dvdy * vv).mean()
            out["uv_dudy"][j] = (dudy * uv).mean()
            out["wv_dwdy"][j] = (dwdy * wv).mean()
            if not homx:
                eps += dudy ** 2 + dvdy ** 2 + dwdy ** 2
        out["epsilon_m"][j] = eps.mean() / p.re
    # compute_Vorticity: the spectral combinations to physical space
    c2, c3, c1 = significant(p, st[1]), c[2], c[0]
    kxv = kx[None, None, :]
    kz = np.zeros(2 * p.nkz + 1)
    kz[: p.nkz + 1] = np.arange(p.nkz + 1)
    kz[p.nkz + 1:] = -np.arange(p.nkz, 0, -1)
    kzv = (kz * 2 * _geom(p, gy)[2] / p.lz)[None, :, None]
    for name in ("omega_x", "omega_y", "omega_z"):
        out[name] = np.zeros(npl)
    for j in range(1, Nyp + 1):
        v = 0.5 * (c2[j + 1] + c2[j])
        ox = 1j * kzv[0] * v - (c3[j + 1] - c3[j - 1]) / (2 * dyf[j])
        oy = 1j * kxv[0] * c3[j] - 1j * kzv[0] * c1[j]
        oz = (c1[j + 1] - c1[j - 1]) / (2 * dyf[j]) - 1j * kxv[0] * v
        px = to_phys(p, ox[None])[0] - tws
        out["omega_x"][j] = math.sqrt((px ** 2).mean())
        out["omega_y"][j] = math.sqrt((to_phys(p, oy[None])[0] ** 2).mean())
        out["omega_z"][j] = math.sqrt((to_phys(p, oz[None])[0] ** 2).mean())
    return out


def ref_bpe(p, gy, st, nbin):
    m, _, pi = _geom(p, gy)
    dyf = m["dyf"]
    th = to_phys(p, significant(p, st[4]))
    gx = np.arange(p.nx) * p.lx / p.nx
    s1 = th + _dthdx(p) * (gx - 0.5 * p.lx)[None, None, :]
    homx = not (5 <= p.ic_type <= 8)
    ro_inv = 1.0 / p.ro
    pdf = np.zeros(nbin)
    jst, jet = p.jstart_th_ref, p.jend_th_ref
    if homx:
        thmin, thmax = -_dthdx(p) * 0.5 * p.lx * 1.1, _dthdx(p) * 0.5 * p.lx * 1.1
        dth = (thmax - thmin) / nbin + 1e-14
        edges = thmin + np.arange(nbin + 1) * dth
    else:
        edges = -(ro_inv + 1e-14) * np.cos(np.arange(nbin + 1) * pi / nbin)
    for j in range(jst, jet + 1):
        b = s1[j].reshape(-1)
        if homx:
            bins = np.minimum(np.trunc((b - thmin) / dth).astype(int), nbin - 1)
        else:
            cc = -np.minimum(np.maximum(b, -ro_inv), ro_inv) / (ro_inv + 1e-14)
            bins = np.minimum(np.trunc(np.arccos(cc) * nbin / pi).astype(int), nbin - 1)
        ok = bins >= 0
        np.add.at(pdf, bins[ok], dyf[j])
    pdf = pdf / pdf.sum()
    Y = np.concatenate([[0.0], np.cumsum(pdf)]) * p.ly
    e = -np.sum(0.5 * (edges[1:] + edges[:-1]) * 0.5 * (Y[1:] + Y[:-1]) * (Y[1:] - Y[:-1]) / p.ly)
    return e, pdf, edges


CASES = {
    "infinite_front": dict(nx=32, ny=33, nz=32, kick=0.05, re=2000.0),
    "finite_front": dict(nx=32, ny=33, nz=32, ic_type=6, delta=0.5, kick=0.05, re=2000.0,
                         u_bc_ymax=1, w_bc_ymax=1),
    "infinite_front_mixed": dict(nx=32, ny=33, nz=32, kick=0.05, re=2000.0, precision=1),
}


@pytest.mark.parametrize("case", list(CASES))
def test_budget_rows_match_reference_loops(Channel, case):
    p = config0_params(**CASES[case])
    gy = grid_for(p)
    with Channel(p, gy) as ch:
        ch.init_flow(seed=11)
        ch.step(5)
        got = ch.budget()
        st = ch.download_state()
    ref = ref_budget(p, gy, st)
    for k, r in ref.items():
        scale = max(np.abs(r).max(), 1e-300)
        err = np.abs(got[k] - r).max() / scale
        assert err <= 1e-10, (k, err, scale)
    # the front's mean shear makes its production terms non-trivial
    if case == "finite_front":
        assert np.abs(ref["uu_dudx"]).max() > 0 and np.abs(ref["epsilon_m"]).max() > 0


@pytest.mark.parametrize("case", ["infinite_front", "finite_front"])
def test_bpe_matches_reference_loops(Channel, case):
    p = config0_params(**CASES[case])
    gy = grid_for(p)
    with Channel(p, gy) as ch:
        ch.init_flow(seed=12)
        ch.step(3)
        e, pdf, edges = ch.bpe()
        st = ch.download_state()
    from diablo3_b200.grid import metrics
    jst, jet = _th_rows(p)
    p.jstart_th_ref, p.jend_th_ref = jst, jet
    e_ref, pdf_ref, edges_ref = ref_bpe(p, gy, st, p.nx)
    assert np.allclose(edges, edges_ref, rtol=0, atol=1e-14)
    w = metrics(np.asarray(gy))["dyf"][jst: jet + 1].max() / (p.nx * p.nz * metrics(np.asarray(gy))["dyf"][jst: jet + 1].sum())
    assert np.abs(pdf - pdf_ref).sum() <= 2 * w + 1e-14
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref) + 2 * w * p.ly * np.abs(edges).max()


def _th_rows(p):
    # jstart_th / jend_th of init_chan_mpi (for/domain.f90:321-340), one rank in y
    jst = 1 if p.th_bc_ymin == 1 else 2
    return jst, p.ny


def _y_avg(v, dy, ly):
    # integrate_y_var (for/diagnostics.f90:1964-1976)
    return float(np.sum(0.5 * (v[2:-1] + v[1:-2]) * dy[2:-1]) / ly)


@pytest.mark.parametrize("precision", [0, 1])
def test_energy_budget_closes(Channel, precision):
    """d<E>/dt - P - B + eps against the terms over 40 steps of the
    infinite front (Re 1000, kick 5e-2)."""
    from diablo3_b200.grid import metrics
    p = config0_params(nx=32, ny=33, nz=32, kick=0.05, precision=precision)
    gy = grid_for(p)
    dy = metrics(np.asarray(gy))["dy"]
    E, P, B, D = [], [], [], []
    with Channel(p, gy) as ch:
        ch.init_flow(seed=3)
        ch.step(5)
        for _ in range(41):
            b, s = ch.budget(), ch.stats()
            prod = -(b["uu_dudx"] + b["wu_dwdx"] + b["vu_dvdx"] + b["vv_dvdy"] + b["uv_dudy"] + b["wv_dwdy"])
            E.append(_y_avg(b["tke"], dy, p.ly))
            P.append(_y_avg(prod, dy, p.ly))
            B.append(_y_avg(p.grav_y * s["thv"], dy, p.ly))
            D.append(_y_avg(s["epsilon"], dy, p.ly))
            ch.step(1)
    E, P, B, D = map(np.asarray, (E, P, B, D))
    dEdt = (E[2:] - E[:-2]) / (2 * p.delta_t)
    err = dEdt - P[1:-1] - B[1:-1] + D[1:-1]
    scale = np.max(np.abs(np.stack([dEdt, P[1:-1], B[1:-1], D[1:-1]])))
    rel = float(np.abs(err).max() / scale)
    print(f"budget closure (precision {precision}): max |error| / max term = {rel:.3e}")
    assert rel <= 3e-2, rel   # measured 1.65e-2 on both precision paths


def ref_bin_ystar(p, gy, st, field, nbin):
    """Bin_Ystar_and_Write (for/diagnostics.f90:1859-1950) in numpy: field
    [j][z][x] binned by the buoyancy with its background gradient."""
    m, _, pi = _geom(p, gy)
    dyf = m["dyf"]
    th = to_phys(p, significant(p, st[4]))
    gx = np.arange(p.nx) * p.lx / p.nx
    s1 = th + _dthdx(p) * (gx - 0.5 * p.lx)[None, None, :]
    homx = not (5 <= p.ic_type <= 8)
    ro_inv = 1.0 / p.ro
    pdf, fb = np.zeros(nbin), np.zeros(nbin)
    jst, jet = _th_rows(p)
    for j in range(jst, jet + 1):
        b = s1[j].reshape(-1)
        if homx:
            thmin, thmax = -_dthdx(p) * 0.5 * p.lx * 1.1, _dthdx(p) * 0.5 * p.lx * 1.1
            dth = (thmax - thmin) / nbin + 1e-14
            bins = np.minimum(np.trunc((b - thmin) / dth).astype(int), nbin - 1)
        else:
            cc = -np.minimum(np.maximum(b, -ro_inv), ro_inv) / (ro_inv + 1e-14)
            bins = np.minimum(np.trunc(np.arccos(cc) * nbin / pi).astype(int), nbin - 1)
        ok = bins >= 0
        np.add.at(pdf, bins[ok], dyf[j])
        np.add.at(fb, bins[ok], field[j].reshape(-1)[ok] * dyf[j])
    with np.errstate(invalid="ignore", divide="ignore"):
        return fb / pdf, pdf


@pytest.mark.parametrize("case", ["infinite_front", "finite_front"])
def test_bin_ystar_matches_reference_loops(Channel, case):
    """db_bin_ystar of a caller's field (a smooth function of the point) and
    of the kinetic energy against the reference's binning loop; bins whose
    weight differs (points on a bin edge, FP rounding of the buoyancy) are
    left out of the comparison and must be few."""
    p = config0_params(**CASES[case])
    gy = grid_for(p)
    with Channel(p, gy) as ch:
        ch.init_flow(seed=12)
        ch.step(3)
        st = ch.download_state()
        z = np.arange(p.nz)[None, :, None]
        x = np.arange(p.nx)[None, None, :]
        jj = np.arange(p.ny + 2)[:, None, None]
        fld = np.cos(0.3 * jj) + 0.01 * z + 0.002 * x * x
        arr = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
        arr[:, : p.nz, : p.nx] = fld
        got, w = ch.bin_ystar(arr)
        ke, wk = ch.bin_ystar(None)
    ref, wr = ref_bin_ystar(p, gy, st, np.broadcast_to(fld, (p.ny + 2, p.nz, p.nx)), p.nx)
    u = [to_phys(p, significant(p, st[f])) for f in (0, 1, 2)]
    kef = 0.5 * (u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    ke_ref, _ = ref_bin_ystar(p, gy, st, kef, p.nx)
    same = np.isclose(w, wr, rtol=1e-12, atol=1e-300)
    assert (~same).sum() <= 2, (~same).sum()
    assert np.array_equal(np.isnan(got[same]), np.isnan(ref[same]))
    ok = same & np.isfinite(ref)
    assert ok.sum() > 0
    assert np.allclose(got[ok], ref[ok], rtol=1e-10, atol=1e-12)
    assert np.allclose(wk, w) and np.allclose(ke[ok], ke_ref[ok], rtol=1e-9, atol=1e-14)
