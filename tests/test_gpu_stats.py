"""Mean and energy-budget profiles (db_stats, save_stats_chan).

1. The FP64 kernel (Parseval sums over the spectral state) against the
   reference's own physical-space definitions (for/diagnostics.f90)
   evaluated in numpy on the same state: 1e-10 of each row's scale (the
   dissipation row, a sum of nine squared gradients, 1e-8), for an
   x-homogeneous flow (IC 4, averages over x and z) and a front (IC 6,
   averages over z only).
2. Long run of the mixed path: after 1000 steps of a 64x65x64 channel its
   mean profiles and energy-budget integrals (TKE, dissipation, chi,
   buoyancy flux) match the FP64 path's.
"""
import numpy as np
import pytest

from _util import config0_params, grid_for, to_phys

pytestmark = pytest.mark.gpu


def _reference_stats(p, ch):
    """The save_stats_chan rows from the physical fields (numpy)."""
    from diablo3_b200.grid import metrics
    m = metrics(ch.gy)
    dy, dyf, gy, gyf = m["dy"], m["dyf"], m["gy"], m["gyf"]
    st = ch.download_state()
    nkx, nkzp = p.nkx, 2 * p.nkz + 1
    c = {f: st[f][:, :nkzp, :nkx + 1] for f in (0, 1, 2, 4)}
    kx = np.arange(nkx + 1) * (2 * np.pi / p.lx)
    kzi = np.concatenate([np.arange(p.nkz + 1), np.arange(-p.nkz, 0)])
    kz = kzi * (2 * np.pi / p.lz)
    u1, u2, u3, th = (to_phys(p, c[f]) for f in (0, 1, 2, 4))
    homx = not (5 <= p.ic_type <= 8)
    dx = {f: to_phys(p, 1j * kx[None, None, :] * c[f]) for f in (0, 1, 2, 4)}
    dz = {f: to_phys(p, 1j * kz[None, :, None] * c[f]) for f in (0, 1, 2, 4)}
    if not homx:   # epsilon's x-derivatives skip the z-mean (compute_TKE_diss k_start = 1)
        cf = {f: c[f] * (kzi != 0)[None, :, None] for f in (0, 1, 2)}
        dxe = {f: to_phys(p, 1j * kx[None, None, :] * cf[f]) for f in (0, 1, 2)}
    else:
        dxe = dx
    ax = (1, 2) if homx else (1,)

    def mean(a):   # ume_xy: over x and z, or over z only
        return a.mean(axis=ax, keepdims=True)

    def avg(a):
        return a.mean(axis=(1, 2))
    f1, f2, f3, ft = u1 - mean(u1), u2 - mean(u2), u3 - mean(u3), th - mean(th)
    n = p.ny + 2
    out = {k: np.zeros(n) for k in ("ume", "vme", "wme", "thme", "urms", "vrms", "wrms", "thrms",
                                   "uv", "wv", "uw", "thv", "epsilon", "chi")}
    out["ume"], out["vme"], out["wme"], out["thme"] = avg(u1), avg(u2), avg(u3), avg(th)
    out["urms"], out["vrms"] = np.sqrt(avg(f1 ** 2)), np.sqrt(avg(f2 ** 2))
    out["wrms"], out["thrms"] = np.sqrt(avg(f3 ** 2)), np.sqrt(avg(ft ** 2))
    out["uw"] = avg(f1 * f3)
    nu = 1.0 / p.re
    m2 = 1.0 / p.ro / p.delta if p.ic_type in (4, 5) else 2.0 / p.lx / p.ro   # flow.f90 dTHdX
    for j in range(2, p.ny + 1):
        a, b = dyf[j - 1] / (2 * dy[j]), dyf[j] / (2 * dy[j])
        out["uv"][j] = np.mean((a * f1[j] + b * f1[j - 1]) * f2[j])
        out["wv"][j] = np.mean((a * f3[j] + b * f3[j - 1]) * f2[j])
        e = (a * dxe[0][j] ** 2 + b * dxe[0][j - 1] ** 2) + dxe[1][j] ** 2 + ((f1[j] - f1[j - 1]) / dy[j]) ** 2
        e += (a * dxe[2][j] ** 2 + b * dxe[2][j - 1] ** 2) + (a * dz[0][j] ** 2 + b * dz[0][j - 1] ** 2)
        e += ((f2[j + 1] - f2[j - 1]) / (gy[j + 1] - gy[j - 1])) ** 2 + ((f3[j] - f3[j - 1]) / dy[j]) ** 2
        e += dz[1][j] ** 2 + (a * dz[2][j] ** 2 + b * dz[2][j - 1] ** 2)
        out["epsilon"][j] = nu * np.mean(e)
    for j in range(1, p.ny + 1):
        out["thv"][j] = np.mean(ft[j] * 0.5 * (f2[j] + f2[j + 1]))
        g2 = (dx[4][j] + m2) ** 2 + ((th[j + 1] - th[j - 1]) / (gyf[j + 1] - gyf[j - 1])) ** 2 + dz[4][j] ** 2
        out["chi"][j] = np.mean(g2)
    return out


@pytest.mark.parametrize("ic", [4, 6])
def test_stats_match_reference_definitions(ic):
    from diablo3_b200.channel import Channel
    p = config0_params(nx=32, ny=33, nz=32, kick=0.05, ic_type=ic)
    gy = grid_for(p)
    ch = Channel(p, gy)
    ch.init_flow(seed=3)
    ch.step(3)
    got = ch.stats()
    ref = _reference_stats(p, ch)
    lo = {"uv": 2, "wv": 2, "epsilon": 2}
    for k, r in ref.items():
        j0 = lo.get(k, 1)
        a, b = got[k][j0:p.ny + 1], r[j0:p.ny + 1]
        scale = max(np.abs(b).max(), 1e-6)   # rows that vanish to rounding (vme) get an absolute bound
        tol = 1e-8 if k == "epsilon" else 1e-10
        assert np.abs(a - b).max() <= tol * scale, (k, np.abs(a - b).max(), scale)
    ch.close()


def test_mixed_long_run_profiles_and_budget():
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import metrics
    res = {}
    for prec in (0, 1):
        p = config0_params(nx=64, ny=65, nz=64, kick=0.05, precision=prec)
        gy = grid_for(p)
        ch = Channel(p, gy)
        ch.init_flow(seed=11)
        ch.step(1000)
        res[prec] = ch.stats()
        ch.close()
    dyf = metrics(gy)["dyf"]
    rows = slice(2, p.ny)

    def integral(s):
        return {"tke": float(np.sum(0.5 * (s["urms"] ** 2 + s["vrms"] ** 2 + s["wrms"] ** 2)[rows] * dyf[rows])),
                "epsilon": float(np.sum(s["epsilon"][rows] * dyf[rows])),
                "chi": float(np.sum(s["chi"][rows] * dyf[rows])),
                "thv": float(np.sum(s["thv"][rows] * dyf[rows]))}
    i64, imx = integral(res[0]), integral(res[1])
    prof = {k: float(np.linalg.norm(res[1][k][rows] - res[0][k][rows]) / np.linalg.norm(res[0][k][rows]))
            for k in ("ume", "wme", "thme")}
    bud = {k: abs(imx[k] - i64[k]) / abs(i64[k]) for k in i64}
    print("mean profiles", prof, "budget", bud, i64)
    assert max(prof.values()) <= 1e-5, prof
    assert max(bud.values()) <= 1e-4, bud
