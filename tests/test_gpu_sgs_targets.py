"""Box-filtered training targets of the learned closure (db_sgs_targets)
against a numpy statement of the same filter, stress, flux and
least-squares fit from the oracle's state (FP32 outputs: 1e-5 relative)."""
import numpy as np
import pytest

from _util import config0_params, grid_for, seed_pair, to_phys

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _numpy_targets(p, o, gy_c, fx, fy, fz):
    met = {k: o.metric(i, p.ny + 2) for i, k in enumerate(("gy", "gyf", "dy", "dyf"))}
    gyf, dyf = met["gyf"], met["dyf"]
    kx = o.metric(4, p.nxp)[: p.nkx + 1]
    kz = o.metric(5, 2 * p.nkz + 1)
    sl = (slice(None), slice(0, 2 * p.nkz + 1), slice(0, p.nkx + 1))
    ikx, ikz = 1j * kx[None, None, :], 1j * kz[None, :, None]
    c = {f: o.cplx(f)[sl] for f in (0, 1, 2, 4)}
    ph = lambda a: to_phys(p, a)
    u = [ph(c[0]), ph(c[1]), ph(c[2])]
    th = ph(c[4])
    dx_ = [ph(ikx * c[f]) for f in (0, 1, 2, 4)]
    dz_ = [ph(ikz * c[f]) for f in (0, 1, 2, 4)]
    nxc, nzc, nyc = p.nx // fx, p.nz // fz, (p.ny - 1) // fy + 1
    cg = np.zeros(nyc + 2)
    cg[1:] = gy_c
    cgyf = np.zeros(nyc + 2)
    cgyf[1:nyc + 1] = 0.5 * (cg[1:nyc + 1] + cg[2:nyc + 2])
    cgyf[0] = 2 * cgyf[1] - cgyf[2]
    feats, tgts = [], []
    for k in range(3, nyc):
        J = fy * (k - 1)
        cells = range(J - fy // 2, J + fy // 2)
        acc = None
        W = 0.0
        for jc in cells:
            iyc = 1.0 / (gyf[jc + 1] - gyf[jc - 1])
            u1, u3, t = u[0][jc], u[2][jc], th[jc]
            u2 = 0.5 * (u[1][jc] + u[1][jc + 1])
            G = [dx_[0][jc], (u[0][jc + 1] - u[0][jc - 1]) * iyc, dz_[0][jc],
                 0.5 * (dx_[1][jc] + dx_[1][jc + 1]), (u[1][jc + 1] - u[1][jc]) / dyf[jc],
                 0.5 * (dz_[1][jc] + dz_[1][jc + 1]),
                 dx_[2][jc], (u[2][jc + 1] - u[2][jc - 1]) * iyc, dz_[2][jc]]
            gt = [dx_[3][jc], (th[jc + 1] - th[jc - 1]) * iyc, dz_[3][jc]]
            q = [u1, u2, u3, t, u1 * u1, u2 * u2, u3 * u3, u1 * u2, u1 * u3, u2 * u3, u1 * t, u2 * t, u3 * t] + G + gt
            # x-z box sums (blocks of fx x fz), weighted by dyf
            blk = [dyf[jc] * a.reshape(nzc, fz, nxc, fx).sum(axis=(1, 3)) for a in q]
            acc = blk if acc is None else [a + b for a, b in zip(acc, blk)]
            W += dyf[jc] * fx * fz
        m = [a / W for a in acc]
        ub, tb = m[0:3], m[3]
        t11, t22, t33 = m[4] - ub[0] ** 2, m[5] - ub[1] ** 2, m[6] - ub[2] ** 2
        t12, t13, t23 = m[7] - ub[0] * ub[1], m[8] - ub[0] * ub[2], m[9] - ub[1] * ub[2]
        tr = (t11 + t22 + t33) / 3
        t11, t22, t33 = t11 - tr, t22 - tr, t33 - tr
        qv = [m[10] - ub[0] * tb, m[11] - ub[1] * tb, m[12] - ub[2] * tb]
        Gb, gb = m[13:22], m[22:25]
        S11, S22, S33 = Gb[0], Gb[4], Gb[8]
        S12, S13, S23 = 0.5 * (Gb[1] + Gb[3]), 0.5 * (Gb[2] + Gb[6]), 0.5 * (Gb[5] + Gb[7])
        SS = S11 ** 2 + S22 ** 2 + S33 ** 2 + 2 * (S12 ** 2 + S13 ** 2 + S23 ** 2)
        TS = t11 * S11 + t22 * S22 + t33 * S33 + 2 * (t12 * S12 + t13 * S13 + t23 * S23)
        gg = gb[0] ** 2 + gb[1] ** 2 + gb[2] ** 2
        qg = qv[0] * gb[0] + qv[1] * gb[1] + qv[2] * gb[2]
        nu = np.where(SS > 0, np.maximum(0, -TS / (2 * np.where(SS > 0, SS, 1))), 0)
        ka = np.where(gg > 0, np.maximum(0, -qg / np.where(gg > 0, gg, 1)), 0)
        f = np.stack(Gb + gb + [np.full_like(nu, 3 * p.lx / nxc), np.full_like(nu, 2 * (cgyf[k] - cgyf[k - 1])),
                                np.full_like(nu, 3 * p.lz / nzc), gb[1]], axis=-1)
        feats.append(f.reshape(-1, 16))
        tgts.append(np.stack([nu, ka], axis=-1).reshape(-1, 2))
    return np.concatenate(feats), np.concatenate(tgts)


def test_sgs_targets_match_numpy(oracle_mod):
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import create_grid
    p = config0_params(nx=32, ny=33, nz=32, use_les=1, les_model_type=5, create_new_flow=0, kick=0.05, re=5000.0)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=41)
    gy_c = create_grid(9, lz=p.ly, cs=1.5, grid_type=1)
    feat, tgt = ch.sgs_targets(gy_c, 4, 4, 4)
    f_ref, t_ref = _numpy_targets(p, o, gy_c, 4, 4, 4)
    f, t = feat.cpu().numpy(), tgt.cpu().numpy()
    assert f.shape == f_ref.shape and t.shape == t_ref.shape
    scale = np.abs(f_ref).max(axis=0) + 1e-30
    assert np.all(np.abs(f - f_ref).max(axis=0) <= 1e-5 * scale)
    for q in range(2):
        assert np.abs(t[:, q] - t_ref[:, q]).max() <= 1e-5 * np.abs(t_ref[:, q]).max()
    assert (t_ref[:, 0] > 0).mean() > 0.2   # the fit is not trivially zero
