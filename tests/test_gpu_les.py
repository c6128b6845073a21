"""LES (les_model_type 5, AMD) parity of the CUDA path with the CPU oracle.

The CUDA path forms the model from transformed x/z derivatives and folds the
SGS stress divergence into the nonlinear-product transforms, where the
reference transforms each tensor separately: the two agree to rounding, so
the FP64 bars are those of the plain path (one substep 1e-12, 20 steps
1e-10 relative L2 per field), and nu_t / kappa_t to 1e-11 of their maximum.
"""
import numpy as np
import pytest

from _util import NAMES, STATE, channel_state, config0_params, grid_for, oracle_state, rel_l2, seed_pair, significant

pytestmark = pytest.mark.gpu

NU_T, KAPPA_T = 9, 10


@pytest.fixture(scope="module")
def Channel():
    from diablo3_b200.channel import Channel
    return Channel


def les_params(**kw):
    base = dict(nx=32, ny=33, nz=32, use_les=1, create_new_flow=0, les_model_type=5, kick=0.05, re=5000.0)
    base.update(kw)
    return config0_params(**base)


def _cmp_state(o, ch, p, tol, cp_base=None):
    so, sg = oracle_state(o, p), channel_state(ch, p)
    errs = {NAMES[f]: rel_l2(sg[f], so[f]) for f in STATE}
    if cp_base is not None:
        errs["cp"] = rel_l2(sg[3] - cp_base, so[3] - cp_base)
    bad = {k: v for k, v in errs.items() if not (v <= tol)}
    assert not bad, f"rel L2 above {tol}: {bad} (all: {errs})"
    return errs


def _cmp_eddy(o, ch, p, tol=1e-11):
    for fid in (NU_T, KAPPA_T):
        a = ch.download_field(fid)[:, : p.nz, : p.nx]
        b = o.real(fid)[:, : p.nz, : p.nx]
        scale = float(np.abs(b).max())
        assert scale > 0.0, "eddy field identically zero: the model did not run"
        err = float(np.abs(a - b).max())
        assert err <= tol * scale, (fid, err, scale)
        assert np.all(a >= 0.0)


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_les_single_substep(oracle_mod, Channel, rk):
    p = les_params()
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=21)
    o.rk_substep(1)
    ch.upload_state({fid: o.cplx(fid).copy() for fid in STATE})
    ch.upload_field(NU_T, o.real(NU_T).copy())
    ch.upload_field(KAPPA_T, o.real(KAPPA_T).copy())
    cp0 = significant(p, o.cplx(3)).copy()
    o.rk_substep(rk)
    ch.rk_chan_1(rk)
    _cmp_eddy(o, ch, p)
    _cmp_state(o, ch, p, 1e-12, cp_base=cp0)


def test_les_20_steps(oracle_mod, Channel):
    p = les_params()
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=22)
    for _ in range(20):
        o.step()
    ch.step(20)
    _cmp_eddy(o, ch, p, tol=1e-10)
    _cmp_state(o, ch, p, 1e-10)
    assert ch.divergence() <= 1e-12


@pytest.mark.parametrize("bcs", [
    # Neumann u/w/th at the bottom: jstart = 1, the raw-strain tau_12 row
    dict(u_bc_ymin=1, w_bc_ymin=1, th_bc_ymin=1, u_bc_ymax=1, w_bc_ymax=1, th_bc_ymax=1),
    # all Dirichlet
    dict(u_bc_ymin=0, w_bc_ymin=0, th_bc_ymin=0, u_bc_ymax=0, w_bc_ymax=0, th_bc_ymax=0,
         th_bc_ymin_c1=-1.0, th_bc_ymax_c1=1.0),
])
def test_les_boundary_variants(oracle_mod, Channel, bcs):
    p = les_params(**bcs)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=23)
    for _ in range(5):
        o.step()
    ch.step(5)
    _cmp_eddy(o, ch, p, tol=1e-10)
    _cmp_state(o, ch, p, 1e-10)


def test_les_spinup_gate(oracle_mod, Channel):
    """create_new_flow: the model starts after time_step 100
    (solver.f90:615); steps 99..102 cross the gate."""
    p = les_params(create_new_flow=1)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=24)
    o.set_clock(time=0.0, time_step=98)
    ch.set_clock(time=0.0, time_step=98)
    for _ in range(2):
        o.step()
    ch.step(2)
    assert float(np.abs(ch.download_field(NU_T)).max()) == 0.0
    for _ in range(2):
        o.step()
    ch.step(2)
    _cmp_eddy(o, ch, p, tol=1e-10)
    _cmp_state(o, ch, p, 1e-10)


def test_les_eddy_field_round_trip(Channel):
    p = les_params()
    gy = grid_for(p)
    with Channel(p, gy) as ch:
        rng = np.random.default_rng(3)
        a = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
        a[:, : p.nz, : p.nx] = rng.random((p.ny + 2, p.nz, p.nx))
        ch.upload_field(KAPPA_T, a)
        assert np.array_equal(ch.download_field(KAPPA_T), a)


def _ref_les_stats(p, gy, st, nu, ka):
    """nu_sgs, kappa_sgs (les.f90:909-935, 1404-1430) and eps_sgs2
    (diagnostics.f90:2057-2118) by the reference's loops, in numpy."""
    from _util import to_phys
    from diablo3_b200.grid import metrics
    m = metrics(np.asarray(gy, np.float64))
    dy, dyf = m["dy"], m["dyf"]
    u1, u2, u3 = (to_phys(p, significant(p, st[f])) for f in (0, 1, 2))   # (planes, z, x)
    nut, kat = nu[:, : p.nz, : p.nx], ka[:, : p.nz, : p.nx]
    n, Nyp, npl = p.nx * p.nz, p.ny, p.ny + 2
    out = np.zeros((3, npl))
    out[0] = nut.sum(axis=(1, 2)) / n
    out[1] = kat.sum(axis=(1, 2)) / n
    s1 = np.zeros_like(u1)
    for j in range(1, Nyp + 1):
        s1[j] = (u1[j] * ((nut[j + 1] * (u1[j + 1] - u1[j]) / dy[j + 1] - nut[j] * (u1[j] - u1[j - 1]) / dy[j])
                          / dyf[j])
                 + u3[j] * ((nut[j + 1] * (u3[j + 1] - u3[j]) / dy[j + 1] - nut[j] * (u3[j] - u3[j - 1]) / dy[j])
                            / dyf[j]))
    for j in range(2, Nyp + 1):
        temp = (0.5 * (s1[j] + s1[j - 1])
                + u2[j] * ((0.5 * (nut[j] + nut[j + 1]) * (u2[j + 1] - u2[j]) / dyf[j]
                            - 0.5 * (nut[j] + nut[j - 1]) * (u2[j] - u2[j - 1]) / dyf[j - 1]) / dy[j]))
        out[2, j] = temp.sum() / n
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_les_stats_match_reference_loops(Channel, precision):
    """db_les_stats (nu_sgs, kappa_sgs, eps_sgs2) against the reference's
    loops on the same state, with nu_t / kappa_t of the AMD closure
    evaluated on that state (as save_stats_LES_OOL runs les_chan before it
    writes).  Bar: 1e-10 of each row's largest value."""
    p = les_params(precision=precision)
    gy = grid_for(p)
    with Channel(p, gy) as ch:
        ch.init_flow(seed=5)
        ch.step(3)
        nu, ka = ch.les_eval(5)
        st = ch.download_state()
        got = ch.les_stats()
    ref = _ref_les_stats(p, gy, st, nu, ka)
    for i, k in enumerate(("nu_sgs", "kappa_sgs", "eps_sgs2")):
        scale = np.abs(ref[i]).max()
        assert scale > 0, k
        err = np.abs(got[k] - ref[i]).max() / scale
        assert err <= 1e-10, (k, err)
    assert got["eps_sgs2"][0] == got["eps_sgs2"][1] == got["eps_sgs2"][-1] == 0.0


def test_les_stats_needs_les(Channel):
    from diablo3_b200 import lib as L
    p = config0_params(nx=32, ny=33, nz=32)
    with Channel(p, grid_for(p)) as ch:
        with pytest.raises(L.DiabloError):
            ch.les_stats()
