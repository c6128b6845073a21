"""Mixed-precision path (precision 1: FP32 transforms, products and SGS;
FP64 state, CN solves, projection) against the FP64 oracle.

Without LES the CN solves run in FP64 on the spectral state, so FP32
rounding enters through the nonlinear terms only.  With LES the physical
fields hold fluctuations about their FP64 plane means and the solves
transform increments, so FP32 rounding scales with the fluctuation and the
change of a substep, not with the stratification the buoyancy carries.
Bars: transforms 1e-6 relative (FP32 round-off over log2 N passes); one
substep 1e-6; after 20 steps, relative L2 1e-5 on each of the nine fields
(cu1, cu2, cu3, cp, cth and the RK history cf1, cf2, cf3, cfth), the
accuracy the mixed path is specified to.  The projection is FP64, so the
divergence after it stays <= 1e-12 of the velocity scale.
"""
import numpy as np
import pytest

from _util import NAMES, STATE, channel_state, config0_params, grid_for, oracle_state, rel_l2, seed_pair, significant

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Channel():
    from diablo3_b200.channel import Channel
    return Channel


BAR_20 = 1e-5   # relative L2 per field after 20 steps


def _check_20(e):
    bad = {k: v for k, v in e.items() if not (v <= BAR_20)}
    assert not bad, f"above {BAR_20}: {bad} (all: {e})"


def _errs(o, ch, p, fields=STATE, cp_base=None):
    so, sg = oracle_state(o, p), channel_state(ch, p)
    e = {NAMES[f]: rel_l2(sg[f], so[f]) for f in fields}
    if cp_base is not None:
        e["cp"] = rel_l2(sg[3] - cp_base, so[3] - cp_base)
    return e


def test_mixed_fft_matches_oracle(oracle_mod, Channel):
    p = config0_params(nx=64, ny=33, nz=64, precision=1)
    gy = grid_for(p)
    o = oracle_mod.Oracle(p, gy)
    rng = np.random.default_rng(1)
    phys = rng.standard_normal((p.ny + 2, p.nz + 2, p.nx + 2))
    a = phys.copy()
    o.fft_to_fourier(a.reshape(-1))
    with Channel(p, gy) as ch:
        cb = ch.fft_xz_to_fourier(phys.copy())
        ca = a.reshape(-1).view(np.complex128).reshape(cb.shape)
        assert rel_l2(significant(p, cb), significant(p, ca)) < 1e-6


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_mixed_single_substep(oracle_mod, Channel, rk):
    p = config0_params(nx=32, ny=33, nz=32, precision=1)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=5)
    o.rk_substep(1)
    ch.upload_state({fid: o.cplx(fid).copy() for fid in STATE})
    cp0 = significant(p, o.cplx(3)).copy()
    o.rk_substep(rk)
    ch.rk_chan_1(rk)
    e = _errs(o, ch, p, cp_base=cp0)
    assert all(v <= 1e-6 for v in e.values()), e


def test_mixed_config0_20_steps(oracle_mod, Channel):
    p = config0_params(precision=1)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=0)
    for _ in range(20):
        o.step()
    ch.step(20)
    e = _errs(o, ch, p)
    _check_20(e)
    u = float(np.abs(significant(p, ch.download_field(0))).max())
    assert ch.divergence() <= 1e-12 * max(1.0, u)


def test_mixed_les_20_steps(oracle_mod, Channel):
    p = config0_params(nx=32, ny=33, nz=32, precision=1, use_les=1, create_new_flow=0, les_model_type=5,
                       kick=0.05, re=5000.0)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=22)
    for _ in range(20):
        o.step()
    ch.step(20)
    e = _errs(o, ch, p)
    _check_20(e)
    a = ch.download_field(9)[:, : p.nz, : p.nx]
    b = o.real(9)[:, : p.nz, : p.nx]
    assert float(np.abs(a - b).max()) <= 1e-4 * float(np.abs(b).max())
