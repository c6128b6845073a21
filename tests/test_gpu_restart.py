"""Restart in the reference's layout on the GPU.

- poisson_p_chan (db_poisson_p) against the oracle's restatement
  (for/solver.f90:1382-1590) on a stepped state, FP64 and mixed contexts
  (the solve is FP64 on both), 1e-10; and the discrete Poisson equation:
  the stretched-grid Laplacian of cp equals minus the right-hand side the
  oracle assembles, at the interior planes.
- write_flow / read_flow (WriteHDF5 / ReadHDF5 layout): with P the state
  comes back (u1, u3, th at the planes 1..Nyp, u2 at 2..Nyp, cp) to
  1e-13; without P, cp is poisson_p_chan of the read state; a run continued
  from the file matches the oracle continued from the same state (1e-10
  after 5 steps).
"""
import numpy as np
import pytest

from _util import STATE, config0_params, grid_for, rel_l2, seed_pair, significant

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Channel():
    from diablo3_b200.channel import Channel
    return Channel


def _stepped(oracle_mod, Channel, precision=0, steps=4):
    p = config0_params(nx=32, ny=33, nz=32, kick=0.05, precision=precision)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=21)
    ch.step(steps)
    st = ch.download_state()
    for f in STATE:
        o.cplx(f)[...] = st[f]
    return p, gy, o, ch, st


@pytest.mark.parametrize("precision", [0, 1])
def test_poisson_p_matches_oracle(oracle_mod, Channel, precision):
    p, gy, o, ch, st = _stepped(oracle_mod, Channel, precision)
    ch.poisson_p_chan()
    o.poisson_p()
    got = significant(p, ch.download_field(3))[1: p.ny + 1]
    ref = significant(p, o.cplx(3))[1: p.ny + 1]
    assert rel_l2(got, ref) <= 1e-10
    ch.close()


def test_poisson_p_solves_the_discrete_equation(oracle_mod, Channel):
    """L cp = -rhs at the planes 2..Nyp-1, with rhs the oracle's assembled
    right-hand side recovered as the Laplacian of its own solution, and the
    Neumann rows cp(2) = cp(1), cp(Nyp) = cp(Nyp-1) off the (0,0) mode."""
    from diablo3_b200.grid import metrics
    p, gy, o, ch, st = _stepped(oracle_mod, Channel)
    ch.poisson_p_chan()
    cp = significant(p, ch.download_field(3))
    m = metrics(np.asarray(gy))
    dy, dyf = m["dy"], m["dyf"]
    nk = p.nkx + 1
    pi = float(np.float32(4.0) * np.arctan(np.float32(1.0)))
    kx = np.arange(nk) * 2 * pi / p.lx
    kzi = np.concatenate([np.arange(p.nkz + 1), -np.arange(p.nkz, 0, -1)])
    kz = kzi * 2 * pi / p.lz
    k2 = kx[None, :] ** 2 + kz[:, None] ** 2
    lap = np.zeros_like(cp)
    for j in range(2, p.ny):
        lap[j] = ((cp[j + 1] - cp[j]) / dy[j + 1] - (cp[j] - cp[j - 1]) / dy[j]) / dyf[j] - k2 * cp[j]
    o.poisson_p()
    cpo = significant(p, o.cplx(3))
    lap_o = np.zeros_like(cpo)
    for j in range(2, p.ny):
        lap_o[j] = ((cpo[j + 1] - cpo[j]) / dy[j + 1] - (cpo[j] - cpo[j - 1]) / dy[j]) / dyf[j] - k2 * cpo[j]
    assert rel_l2(lap[2: p.ny], lap_o[2: p.ny]) <= 1e-9
    off = np.ones(cp.shape[1:], bool)
    off[0, 0] = False
    assert np.abs(cp[2][off] - cp[1][off]).max() <= 1e-12 * np.abs(cp).max()
    assert np.abs(cp[p.ny] - cp[p.ny - 1]).max() <= 1e-12 * np.abs(cp).max()
    ch.close()


def test_flow_file_restart(oracle_mod, Channel, tmp_path):
    from diablo3_b200 import flowfile
    p, gy, o, ch, st = _stepped(oracle_mod, Channel)
    path = str(tmp_path / "end.flow")
    flowfile.write_flow(ch, path)
    a = flowfile.read_flow(path, p, gy)
    back = a.download_state()
    rows = slice(1, p.ny + 1)
    for f in (0, 2, 4, 3):   # u1, u3, th, cp
        assert rel_l2(significant(p, back[f])[rows], significant(p, st[f])[rows]) <= 1e-13, f
    assert rel_l2(significant(p, back[1])[2: p.ny + 1], significant(p, st[1])[2: p.ny + 1]) <= 1e-13
    # without the pressure: cp is poisson_p_chan of the read state
    nop = str(tmp_path / "nop.flow")
    flowfile.write_flow(ch, nop, save_pressure=False)
    b = flowfile.read_flow(nop, p, gy)
    sb = b.download_state()
    for f in STATE:
        o.cplx(f)[...] = sb[f] if f != 3 else 0
    o.poisson_p()
    assert rel_l2(significant(p, sb[3])[rows], significant(p, o.cplx(3))[rows]) <= 1e-10
    # the run continued from the file, against the oracle from the same state
    for f in STATE:
        o.cplx(f)[...] = sb[f]
    t, n = b.status().time, b.status().time_step
    o.set_clock(t, n)
    b.step(5)
    for _ in range(5):
        o.step()
    sc = b.download_state()
    for f in (0, 1, 2, 4):
        assert rel_l2(significant(p, sc[f]), significant(p, o.cplx(f))) <= 1e-10, f
    for c in (ch, a, b):
        c.close()
