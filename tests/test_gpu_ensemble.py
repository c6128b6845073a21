"""Ensembles: one graph launch per step advances every member exactly as
stepping that member alone does (same kernels: bit-identical state)."""
import numpy as np
import pytest

from _util import STATE, channel_state, config0_params, grid_for

pytestmark = pytest.mark.gpu


def test_ensemble_members_equal_solo_runs():
    from diablo3_b200.channel import Channel
    from diablo3_b200.ensemble import Ensemble
    ps = [config0_params(nx=32, ny=33, nz=32, dthdx_override=m2) for m2 in (0.7, 1.0, 1.3)]
    gy = grid_for(ps[0])
    ens = Ensemble(ps, gy, seeds=[3, 4, 5])
    solo = []
    for p, sd in zip(ps, (3, 4, 5)):
        ch = Channel(p, gy)
        ch.init_flow(seed=sd)
        solo.append(ch)
    ens.step(6)
    for ch in solo:
        ch.step(6)
    for a, b, p in zip(ens.members, solo, ps):
        sa, sb = channel_state(a, p), channel_state(b, p)
        for f in STATE:
            assert np.array_equal(sa[f], sb[f]), f
        assert a.status().time_step == b.status().time_step == 6
    # members differ from each other (different seeds and fronts)
    assert not np.array_equal(channel_state(ens.members[0], ps[0])[0], channel_state(ens.members[1], ps[1])[0])
    ens.close()


def test_ensemble_mixed_precision_members_track_fp64():
    from diablo3_b200.channel import Channel
    from diablo3_b200.ensemble import Ensemble
    ps = [config0_params(nx=32, ny=33, nz=32, precision=1, dthdx_override=m2) for m2 in (0.8, 1.2)]
    gy = grid_for(ps[0])
    ens = Ensemble(ps, gy, seeds=[7, 8])
    ens.step(10)
    for i, m2 in enumerate((0.8, 1.2)):
        p64 = config0_params(nx=32, ny=33, nz=32, dthdx_override=m2)
        ref = Channel(p64, gy)
        ref.init_flow(seed=7 + i)
        ref.step(10)
        a, b = channel_state(ens.members[i], ps[i]), channel_state(ref, p64)
        for f in (0, 1, 2, 4):
            err = np.linalg.norm(a[f] - b[f]) / np.linalg.norm(b[f])
            assert err <= 1e-6, (i, f, err)
    ens.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_form_equals_member_graphs(precision):
    """Members without LES at a fixed dt are batched (each kernel of the step
    launched once per group of members, the member's arguments from a
    device table); the per-member graph branches, one group and two groups
    give bit-identical states.  nx != nz and unequal forcing per member."""
    from diablo3_b200.ensemble import Ensemble
    ps = [config0_params(nx=64, ny=33, nz=32, precision=precision, dthdx_override=m2)
          for m2 in (0.6, 0.9, 1.4, 1.1)]
    gy = grid_for(ps[0])
    seeds = [11, 12, 13, 14]
    a = Ensemble(ps, gy, seeds=seeds)
    b = Ensemble(ps, gy, seeds=seeds)
    c = Ensemble(ps, gy, seeds=seeds)
    assert a.batched and b.batched and a.groups == 1
    b.batched = False
    c.groups = 2
    assert not b.batched and c.groups == 2
    for e in (a, b, c):
        e.step(4)
    for e in (a, b, c):
        e.step(3)
    assert a.kernels_per_step() == 26                       # one launch per kernel for all members
    assert c.kernels_per_step() == 2 * 26                   # one per kernel and group
    assert b.kernels_per_step() > 2 * a.kernels_per_step()  # each member's own kernels
    for ma, mb, mc, p in zip(a.members, b.members, c.members, ps):
        sa, sb, sc = channel_state(ma, p), channel_state(mb, p), channel_state(mc, p)
        for f in STATE:
            assert np.array_equal(sa[f], sb[f]), f
            assert np.array_equal(sc[f], sb[f]), f
        st_a, st_b, st_c = ma.status(), mb.status(), mc.status()
        assert st_a.flags == st_b.flags == st_c.flags == 0
        assert st_a.time_step == st_b.time_step == st_c.time_step == 7
        assert st_a.time == st_b.time == st_c.time
    # the batched form again on the second ensemble continues identically
    b.batched = True
    a.step(2)
    b.step(2)
    for ma, mb, p in zip(a.members, b.members, ps):
        assert np.array_equal(channel_state(ma, p)[0], channel_state(mb, p)[0])
    a.close()
    b.close()
    c.close()


def test_batched_form_only_where_members_qualify():
    """Members with a CFL-limited dt (or LES) step through the per-member
    graph branches; asking for the batched form is an argument error."""
    from diablo3_b200 import lib as L
    from diablo3_b200.ensemble import Ensemble
    ps = [config0_params(nx=32, ny=33, nz=32, variable_dt=1, dthdx_override=m2) for m2 in (0.8, 1.2)]
    gy = grid_for(ps[0])
    ens = Ensemble(ps, gy, seeds=[1, 2])
    assert not ens.batched
    with pytest.raises(L.DiabloError):
        ens.batched = True
    ens.step(2)
    assert all(m.status().time_step == 2 and m.status().flags == 0 for m in ens.members)
    ens.close()
