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
