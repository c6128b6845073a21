"""Accuracy of the timed configurations at their stated sizes.

- Config 2 (256x129x256 AMD LES of a finite front, Re 1e5): the mixed path
  against the FP64 path from the same state after 200 steps with the LES on
  from the first step (create_new_flow = 0, the gate of
  for/solver.f90:615).  The dt is held fixed at 2e-3 (CFL ~0.1 on this
  grid) so both arms reach the same times; the bench runs the same flow
  with the CFL-limited dt.  Reported: the rel-L2 of every state field and
  of the horizontal-mean u1, u3, th profiles (measured: state <= 7.4e-7,
  cf <= 1.2e-5, mean profiles <= 3e-8).
- Config 4 (64 members of 128x65x128, Ri_i ~ U[0.5, 2] from PCG64(1000),
  Re 2000, mixed precision, one graph launch per step): members 0, 31 and
  63 against solo FP64 runs of the same parameters and seed after 50 steps
  (measured: state <= 8.1e-7, cf <= 2.3e-5).
"""
import numpy as np
import pytest

from _util import STATE, NAMES, channel_state

pytestmark = pytest.mark.gpu


def _rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def test_config2_mixed_amd_tracks_fp64_amd():
    from diablo3_b200 import les_filter
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import create_grid
    from diablo3_b200.workloads import workload_params
    p64 = workload_params("config2")
    p64.variable_dt, p64.delta_t = 0, 2e-3
    pmx = workload_params("config2")
    pmx.variable_dt, pmx.delta_t, pmx.precision = 0, 2e-3, 1
    gy = create_grid(p64.ny, lz=p64.ly, cs=1.5, grid_type=1)
    a = Channel(p64, gy)
    a.init_flow(seed=0)
    b = Channel(pmx, gy)
    b.upload_state(a.download_state())
    a.step(200)
    b.step(200)
    assert a.status().flags == 0 and b.status().flags == 0
    sa, sb = channel_state(a, p64), channel_state(b, pmx)
    errs = {NAMES[f]: _rel(sb[f], sa[f]) for f in STATE}
    rows = slice(2, p64.ny)
    pa, pb = les_filter.mean_profiles(a), les_filter.mean_profiles(b)
    perr = les_filter.profile_errors(pb, pa, rows)
    print("config 2, 200 steps, mixed vs FP64: fields", errs, "mean profiles", perr)
    for f in ("cu1", "cu2", "cu3", "cp", "cth"):
        assert errs[f] <= 1e-5, (f, errs)
    for f in ("cf1", "cf2", "cf3", "cfth"):
        assert errs[f] <= 1e-4, (f, errs)
    assert max(perr.values()) <= 1e-6, perr
    a.close()
    b.close()


def test_config4_members_track_solo_fp64():
    from diablo3_b200.channel import Channel
    from diablo3_b200.ensemble import Ensemble, config4_members
    from diablo3_b200.grid import create_grid
    ps, ri = config4_members(64, precision=1)
    p64s, _ = config4_members(64, precision=0)
    gy = create_grid(ps[0].ny, lz=ps[0].ly, cs=1.5, grid_type=1)
    ens = Ensemble(ps, gy, seeds=list(range(64)))
    ens.step(50)
    for i in (0, 31, 63):
        solo = Channel(p64s[i], gy)
        solo.init_flow(seed=i)
        solo.step(50)
        sa, sb = channel_state(ens.members[i], ps[i]), channel_state(solo, p64s[i])
        errs = {NAMES[f]: _rel(sa[f], sb[f]) for f in STATE}
        print(f"config 4 member {i} (Ri {ri[i]:.3f}), 50 steps, mixed vs solo FP64:", errs)
        for f in ("cu1", "cu2", "cu3", "cp", "cth"):
            assert errs[f] <= 1e-5, (i, f, errs)
        for f in ("cf1", "cf2", "cf3", "cfth"):
            assert errs[f] <= 1e-4, (i, f, errs)
        assert ens.members[i].status().time_step == solo.status().time_step == 50
        solo.close()
    ens.close()
