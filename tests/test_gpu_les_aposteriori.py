"""A-posteriori check of the learned closure: LES started from a filtered
resolved run, compared with that run filtered onto the LES grid.

The closure is trained (tensor-core Adam) on box-filtered snapshots of one
resolved realisation (seed 6).  A second realisation (seed 5) is spun up,
filtered onto the 16x17x16 LES grid and continued; from the same filtered
state an FP64 AMD LES (les_model_type 5) and a mixed-precision LES with the
learned closure (les_model_type 6) advance over the same window.  The
horizontal-mean u1, u3 and buoyancy profiles of each LES are compared with
the filtered resolved run after every 40 steps, as the error of their change
since the common filtered start (the part of a profile both inherit from
the initial state says nothing about a closure): summed over fields and
checkpoints the learned closure's error is no larger than AMD's.
"""
import numpy as np
import pytest

from _util import config0_params, grid_for

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_learned_closure_mean_profiles_vs_filtered_dns():
    from diablo3_b200 import les_filter, sgs_train
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import create_grid
    p = config0_params(nx=64, ny=65, nz=64, re=2000.0, kick=0.1)
    gy = grid_for(p)
    gy_c = create_grid(17, lz=p.ly, cs=1.5, grid_type=1)
    # training data from an independent realisation
    tr = Channel(p, gy)
    tr.init_flow(seed=6)
    snaps = []
    for _ in range(4):
        tr.step(40)
        snaps.append(tr.sgs_targets(gy_c, 4, 4, 4))
    tr.close()
    feat = torch.cat([s[0] for s in snaps]).contiguous()
    tgt = torch.cat([s[1] for s in snaps]).contiguous()
    net, losses = sgs_train.train(feat, tgt, steps=600, batch=1 << 30, lr=2e-3, seed=1)
    assert losses[-1] < 0.5 * losses[0]
    # evaluation realisation, filtered onto the LES grid
    dns = Channel(p, gy)
    dns.init_flow(seed=5)
    dns.step(80)
    pc = config0_params(nx=16, ny=17, nz=16, re=2000.0, use_les=1, create_new_flow=0, les_model_type=5)
    fields = les_filter.filter_state_to_les(dns, pc, gy_c)
    amd = Channel(pc, gy_c)
    amd.init_flow(fields=fields)
    pl = config0_params(nx=16, ny=17, nz=16, re=2000.0, use_les=1, create_new_flow=0, les_model_type=6,
                        precision=1)
    lrn = Channel(pl, gy_c)
    lrn.set_sgs_net(net)
    lrn.init_flow(fields=fields)
    rows = slice(2, pc.ny)   # away from the wall rows the BCs set
    ref0 = les_filter.filtered_mean_profiles(dns, gy_c)
    a0, l0 = les_filter.mean_profiles(amd), les_filter.mean_profiles(lrn)
    tot = {"amd": 0.0, "learned": 0.0}
    for w in range(4):
        dns.step(40)
        amd.step(40)
        lrn.step(40)
        ref = les_filter.filtered_mean_profiles(dns, gy_c)
        pa, pl_ = les_filter.mean_profiles(amd), les_filter.mean_profiles(lrn)
        e_a = les_filter.evolution_errors(pa, a0, ref, ref0, rows)
        e_l = les_filter.evolution_errors(pl_, l0, ref, ref0, rows)
        print(f"after {40 * (w + 1)} steps: profile AMD {les_filter.profile_errors(pa, ref, rows)} "
              f"learned {les_filter.profile_errors(pl_, ref, rows)}")
        print(f"   evolution AMD {e_a}  learned {e_l}")
        assert all(np.isfinite(v) for v in list(e_a.values()) + list(e_l.values()))
        tot["amd"] += sum(e_a.values())
        tot["learned"] += sum(e_l.values())
    print(tot)
    assert lrn.status().flags & 1 == 0 and amd.status().flags & 1 == 0
    assert tot["learned"] <= tot["amd"], tot
    for ch in (dns, amd, lrn):
        ch.close()
    net.close()
