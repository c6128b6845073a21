"""End to end: resolved runs of this code -> box-filtered targets -> the
closure trained on the tensor cores -> on held-out filtered snapshots it
predicts the least-squares eddy viscosity and diffusivity better than AMD
(les_model_type 5) evaluated on the same filtered fields."""
import numpy as np
import pytest

from _util import config0_params, grid_for

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_trained_closure_beats_amd_on_held_out_filtered_dns():
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import create_grid
    from diablo3_b200 import sgs_train
    p = config0_params(nx=64, ny=65, nz=64, re=2000.0, kick=0.1)
    gy = grid_for(p)
    gy_c = create_grid(17, lz=p.ly, cs=1.5, grid_type=1)
    ch = Channel(p, gy)
    ch.init_flow(seed=5)
    snaps = []
    for _ in range(4):
        ch.step(40)
        snaps.append(ch.sgs_targets(gy_c, 4, 4, 4))
    feat = torch.cat([s[0] for s in snaps[:3]]).contiguous()
    tgt = torch.cat([s[1] for s in snaps[:3]]).contiguous()
    net, losses = sgs_train.train(feat, tgt, steps=600, batch=1 << 30, lr=2e-3, seed=1)
    assert losses[-1] < 0.5 * losses[0]
    res = sgs_train.compare_with_amd(net, snaps[3][0], snaps[3][1])
    print(res)
    assert res["net"][0] < res["amd"][0], res
    assert res["net"][1] < res["amd"][1], res
