"""Checkpoint / restart: a run restarted from a checkpoint continues
bit-identically to the uninterrupted run (FP64 DNS with CFL-limited dt, and
mixed-precision AMD LES whose eddy viscosity carries over)."""
import numpy as np
import pytest

from _util import STATE, config0_params, grid_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["dns_fp64_variable_dt", "les_mixed"])
def test_restart_is_bit_identical(case, tmp_path):
    from diablo3_b200 import checkpoint
    from diablo3_b200.channel import Channel
    kw = dict(nx=32, ny=33, nz=32, kick=0.05)
    if case.startswith("dns"):
        kw.update(variable_dt=1, cfl=0.5)
    else:
        kw.update(use_les=1, create_new_flow=0, les_model_type=5, re=5000.0, precision=1)
    p = config0_params(**kw)
    gy = grid_for(p)
    a = Channel(p, gy)
    a.init_flow(seed=4)
    a.step(5)
    path = str(tmp_path / "run.ckpt")
    checkpoint.save(a, path)
    a.step(5)
    b = checkpoint.load(path)
    b.step(5)
    sa, sb = a.download_state(), b.download_state()
    for fid in STATE:
        assert np.array_equal(sa[fid], sb[fid]), fid
    ta, tb = a.status(), b.status()
    assert ta.time_step == tb.time_step and ta.time == tb.time and ta.delta_t == tb.delta_t
    a.close()
    b.close()
