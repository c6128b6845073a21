"""Failure detection on the GPU, without faulting it.

- A NaN uploaded from the host into cu1 is reported as DB_FLAG_NONFINITE
  after one step (the CN solves check the new state), and the host driver
  ends the run with FlowError; after a clean upload the context steps on.
- With the first TMA wait of the products and x-pass kernels limited to one
  poll, those waits give up before their copies land: the kernels record
  DB_FLAG_WAIT_TIMEOUT, wait (within the built-in bound) for the copies
  they issued and return; the context stays usable, and with the limit
  lifted the next steps equal those of an untouched channel bit for bit.
- The host driver over a real channel stops on stop.now and on time_limit.
- A truncated checkpoint is refused before a context is made.
"""
import numpy as np
import pytest

from _util import STATE, channel_state, config0_params, grid_for, rel_l2, seed_pair

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Channel():
    from diablo3_b200.channel import Channel
    return Channel


def test_nonfinite_state_flagged(oracle_mod, Channel, tmp_path):
    from diablo3_b200 import driver
    p = config0_params(nx=32, ny=33, nz=32)
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=4)
    good = ch.download_state()
    bad = good[0].copy()
    bad[10, 3, 2] = np.nan
    ch.upload_field(0, bad)
    ch.step(1)
    assert ch.status().flags & 1
    ch.upload_field(0, bad)
    with pytest.raises(driver.FlowError, match="non-finite"):
        driver.run(ch, run_dir=str(tmp_path), max_steps=3)
    # a clean state and cleared status: the context steps on
    ch.upload_state(good)
    ch.clear_status()
    ch.step(2)
    assert ch.status().flags == 0 and ch.divergence() < 1e-12
    ch.close()


def test_wait_timeout_flag_and_recovery(Channel):
    p = config0_params(nx=64, ny=33, nz=64)
    gy = grid_for(p)
    a = Channel(p, gy)
    a.init_flow(seed=9)
    start = a.download_state()
    b = Channel(p, gy)
    b.upload_state(start)
    a.set_wait_limit(1)
    a.step(1)
    assert a.status().flags & 16, "no wait gave up with a one-poll limit"
    a.set_wait_limit(0)
    a.clear_status()
    a.upload_state(start)
    a.set_clock(0.0, 0, 1e300, 1e300)
    a.step(3)
    b.step(3)
    assert a.status().flags == 0
    sa, sb = channel_state(a, p), channel_state(b, p)
    for f in STATE:
        assert np.array_equal(sa[f], sb[f]), f
    a.close()
    b.close()


def test_driver_stops_on_stop_file_and_time_limit(Channel, tmp_path):
    from diablo3_b200 import driver
    p = config0_params(nx=32, ny=33, nz=32, time_limit=5.5e-3)   # dt 1e-3: the sixth step reaches it
    gy = grid_for(p)
    ch = Channel(p, gy)
    ch.init_flow(seed=2)
    r = driver.run(ch, run_dir=str(tmp_path), max_steps=50)
    assert r.reasons == ["time-limit"] and r.steps == 6
    (tmp_path / "stop.now").write_text("")
    r = driver.run(ch, run_dir=str(tmp_path), time_limit=1e9, max_steps=50)
    assert r.reasons == ["stop.now"] and r.steps == 1
    ch.close()


def test_truncated_checkpoint_refused(Channel, tmp_path):
    from diablo3_b200 import checkpoint
    p = config0_params(nx=32, ny=33, nz=32)
    ch = Channel(p, grid_for(p))
    ch.init_flow(seed=1)
    path = str(tmp_path / "run.ckpt")
    checkpoint.save(ch, path)
    ch.close()
    data = open(path, "rb").read()
    with open(path, "wb") as f:
        f.write(data[: len(data) // 2])
    with pytest.raises(checkpoint.CheckpointError, match="truncated"):
        checkpoint.load(path)
