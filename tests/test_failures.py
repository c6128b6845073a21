"""Failure detection and end-run control on the host (no GPU).

The reference stops a run on wall time, on its end time or on a file
``stop.now`` (for/tools.f90:41-69) and stops on malformed input
(for/parameters.f90:96, 211).  Here: end_run's three conditions; the time
loop (for/diablo.f90:62-129) over a stand-in channel stopping on each, with
its statistics and flow saves at their times and FlowError when the device
reports a non-finite state or a bounded wait that gave up; checkpoint files
that are not, are cut short, or changed; and malformed input files, each
rejected with its own error.
"""
import math
import os

import numpy as np
import pytest

from diablo3_b200 import checkpoint, driver
from diablo3_b200 import lib as L
from diablo3_b200.params import InputError, make_params, read_inputs

from test_host import _write_run


def test_end_run_conditions(tmp_path):
    d = str(tmp_path)
    assert driver.end_run(0.5, 1.0, 10.0, 1.0, d) == []
    assert driver.end_run(0.5, 11.0, 10.0, 1.0, d) == ["wall-time"]
    assert driver.end_run(1.0, 1.0, 10.0, 1.0, d) == ["time-limit"]
    (tmp_path / "stop.now").write_text("")
    assert driver.end_run(0.5, 1.0, 10.0, 1.0, d) == ["stop.now"]
    assert driver.end_run(2.0, 20.0, 10.0, 1.0, d) == ["wall-time", "time-limit", "stop.now"]


class FakeChannel:
    """Clock and status of a channel, advanced by dt per step."""

    def __init__(self, dt=0.125, flags_at=None, on_step=None, **kw):
        self.p = make_params(nx=16, ny=17, nz=16, delta_t=dt, **kw)
        self.t, self.n, self.flags = 0.0, 0, 0
        self.flags_at = flags_at or {}
        self.on_step = on_step
        self.clock_sets = []

    def step(self, k=1):
        for _ in range(k):
            self.t += self.p.delta_t
            self.n += 1
            self.flags |= self.flags_at.get(self.n, 0)
            if self.on_step:
                self.on_step(self.n)

    def status(self):
        s = L.DbStatus()
        s.time, s.time_step, s.delta_t, s.flags = self.t, self.n, self.p.delta_t, self.flags
        return s

    def set_clock(self, t, n, sst, sft):
        self.clock_sets.append((t, n, sst, sft))


def test_run_stops_at_time_limit_with_saves(tmp_path):
    ch = FakeChannel(time_limit=1.0, save_stats_dt=0.25, save_flow_dt=0.5)
    seen = {"stats": [], "flow": []}
    r = driver.run(ch, run_dir=str(tmp_path), save_stats=lambda c: seen["stats"].append(c.t),
                   save_flow=lambda c: seen["flow"].append(c.t))
    assert r.reasons == ["time-limit"] and r.steps == 8 and r.time == 1.0
    assert seen["stats"] == [0.25, 0.5, 0.75, 1.0] and seen["flow"] == [0.5, 1.0]
    # the device's next-event dt scheduling is told each new save time
    assert ch.clock_sets[0][2:] == (0.25, 0.5) and ch.clock_sets[-1][2:] == (1.25, 1.5)


def test_run_stops_on_stop_file(tmp_path):
    def touch(n):
        if n == 3:
            (tmp_path / "stop.now").write_text("")
    ch = FakeChannel(on_step=touch)
    r = driver.run(ch, run_dir=str(tmp_path), max_steps=100)
    assert r.reasons == ["stop.now"] and r.steps == 3


def test_run_stops_on_wall_time(tmp_path):
    ticks = iter(range(1000))
    ch = FakeChannel()
    r = driver.run(ch, wall_time_limit=4.5, run_dir=str(tmp_path), max_steps=100, clock=lambda: float(next(ticks)))
    assert r.reasons == ["wall-time"] and r.steps == 5


def test_run_max_steps_without_stop(tmp_path):
    r = driver.run(FakeChannel(), run_dir=str(tmp_path), max_steps=7)
    assert r.reasons == [] and r.steps == 7


@pytest.mark.parametrize("flag,words", [(1, "non-finite"), (2, "dt <= 0"), (16, "wait gave up")])
def test_run_ends_on_device_flags(tmp_path, flag, words):
    ch = FakeChannel(flags_at={4: flag})
    with pytest.raises(driver.FlowError) as ei:
        driver.run(ch, run_dir=str(tmp_path), max_steps=100)
    assert ei.value.flags == flag and ei.value.time_step == 4 and words in str(ei.value)


def _ckpt(tmp_path):
    rng = np.random.default_rng(3)
    arrays = [("spec0", rng.standard_normal((5, 6, 4)) + 1j), ("nu_t", rng.standard_normal((5, 6, 8)))]
    path = str(tmp_path / "c.ckpt")
    checkpoint.write(path, {"params": {"nx": 8}, "gy": [0.0, 1.0], "time": 0.5, "time_step": 7}, arrays)
    return path, arrays


def test_checkpoint_reads_back(tmp_path):
    path, arrays = _ckpt(tmp_path)
    hdr, got = checkpoint.read(path)
    assert hdr["time_step"] == 7
    for n, a in arrays:
        assert np.array_equal(got[n], a)


def test_checkpoint_truncated(tmp_path):
    path, _ = _ckpt(tmp_path)
    data = open(path, "rb").read()
    for cut in (len(data) - 100, 30, 12, 5):
        with open(path, "wb") as f:
            f.write(data[:cut])
        with pytest.raises(checkpoint.CheckpointError):
            checkpoint.read(path)


def test_checkpoint_corrupt_bytes(tmp_path):
    path, _ = _ckpt(tmp_path)
    data = bytearray(open(path, "rb").read())
    data[-50] ^= 0x10   # one bit of the last array
    with open(path, "wb") as f:
        f.write(bytes(data))
    with pytest.raises(checkpoint.CheckpointError, match="CRC"):
        checkpoint.read(path)


def test_checkpoint_bad_header_and_trailing_bytes(tmp_path):
    path, _ = _ckpt(tmp_path)
    data = open(path, "rb").read()
    bad = data[:16] + b"#" + data[17:]   # the JSON header no longer parses
    with open(path, "wb") as f:
        f.write(bad)
    with pytest.raises(checkpoint.CheckpointError, match="header"):
        checkpoint.read(path)
    with open(path, "wb") as f:
        f.write(data + b"x")
    with pytest.raises(checkpoint.CheckpointError, match="after the last array"):
        checkpoint.read(path)
    with open(path, "wb") as f:
        f.write(b"NOTMAGIC" + data[8:])
    with pytest.raises(checkpoint.CheckpointError, match="not a checkpoint"):
        checkpoint.read(path)


def test_malformed_inputs_rejected(tmp_path):
    _write_run(tmp_path)
    read_inputs(str(tmp_path))   # the intact run directory parses
    chan = (tmp_path / "input_chan.dat").read_text()
    # input_chan.dat cut after the BC rows began
    (tmp_path / "input_chan.dat").write_text("\n".join(chan.splitlines()[:22]) + "\n")
    with pytest.raises(InputError, match="ends before"):
        read_inputs(str(tmp_path))
    # a value that is not a number
    (tmp_path / "input_chan.dat").write_text(chan.replace("2.0\n", "two\n", 1))
    with pytest.raises(InputError, match="unreadable"):
        read_inputs(str(tmp_path))
    # a missing file
    (tmp_path / "input_chan.dat").unlink()
    with pytest.raises(InputError, match="missing input_chan.dat"):
        read_inputs(str(tmp_path))
    # grid_def.all without Nx
    (tmp_path / "input_chan.dat").write_text(chan)
    g = (tmp_path / "grid_def.all").read_text()
    (tmp_path / "grid_def.all").write_text("\n".join(x for x in g.splitlines() if "Nx" not in x) + "\n")
    with pytest.raises(InputError):
        read_inputs(str(tmp_path))
