"""The reference driver's time loop and stop conditions on the host.

``end_run`` restates for/tools.f90:41-69: a run stops when the wall time
since its start exceeds ``wall_time_limit``, when the simulated time has
reached ``time_limit``, or when a file ``stop.now`` exists in the run
directory (every condition that holds is reported, as the reference prints
each).  ``run`` is the loop of for/diablo.f90:62-129 over a Channel: one
time step (three RK substeps, time += dt), the stop check, the statistics
and flow saves when their times are reached (after which the save times
advance by their intervals and the device's next-event dt scheduling is
told), and the exit once a stop condition held.

Beyond the reference, the loop reads the library's status after every step
and ends the run with ``FlowError`` when the device flagged a non-finite
state or a bounded device wait that gave up: the reference has no such
check and would carry NaNs on.
"""
from __future__ import annotations

import math
import os
import time as _time
from dataclasses import dataclass, field

FLAG_NONFINITE = 1
FLAG_DT_NONPOS = 2
FLAG_WAIT_TIMEOUT = 16

STOP_FILE = "stop.now"


class FlowError(RuntimeError):
    """The device reported a state the run cannot continue from."""

    def __init__(self, flags: int, time_step: int):
        what = []
        if flags & FLAG_NONFINITE:
            what.append("non-finite velocity or buoyancy")
        if flags & FLAG_DT_NONPOS:
            what.append("courant found dt <= 0")
        if flags & FLAG_WAIT_TIMEOUT:
            what.append("a bounded device wait gave up (the step's data are invalid)")
        super().__init__(f"step {time_step}: " + "; ".join(what))
        self.flags = flags
        self.time_step = time_step


def end_run(time: float, elapsed_wall: float, wall_time_limit: float, time_limit: float,
            run_dir: str = ".") -> list[str]:
    """Stop conditions of end_run (for/tools.f90:41-69): a list of the
    reasons that hold, empty when the run goes on."""
    why = []
    if elapsed_wall > wall_time_limit:
        why.append("wall-time")
    if time >= time_limit:
        why.append("time-limit")
    if os.path.exists(os.path.join(run_dir, STOP_FILE)):
        why.append(STOP_FILE)
    return why


@dataclass
class RunResult:
    steps: int = 0                      # time steps taken by this call
    reasons: list = field(default_factory=list)   # why it stopped (empty: max_steps reached)
    stats_saved: int = 0
    flows_saved: int = 0
    time: float = 0.0
    time_step: int = 0


def run(ch, wall_time_limit: float = math.inf, time_limit: float | None = None, run_dir: str = ".",
        save_stats=None, save_flow=None, max_steps: int | None = None, clock=_time.monotonic,
        save_stats_time: float | None = None, save_flow_time: float | None = None) -> RunResult:
    """Advance `ch` until a stop condition of end_run holds (or max_steps).

    save_stats(ch) / save_flow(ch) are called when the simulated time
    reaches the next save time (diablo.f90:87-123); the save times start at
    the given values (default: the current time plus the interval) and then
    advance by p.save_stats_dt / p.save_flow_dt.  time_limit defaults to
    p.time_limit.  clock is the wall clock (seconds), replaceable in tests.
    """
    p = ch.p
    tlim = p.time_limit if time_limit is None else time_limit
    st = ch.status()
    sst = st.time + p.save_stats_dt if save_stats_time is None else save_stats_time
    sft = st.time + p.save_flow_dt if save_flow_time is None else save_flow_time
    ch.set_clock(st.time, st.time_step, sst, sft)   # the device schedules dt to hit them
    res = RunResult(time=st.time, time_step=st.time_step)
    start = clock()
    while max_steps is None or res.steps < max_steps:
        ch.step(1)
        res.steps += 1
        st = ch.status()
        res.time, res.time_step = st.time, st.time_step
        bad = st.flags & (FLAG_NONFINITE | FLAG_DT_NONPOS | FLAG_WAIT_TIMEOUT)
        if bad:
            raise FlowError(bad, st.time_step)
        why = end_run(st.time, clock() - start, wall_time_limit, tlim, run_dir)
        moved = False
        if st.time >= sst:
            if save_stats is not None:
                save_stats(ch)
            res.stats_saved += 1
            sst += p.save_stats_dt
            moved = True
        if st.time >= sft:
            if save_flow is not None:
                save_flow(ch)
            res.flows_saved += 1
            sft += p.save_flow_dt
            moved = True
        if moved:
            ch.set_clock(st.time, st.time_step, sst, sft)
        if why:
            res.reasons = why
            break
    return res


__all__ = ["end_run", "run", "RunResult", "FlowError", "STOP_FILE"]
