#!/usr/bin/env python
"""Throughput of DIABLO's channel RK substep (RKW3 + CN, rk_chan_1) on B200.

Metric: grid-point RK substeps per second, whole job.  A bench step is one
full RKW3 time step (three substeps) of the 512x257x512 FP64 DNS (infinite
front, Re 5000, Ri 1, CFL 0.5 with variable dt), state resident in HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With the defaults the line also carries, measured in the same run, the
metric's second arm: ``mixed_dns`` (the same DNS on the mixed-precision
path) and ``config3`` (the 128x65x128 LES, FP64 AMD against the mixed
learned closure, per unit simulated time).

N > 1 runs N independent replicas (one per GPU, launched by torchrun): the
substep has no data-parallel exchange on one instance, so nothing is sharded
and no collective sits on the data path; rank timings are reduced with MAX.
"""
from __future__ import annotations

import argparse
import json

import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt RK substeps/s on 1 B200: FP64 plain vs mixed+learned SGS at stated err"
UNIT = "grid-pt substeps/s"


from diablo3_b200.workloads import WORKLOAD_DESC, workload_params  # noqa: E402


def workload_suffix(args) -> str:
    s = ""
    if args.les:
        s += ", AMD LES (les_model_type 5) on every substep"
    if args.precision == "mixed":
        s += ", mixed precision (FP32 transforms/products/SGS; FP64 state, CN and Poisson solves)"
    return s


L2_BYTES = 126e6


def resident_bytes(p) -> float:
    """Device bytes of one context's fields (what db_init allocates for the
    state, scratch and, with LES, the closure arrays)."""
    from diablo3_b200 import roofline
    u = roofline.units(p)
    S, X, P = u["S"], u["Xh"], u["P"]
    b = 15 * S + 8 * X + 8 * P
    if getattr(p, "use_les", 0):
        pts = p.nx * p.nz * (p.ny + 2)
        # 21 physical closure fields, FP64 solve scratch (8 fields), ghost
        # overlay (16 spectral planes sets), features + outputs (18 FP32)
        b += 21 * P + 8 * 8 * pts + 16 * S + 18 * 4 * pts
        if not getattr(p, "precision", 0):
            b += 8 * S   # FP64 z-pass scratch
    return float(b)


def l2_note(b: float) -> str:
    if b > 10 * L2_BYTES:
        return f"fields ~{b / 1e9:.1f} GB resident in HBM, far above the 126 MB L2 (no flush needed)"
    if b > L2_BYTES:
        return (f"fields ~{b / 1e6:.0f} MB resident in HBM, above the 126 MB L2; every step streams all of "
                f"them, but single kernels' inputs can be L2 hits (no flush)")
    return f"fields ~{b / 1e6:.0f} MB: L2-resident (latency case, not an HBM measurement)"


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU baseline: the oracle (C restatement of the reference) on host cores

def cpu_baseline(name: str, min_seconds: float = 10.0) -> dict:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from diablo3_b200.grid import create_grid
    from diablo3_b200.ic import initial_fields
    p = workload_params(name)
    if name == "config1":
        p.ny = 65  # bounded sample: full x-z planes, fewer wall-normal points
    gy = create_grid(p.ny, lz=p.ly, cs=1.5, grid_type=1)
    o = pyoracle.Oracle(p, gy)
    o.init_from_physical(*initial_fields(p, gy, seed=0))
    n = p.nx * p.ny * p.nz
    count, t0 = 0, time.perf_counter()
    while True:
        o.rk_substep(count % 3 + 1)
        count += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or count >= 30:
            break
    o.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n * count / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{count} substeps of {p.nx}x{p.ny}x{p.nz} (same x-z planes as the workload, "
                      f"{p.ny} of its wall-normal points), {el:.1f} s, OpenMP C oracle"}


def run_reference(args) -> None:
    from diablo3_b200 import replicas
    if not replicas.from_env().leader:   # under torchrun rank 0 alone runs and prints it
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    per = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(args.config, min_seconds=2.0)
        if i >= args.warmup:
            per.append(r)
    v = statistics.median(x["value"] for x in per)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC[args.config], "parallelism": "host cores"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": per[0]["cores"], "kind": "port",
                         "sample": per[0]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# config 4: 64 independent 128x65x128 channels, one graph launch per step;
# the members are batched (each kernel of the step launched once for all)

def run_ensemble(args) -> None:
    import torch
    from diablo3_b200 import roofline
    from diablo3_b200.ensemble import Ensemble, config4_members
    from diablo3_b200.grid import create_grid
    n_inst = int(os.environ.get("DB_ENSEMBLE_N", "64"))
    prec = 0 if args.precision == "fp64" else 1
    ps, ri = config4_members(n_inst, precision=prec)
    gy = create_grid(ps[0].ny, lz=ps[0].ly, cs=1.5, grid_type=1)
    stream = torch.cuda.Stream()
    ens = Ensemble(ps, gy, stream=stream.cuda_stream)

    def timed():
        for _ in range(args.warmup):
            ens.step(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ens.step(1)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    batched, groups = ens.batched, ens.groups
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    time.sleep(0.5)
    ms = timed()
    clk = clocks.stop()
    kps = ens.kernels_per_step()
    branches = one_group = None

    def other(g):
        ens.groups = g
        ms_o = timed()
        return {"ms_per_step": ms_o / args.steps, "kernels_per_step": ens.kernels_per_step(),
                "value": n_inst * ps[0].nx * ps[0].ny * ps[0].nz * 3 * args.steps / (ms_o / 1e3)}

    if batched and not args.no_extras:   # the other forms on the same members, for comparison
        if groups > 1:
            one_group = other(1)
        branches = other(0)
    p0 = ps[0]
    npts = p0.nx * p0.ny * p0.nz
    value = n_inst * npts * 3 * args.steps / (ms / 1e3)
    peak, peak_kind = measured_peak_hbm()
    alg = roofline.substep_bytes(p0) * n_inst
    achieved = alg / (ms / args.steps / 3 / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == 0 else "f32+f64", "data": "synthetic (seeded infinite-front ICs, no dataset)",
        "config": {"workload": f"ensemble of {n_inst} independent {p0.nx}x{p0.ny}x{p0.nz} channels (seed i, "
                               f"Ri_i ~ U[0.5, 2], Re 2000), one CUDA graph launch per time step"
                               + (", mixed precision" if prec else ""),
                   "instances": n_inst, "grid_xyz": [p0.nx, p0.ny, p0.nz], "points": n_inst * npts,
                   "parallelism": (f"single GPU, members batched in {groups} groups: each kernel launched once "
                                   f"per group, the groups on parallel graph branches"
                                   if batched else "single GPU, one graph branch per member"),
                   "l2": l2_note(n_inst * resident_bytes(p0))},
        "roofline": {"bound": "hbm", "kernel": "whole step, all members", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None},
        "clocks": clk,
        "gpu_launches": kps * args.steps,
        "per_member_graphs": branches,
        "one_group": one_group,
    }
    print(json.dumps(line), flush=True)
    ens.close()


def _timed_run(ch, stream, steps, warmup):
    """Warm-up, then `steps` steps timed with CUDA events; returns
    (ms per step, simulated time advanced per wall second)."""
    import torch
    for _ in range(warmup):
        ch.step(1)
    torch.cuda.synchronize()
    t0 = ch.status().time
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ch.step(1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st = ch.status()
    if st.flags & 1:
        raise SystemExit("non-finite values in the flow: run rejected")
    return ms / steps, (st.time - t0) / (ms / 1e3)


def _dns_timed(ch, p, stream, steps, rk, local, precision, les):
    """Time `steps` steps of a warmed-up channel: CUDA events around the
    region (max over ranks), stage events inside the step graph, clocks
    sampled meanwhile; the dominant stage's roofline against the measured
    HBM copy bandwidth."""
    import ctypes

    import numpy as np
    import torch

    from diablo3_b200 import lib as L
    from diablo3_b200 import replicas, roofline
    ch._ck(ch.L.db_set_timing(ch.h, 1))
    ch.step(1)  # capture the timed graph (not timed)
    torch.cuda.synchronize()
    n0 = ctypes.c_longlong()
    ch._ck(ch.L.db_kernel_launches(ch.h, ctypes.byref(n0)))
    stage_ms = np.zeros(len(L.STAGES))
    buf = (ctypes.c_double * len(L.STAGES))()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    replicas.barrier(rk)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        ch.step(1)
        ch._ck(ch.L.db_stage_times(ch.h, buf, len(L.STAGES)))
        stage_ms += np.array(buf[:])
    ev1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier(rk)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    ch._ck(ch.L.db_set_timing(ch.h, 0))
    n1 = ctypes.c_longlong()
    ch._ck(ch.L.db_kernel_launches(ch.h, ctypes.byref(n1)))
    ms_max = replicas.max_over_ranks(rk, ms)
    npts = p.nx * p.ny * p.nz
    value = replicas.job_rate(npts, 3 * steps, rk, ms_max)
    if ch.status().flags & 1:
        raise SystemExit("non-finite values in the flow: run rejected")
    peak, peak_kind = measured_peak_hbm()
    per_stage = stage_ms / (3 * steps)  # ms per launch (per substep)
    dom = int(np.argmax(per_stage))
    dom_name = L.STAGES[dom]
    alg = roofline.stage_bytes(p)[dom_name]
    achieved = alg / (per_stage[dom] / 1e3) / 1e9
    traffic = None if les else roofline.profiled_traffic(dom_name, ROOT, precision)
    t_sub = ms_max / steps / 3 / 1e3
    return {
        "ms_max": ms_max, "value": value, "clocks": clk, "gpu_launches": int(n1.value - n0.value),
        "stages_ms_per_substep": {L.STAGES[i]: round(float(per_stage[i]), 4) for i in range(len(L.STAGES))},
        "stages_note": ("without LES: zpass_rhs = the z-FFT of the product fields, thomas = the spectral "
                        "RHS joined with the CN solves, courant = the third substep's CFL transforms "
                        "(averaged over the three substeps)") if not getattr(p, "use_les", 0) else
                       "with LES: the reference's stage sequence (physical CN solves)",
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "alg_bytes_per_launch": alg,
                     "step_alg_bytes": roofline.substep_bytes(p),
                     "step_frac": roofline.substep_bytes(p) / t_sub / 1e9 / peak,
                     "ref_seq_bytes": roofline.reference_substep_bytes(p),
                     "ref_seq_frac": roofline.reference_substep_bytes(p) / t_sub / 1e9 / peak},
    }


def les_compare(config: str, steps: int, warmup: int, autotune: bool = True) -> dict:
    """Config 2 (256x129x256): FP64 AMD LES against the mixed-precision AMD
    LES.  Config 3 (128x65x128): FP64 AMD LES against the mixed-precision
    LES with the learned closure (les_model_type 6).  Both arms run the same
    IC with CFL-limited dt; the comparison is simulated time per wall second.
    The network of config 3 is the one trained on a resolved (512x257x512
    FP64) run of the same flow filtered onto this grid; its accuracy against
    the filtered resolved run is what the closure tests establish."""
    import torch
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import create_grid
    p64 = workload_params(config)
    gy = create_grid(p64.ny, lz=p64.ly, cs=1.5, grid_type=1)
    stream = torch.cuda.Stream()
    npts = p64.nx * p64.ny * p64.nz
    a = Channel(p64, gy, stream=stream.cuda_stream)
    a.init_flow(seed=0)
    if autotune:
        a.autotune()
    ms_a, rate_a = _timed_run(a, stream, steps, warmup)
    net = None
    if config == "config3":
        # the network trained on a 512x257x512 FP64 DNS of this flow filtered
        # 4x4x4 onto this grid (closure_study.run; weights in the package)
        from diablo3_b200 import closure_study
        net = closure_study.load_net(os.path.join(ROOT, "diablo3_b200", "data", "closure_config3.npz"))
    a.close()
    pm = workload_params(config)
    pm.precision = 1
    if net is not None:
        pm.les_model_type = 6
    b = Channel(pm, gy, stream=stream.cuda_stream)
    if net is not None:
        b.set_sgs_net(net)
    b.init_flow(seed=0)
    if autotune:
        b.autotune()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    time.sleep(0.5)
    ms_b, rate_b = _timed_run(b, stream, steps, warmup)
    clk = clocks.stop()
    b.close()
    arm_b = "mixed precision, learned closure (les_model_type 6)" if net is not None else "mixed precision, AMD"
    return {
        "workload": WORKLOAD_DESC[config] + "; " + arm_b + " vs FP64 AMD", "grid_xyz": [p64.nx, p64.ny, p64.nz],
        "points": npts, "l2": l2_note(resident_bytes(pm)), "steps": steps, "warmup": warmup,
        "fp64_amd": {"ms_per_step": ms_a, "sim_time_per_wall_s": rate_a,
                     "grid_pt_substeps_per_s": npts * 3 / (ms_a / 1e3)},
        "candidate": {"arm": arm_b, "ms_per_step": ms_b, "sim_time_per_wall_s": rate_b,
                      "grid_pt_substeps_per_s": npts * 3 / (ms_b / 1e3)},
        "speedup_per_unit_sim_time": rate_b / rate_a,
        "network": "trained on a 512x257x512 FP64 DNS of the flow filtered 4x4x4 onto this grid "
                   "(diablo3_b200/closure_study.py, weights diablo3_b200/data/closure_config3.npz)"
        if net is not None else None,
        "clocks": clk,
    }


def run_les_compare(args) -> None:
    c = les_compare(args.config, args.steps, args.warmup, not args.no_autotune)
    ms_b = c["candidate"]["ms_per_step"]
    line = {
        "metric": METRIC, "value": c["points"] * 3 / (ms_b / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_b, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded finite-front IC, no dataset)",
        "config": {"workload": c["workload"], "grid_xyz": c["grid_xyz"], "points": c["points"],
                   "parallelism": "single GPU", "l2": c["l2"]},
        "les_compare": {k: c[k] for k in ("fp64_amd", "candidate", "speedup_per_unit_sim_time", "network")},
        "clocks": c["clocks"],
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="config1", choices=["config1", "config0", "slab", "config2", "config3", "config4"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="mixed: FP32 transforms/products/SGS, FP64 state and solves (default: fp64; "
                         "config4, the closure-data ensemble, is defined in mixed precision)")
    ap.add_argument("--les", action="store_true", help="AMD LES closure (les_model_type 5) on")
    ap.add_argument("--no-autotune", action="store_true", help="keep the built-in launch shapes")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision DNS and the 128x65x128 LES comparison keys "
                         "(--config config4: the per-member graph comparison)")
    args = ap.parse_args()
    if args.precision is None:
        args.precision = "mixed" if args.config == "config4" else "fp64"
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.config == "config4":
        return run_ensemble(args)
    if args.config in ("config2", "config3"):
        return run_les_compare(args)

    import ctypes

    import numpy as np
    import torch

    from diablo3_b200 import lib as L
    from diablo3_b200 import roofline
    from diablo3_b200.channel import Channel
    from diablo3_b200.grid import create_grid

    from diablo3_b200 import replicas
    rk = replicas.from_env()
    world, rank, local = rk.world, rk.rank, rk.local
    torch.cuda.set_device(local)
    replicas.init(rk, "nccl")

    p = workload_params(args.config)
    if args.precision == "mixed":
        p.precision = 1
    if args.les:
        p.use_les, p.les_model_type, p.create_new_flow = 1, 5, 0
    gy = create_grid(p.ny, lz=p.ly, cs=1.5, grid_type=1)
    stream = torch.cuda.Stream()
    ch = Channel(p, gy, stream=stream.cuda_stream)
    ch.init_flow(seed=rank)
    npts = p.nx * p.ny * p.nz

    def barrier():
        replicas.barrier(rk)

    tuned = None
    if not args.no_autotune:   # launch shapes timed before the warm-up (not in the timed region)
        rep = ch.autotune()
        tuned = rep.strip().splitlines()[-1].replace("chosen: ", "")
    for _ in range(args.warmup):
        ch.step(1)
    torch.cuda.synchronize()

    dns = _dns_timed(ch, p, stream, args.steps, rk, local, args.precision, args.les)
    ms_max, value, clk = dns["ms_max"], dns["value"], dns["clocks"]

    # end to end through the C-ABI with host buffers: each step uploads the
    # fields a full RK step reads and downloads the ones it writes (U, V, W,
    # TH, P; the CF history is rebuilt inside the step)
    e2e = None
    if not args.no_e2e:
        host = {f: torch.empty(ch.new_spectral().shape, dtype=torch.complex128, pin_memory=True).numpy()
                for f in L.STEP_FIELDS}
        ke = max(1, min(3, args.steps))
        h2d_bytes, d2h_bytes = roofline.state_transfer_bytes(p, len(L.STEP_FIELDS))
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        saved = ch.download_state()
        for f in L.STEP_FIELDS:   # the first step's inputs, in the pinned buffers too
            host[f][...] = saved[f]
        e0.record(stream)
        for _ in range(ke):
            for f in L.STEP_FIELDS:
                ch.upload_field(f, host[f])
            ch.step(1)
            for f in L.STEP_FIELDS:
                ch._ck(ch.L.db_download_field(ch.h, f, L.dptr(host[f].view(np.float64).reshape(-1))))
        e1.record(stream)
        torch.cuda.synchronize()
        te = replicas.max_over_ranks(rk, e0.elapsed_time(e1))
        e2e = {"value": replicas.job_rate(npts, 3 * ke, rk, te), "unit": UNIT,
               "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
               "steps": ke, "path": "db_upload_field x5 (CU1, CU2, CU3, CP, CTH) + db_rk_steps(1) + "
                                    "db_download_field x5, reference-layout host arrays"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.config)

    # the metric's second arm in the same run (one GPU, the default workload):
    # the mixed-precision DNS, and the 128x65x128 LES comparison (FP64 AMD
    # against the mixed learned closure, per unit simulated time)
    extras = {}
    if world == 1 and not args.no_extras and args.config == "config1" and args.precision == "fp64" and not args.les:
        ch.close()
        ch = None
        ke = max(3, min(args.steps, 10))
        pm = workload_params("config1")
        pm.precision = 1
        chm = Channel(pm, gy, stream=stream.cuda_stream)
        chm.init_flow(seed=rank)
        tm = None
        if not args.no_autotune:
            tm = chm.autotune().strip().splitlines()[-1].replace("chosen: ", "")
        for _ in range(args.warmup):
            chm.step(1)
        torch.cuda.synchronize()
        dm = _dns_timed(chm, pm, stream, ke, rk, local, "mixed", False)
        chm.close()
        extras["mixed_dns"] = {
            "workload": WORKLOAD_DESC["config1"] + workload_suffix(argparse.Namespace(les=False, precision="mixed")),
            "value": dm["value"], "unit": UNIT, "steps": ke, "ms_per_step": dm["ms_max"] / ke,
            "dtype": "f32+f64", "launch_shapes": tm or "built-in defaults", "gpu_launches": dm["gpu_launches"],
            "stages_ms_per_substep": dm["stages_ms_per_substep"], "roofline": dm["roofline"],
            "clocks": dm["clocks"]}
        extras["config3"] = les_compare("config3", ke, args.warmup, not args.no_autotune)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded infinite-front IC, no dataset)",
        "config": {"workload": WORKLOAD_DESC[args.config] + workload_suffix(args), "grid_xyz": [p.nx, p.ny, p.nz],
                   "points": npts, "substeps_per_step": 3,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": l2_note(resident_bytes(p)),
                   "launch_shapes": tuned or "built-in defaults"},
        "gpu_launches": dns["gpu_launches"],
        "stages_ms_per_substep": dns["stages_ms_per_substep"],
        "roofline": dns["roofline"],
        "clocks": clk,
    }
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    line.update(extras)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ch is not None:
        ch.close()
    replicas.finish(rk)


if __name__ == "__main__":
    main()
