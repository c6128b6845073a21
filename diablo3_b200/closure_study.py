"""A-posteriori study of the learned closure at the config-3 size, with
training data from a resolved run.

The flow is config 3's finite front (IC 6, width 0.5, Re 1e4).  A resolved
FP64 DNS at 512x257x512 (no closure) is spun up from seeded noise; its
state is box-filtered 4x4x4 onto the 128x65x128 LES grid by
``db_sgs_targets`` at several times (features and the least-squares
nu_t, kappa_t of the exact filtered stress and flux), and the 16-64-64-64-2
network is trained on them with the tensor-core Adam (``sgs_train``).  For
each evaluation seed another resolved realisation is spun up, filtered
onto the LES grid (``les_filter``), and continued; from the same filtered
state an FP64 AMD LES (les_model_type 5) and a mixed-precision LES with the
learned closure (les_model_type 6) advance over the same window with the
same fixed dt.  After every window the change of the horizontal-mean u1,
u3 and buoyancy profiles since the common start is compared with that of
the filtered resolved run (relative L2 over the rows away from the walls).

``run()`` returns the per-seed, per-window errors and their sums, and the
network's parameters with its normalisation (``save_net`` / ``load_net``
keep them in an .npz file).  ``diablo3_b200/data/closure_config3.npz`` is
the network of ``run(nsnap=6, train_steps=4000)`` (the 128x65x128 bench
comparison loads it); regenerate it with
``python -m diablo3_b200.closure_study diablo3_b200/data/closure_config3.npz``.
"""
from __future__ import annotations

import numpy as np

FX = FY = FZ = 4


def dns_params(nx: int = 512, ny: int = 257, nz: int = 512, dt: float = 2e-3, kick: float = 0.05):
    """Config 3's flow, resolved (no closure), fixed dt."""
    from .workloads import workload_params
    p = workload_params("config3")
    p.nx, p.ny, p.nz = nx, ny, nz
    p.use_les, p.variable_dt, p.delta_t, p.kick = 0, 0, dt, kick
    return p


def les_params(model: int, precision: int, nx: int = 128, ny: int = 65, nz: int = 128, dt: float = 2e-3):
    """Config 3's LES (les_model_type 5 or 6), fixed dt, the closure on
    from the first step."""
    from .workloads import workload_params
    p = workload_params("config3")
    p.nx, p.ny, p.nz = nx, ny, nz
    p.use_les, p.les_model_type, p.create_new_flow = 1, model, 0
    p.variable_dt, p.delta_t, p.precision = 0, dt, precision
    return p


def _grid(n):
    from .grid import create_grid
    return create_grid(n, lz=2.0, cs=1.5, grid_type=1)


def save_net(path: str, net_state: dict) -> None:
    np.savez(path, **net_state)


def load_net(path: str):
    """An SgsNet with the parameters, normalisation and training range
    stored by save_net."""
    from .sgs_net import SgsNet
    d = np.load(path)
    net = SgsNet()
    net.set(d["params"], d["mean"], d["std"], d["scale"])
    net.set_range(d["lo"], d["hi"])
    return net


def training_set(p_dns, gy_les, seed: int, spinup: int, nsnap: int, every: int):
    """Filtered training data (CUDA tensors) from one resolved realisation."""
    import torch
    from .channel import Channel
    ch = Channel(p_dns, _grid(p_dns.ny))
    ch.init_flow(seed=seed)
    ch.step(spinup)
    snaps = []
    for _ in range(nsnap):
        ch.step(every)
        snaps.append(ch.sgs_targets(gy_les, FX, FY, FZ))
    ch.close()
    feat = torch.cat([s[0] for s in snaps]).contiguous()
    tgt = torch.cat([s[1] for s in snaps]).contiguous()
    return feat, tgt


def train_net(feat, tgt, steps: int, lr: float = 2e-3, seed: int = 1):
    """Tensor-core Adam on the whole set; returns the net, its stored state
    and the loss history."""
    from . import sgs_train
    net, losses = sgs_train.train(feat, tgt, steps=steps, batch=1 << 30, lr=lr, seed=seed)
    fh = feat.detach().cpu().numpy()
    th = tgt.detach().cpu().numpy()
    mean, std = sgs_train.normalisation(fh)
    scale = np.sqrt(np.mean(th.astype(np.float64) ** 2, axis=0)).astype(np.float32)
    scale = np.where(scale > 0, scale, 1.0).astype(np.float32)
    lo, hi = sgs_train.training_range(fh)
    state = {"params": net.get(), "mean": mean, "std": std, "scale": scale, "lo": lo, "hi": hi}
    return net, state, losses


def aposteriori(net, p_dns, seed: int, spinup: int, windows: int, every: int):
    """AMD (FP64) and learned (mixed) LES against the filtered resolved run
    of one realisation: per window, the evolution errors of the mean u1, u3
    and buoyancy profiles."""
    from . import les_filter
    from .channel import Channel
    gy_f, gy_c = _grid(p_dns.ny), _grid(p_dns.ny // FY + 1)
    dns = Channel(p_dns, gy_f)
    dns.init_flow(seed=seed)
    dns.step(spinup)
    pa = les_params(5, 0, p_dns.nx // FX, p_dns.ny // FY + 1, p_dns.nz // FZ, p_dns.delta_t)
    pl = les_params(6, 1, p_dns.nx // FX, p_dns.ny // FY + 1, p_dns.nz // FZ, p_dns.delta_t)
    fields = les_filter.filter_state_to_les(dns, pa, gy_c, FX)
    amd = Channel(pa, gy_c)
    amd.init_flow(fields=fields)
    lrn = Channel(pl, gy_c)
    lrn.set_sgs_net(net)
    lrn.init_flow(fields=fields)
    rows = slice(2, pa.ny)
    ref0 = les_filter.filtered_mean_profiles(dns, gy_c)
    a0, l0 = les_filter.mean_profiles(amd), les_filter.mean_profiles(lrn)
    out = []
    for _ in range(windows):
        dns.step(every)
        amd.step(every)
        lrn.step(every)
        ref = les_filter.filtered_mean_profiles(dns, gy_c)
        e_a = les_filter.evolution_errors(les_filter.mean_profiles(amd), a0, ref, ref0, rows)
        e_l = les_filter.evolution_errors(les_filter.mean_profiles(lrn), l0, ref, ref0, rows)
        out.append({"amd": e_a, "learned": e_l})
    flags = (amd.status().flags, lrn.status().flags)
    for ch in (dns, amd, lrn):
        ch.close()
    return out, flags


def run(nx: int = 512, ny: int = 257, nz: int = 512, train_seed: int = 6, eval_seeds=(5, 7),
        spinup: int = 300, nsnap: int = 4, every: int = 50, windows: int = 4, train_steps: int = 1500,
        dt: float = 2e-3, net_path: str | None = None):
    p = dns_params(nx, ny, nz, dt)
    gy_c = _grid(ny // FY + 1)
    feat, tgt = training_set(p, gy_c, train_seed, spinup, nsnap, every)
    net, state, losses = train_net(feat, tgt, train_steps)
    from . import sgs_train
    fit = sgs_train.compare_with_amd(net, feat, tgt)
    del feat, tgt
    if net_path:
        save_net(net_path, state)
    per_seed, flags = {}, {}
    tot = {"amd": 0.0, "learned": 0.0}
    by_field = {"amd": {}, "learned": {}}
    for sd in eval_seeds:
        res, fl = aposteriori(net, p, sd, spinup, windows, every)
        per_seed[sd], flags[sd] = res, fl
        for w in res:
            for arm in ("amd", "learned"):
                tot[arm] += sum(w[arm].values())
                for k, v in w[arm].items():
                    by_field[arm][k] = by_field[arm].get(k, 0.0) + v
    net.close()
    return {"loss_first": float(losses[0]), "loss_last": float(losses[-1]), "fit_vs_targets": fit,
            "per_seed": per_seed, "flags": flags, "total": tot, "by_field": by_field,
            "setup": {"dns": [nx, ny, nz], "les": [nx // FX, ny // FY + 1, nz // FZ], "dt": dt,
                      "spinup": spinup, "snapshots": nsnap, "every": every, "windows": windows,
                      "train_steps": train_steps, "train_seed": train_seed, "eval_seeds": list(eval_seeds)}}


__all__ = ["dns_params", "les_params", "save_net", "load_net", "training_set", "train_net", "aposteriori", "run"]


if __name__ == "__main__":
    import json
    import sys
    out = sys.argv[1] if len(sys.argv) > 1 else "closure_config3.npz"
    r = run(nsnap=6, train_steps=4000, net_path=out)
    print(json.dumps({k: r[k] for k in ("loss_first", "loss_last", "fit_vs_targets", "total", "by_field", "setup")},
                     default=str))
