"""Training and evaluation of the learned SGS closure.

The data come from resolved runs of this code: Channel.sgs_targets box-filters
the state onto the LES grid and fits nu_t, kappa_t to the exact subgrid
stress and flux.  Training runs on the tensor cores (SgsNet.train_step).
The reference closure, AMD (les_model_type 5), is both the fallback outside
the training range and the yardstick: `amd_from_features` evaluates its
eddy coefficients on the same filtered gradients and filter widths.
"""
from __future__ import annotations

import numpy as np

from .sgs_net import NFEAT, SgsNet, init_params

C_AMD = 0.2887   # for/les.f90:25


def amd_from_features(feat: np.ndarray):
    """AMD nu_t and kappa_t (for/les.f90:574-795, 1216-1358 in tensor form)
    from closure features: gradients G_ik = du_i/dx_k, scalar gradient g,
    filter widths (delta_x, delta_y, delta_z)."""
    f = np.asarray(feat, np.float64)
    G = f[:, 0:9].reshape(-1, 3, 3)
    g = f[:, 9:12]
    d = f[:, 12:15]
    D = G * (d[:, None, :] / d[:, :, None])
    S = 0.5 * (D + D.transpose(0, 2, 1))
    W = 0.5 * (D - D.transpose(0, 2, 1))
    num = -np.einsum("nij,njk,nki->n", S, S, S) + np.einsum("nij,njk,nki->n", S, W, W)
    den = np.einsum("nij,nij->n", D, D)
    coef = C_AMD ** 2 * 3.0 / np.sum(1.0 / d ** 2, axis=1)
    nu = coef * np.where((num > 0) & (den > 0), num / np.where(den > 0, den, 1.0), 0.0)
    d2 = d ** 2
    numt = -np.einsum("ni,nik,nk,nk->n", g, G, d2, g)
    dent = np.einsum("nk,nk->n", d2, g * g)
    ka = coef * np.where((numt > 0) & (dent > 0), numt / np.where(dent > 0, dent, 1.0), 0.0)
    return nu, ka


def normalisation(feat: np.ndarray):
    """Per-feature mean and standard deviation (1 for constant features)."""
    f = np.asarray(feat, np.float64)
    mean = f.mean(axis=0)
    std = f.std(axis=0)
    std = np.where(std > 1e-12 * (np.abs(mean) + 1e-30), std, np.maximum(np.abs(mean), 1.0))
    return mean.astype(np.float32), std.astype(np.float32)


def training_range(feat: np.ndarray, margin: float = 0.05):
    """Feature bounds of the training set, widened by `margin` of the span."""
    f = np.asarray(feat, np.float64)
    lo, hi = f.min(axis=0), f.max(axis=0)
    span = np.maximum(hi - lo, 1e-12 * (np.abs(hi) + 1.0))
    return (lo - margin * span).astype(np.float32), (hi + margin * span).astype(np.float32)


def train(feat, target, steps: int = 500, batch: int = 65536, lr: float = 1e-3, seed: int = 0,
          net: SgsNet | None = None, log_every: int = 0):
    """Fit a network to (features, targets) given as CUDA tensors; returns
    the network and the loss history (mean squared error per batch)."""
    import torch
    fh = feat.detach().cpu().numpy()
    th = target.detach().cpu().numpy()
    mean, std = normalisation(fh)
    scale = np.sqrt(np.mean(th.astype(np.float64) ** 2, axis=0)).astype(np.float32)
    scale = np.where(scale > 0, scale, 1.0).astype(np.float32)
    net = net or SgsNet()
    net.set(init_params(seed), mean, std, scale)
    lo, hi = training_range(fh)
    net.set_range(lo, hi)
    n = feat.shape[0]
    g = torch.Generator(device=feat.device).manual_seed(seed)
    losses = []
    for it in range(steps):
        if batch >= n:
            fb, tb = feat, target
        else:
            idx = torch.randint(0, n, (batch,), device=feat.device, generator=g)
            fb, tb = feat[idx].contiguous(), target[idx].contiguous()
        losses.append(net.train_step(fb, tb, lr=lr))
        if log_every and it % log_every == 0:
            print(f"step {it}: loss {losses[-1]:.4e}", flush=True)
    return net, np.array(losses)


def relative_errors(pred: np.ndarray, target: np.ndarray):
    """Relative L2 error per output column."""
    p = np.asarray(pred, np.float64)
    t = np.asarray(target, np.float64)
    return [float(np.linalg.norm(p[:, q] - t[:, q]) / max(np.linalg.norm(t[:, q]), 1e-300)) for q in range(t.shape[1])]


def compare_with_amd(net: SgsNet, feat, target):
    """Relative errors of the network and of AMD against the filtered-DNS
    targets on the same points: {'net': [nu, kappa], 'amd': [nu, kappa]}."""
    out = net.forward(feat).detach().cpu().numpy()
    fh = feat.detach().cpu().numpy()
    th = target.detach().cpu().numpy()
    nu, ka = amd_from_features(fh)
    return {"net": relative_errors(out, th), "amd": relative_errors(np.stack([nu, ka], 1), th)}


__all__ = ["amd_from_features", "normalisation", "training_range", "train", "compare_with_amd",
           "relative_errors", "NFEAT"]
