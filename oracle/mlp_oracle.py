"""CPU oracle of the learned SGS closure's MLP (TEST INFRASTRUCTURE: only
tests/ may use it).  It states the network and its gradient in numpy, with
the same BF16 roundings as the tensor-core kernels: inputs, hidden
activations, weights of the three tensor-core layers and the back-propagated
dz of those layers are rounded to BF16 (round to nearest even), products are
summed in float64 (the device sums in FP32).  `quantized=False` gives the
plain FP64 network for finite-difference checks.
"""
from __future__ import annotations

import numpy as np

OFF = {"W1": (0, (64, 16)), "b1": (1024, (64,)), "W2": (1088, (64, 64)), "b2": (5184, (64,)),
       "W3": (5248, (64, 64)), "b3": (9344, (64,)), "W4": (9408, (2, 64)), "b4": (9536, (2,))}
NPARAMS = 9538


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    return {k: p[o:o + int(np.prod(sh))].reshape(sh) for k, (o, sh) in OFF.items()}


GELU_K = np.sqrt(2.0 / np.pi)
GELU_C = 0.044715


def gelu(x):
    """GELU, tanh form (Hendrycks & Gimpel 2016), as the closure kernels use it."""
    return 0.5 * x * (1.0 + np.tanh(GELU_K * (x + GELU_C * x ** 3)))


def gelu_d(x):
    t = np.tanh(GELU_K * (x + GELU_C * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_K * (1.0 + 3.0 * GELU_C * x * x)


def softplus(y):
    return np.where(y > 20.0, y, np.log1p(np.exp(np.minimum(y, 20.0))))


def sigmoid(y):
    return 1.0 / (1.0 + np.exp(-y))


def forward(params, feat, mean, std, out_scale, quantized=True):
    """Returns (out[n][2], cache)."""
    q = bf16 if quantized else (lambda a: np.asarray(a, np.float64))
    P = unpack(params)
    x = q((np.asarray(feat, np.float64) - mean) / std)
    W1, W2, W3 = q(P["W1"]), q(P["W2"]), q(P["W3"])
    z1 = x @ W1.T + P["b1"]
    h1 = q(gelu(z1))
    z2 = h1 @ W2.T + P["b2"]
    h2 = q(gelu(z2))
    z3 = h2 @ W3.T + P["b3"]
    h3 = gelu(z3)
    y = h3 @ P["W4"].T + P["b4"]
    out = softplus(y) * out_scale
    return out, dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3, y=y, W2=W2, W3=W3, P=P)


def loss_and_grad(params, feat, target, mean, std, out_scale, quantized=True):
    """Mean over points of the summed squared error of both outputs, and its
    gradient with respect to the packed parameters."""
    q = bf16 if quantized else (lambda a: np.asarray(a, np.float64))
    out, c = forward(params, feat, mean, std, out_scale, quantized)
    n = out.shape[0]
    e = out - target
    loss = float(np.sum(e * e) / n)
    dy = (2.0 / n) * e * out_scale * sigmoid(c["y"])
    P = c["P"]
    g = {}
    g["W4"] = dy.T @ c["h3"]
    g["b4"] = dy.sum(0)
    dz3 = q((dy @ P["W4"]) * gelu_d(c["z3"]))
    g["W3"] = dz3.T @ c["h2"]
    g["b3"] = dz3.sum(0)
    dz2 = q((dz3 @ c["W3"]) * gelu_d(c["z2"]))
    g["W2"] = dz2.T @ c["h1"]
    g["b2"] = dz2.sum(0)
    dz1 = q((dz2 @ c["W2"]) * gelu_d(c["z1"]))
    g["W1"] = dz1.T @ c["x"]
    g["b1"] = dz1.sum(0)
    grad = np.zeros(NPARAMS)
    for k, (o, sh) in OFF.items():
        grad[o:o + int(np.prod(sh))] = np.asarray(g[k]).reshape(-1)
    return loss, grad
