"""Tensor-core MLP of the learned SGS closure against its CPU oracle.

The oracle (oracle/mlp_oracle.py) repeats the kernels' BF16 roundings, so
the comparison isolates FP32-vs-FP64 summation and the rare BF16 rounding
that lands on the other side of a tie: GEMM tiles 1e-5 relative, network
outputs 2e-3 relative L2, gradients 1e-2 relative L2 per parameter block.
Against the unrounded FP64 network (central differences) the bar is 5e-2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def mods():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import mlp_oracle
    from diablo3_b200 import sgs_net
    return sgs_net, mlp_oracle


def _bits(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def _from_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("K,N", [(16, 64), (64, 64), (128, 80), (128, 32), (256, 256)])
def test_tensor_core_gemm_tile(mods, K, N):
    sgs_net, _ = mods
    rng = np.random.default_rng(K * 1000 + N)
    a = _bits(rng.standard_normal((128, K)))
    b = _bits(rng.standard_normal((N, K)))
    d = sgs_net.gemm_check(a, b)
    ref = _from_bits(a) @ _from_bits(b).T
    assert np.abs(d - ref).max() <= 1e-5 * np.abs(ref).max() * np.sqrt(K)


def _problem(n, seed):
    rng = np.random.default_rng(seed)
    feat = rng.standard_normal((n, 16)).astype(np.float32) * 2.0 + 0.5
    mean = np.full(16, 0.5, np.float32)
    std = np.full(16, 2.0, np.float32)
    scale = np.array([1e-3, 2e-3], np.float32)
    w = rng.standard_normal((2, 16)) / 4.0
    tgt = (np.log1p(np.exp((feat - mean) / std @ w.T)) * scale).astype(np.float32)
    return feat, tgt, mean, std, scale


def test_forward_matches_oracle(mods):
    sgs_net, orc = mods
    n = 1000   # not a multiple of 128: padded last tile
    feat, _, mean, std, scale = _problem(n, 1)
    params = sgs_net.init_params(3)
    net = sgs_net.SgsNet()
    net.set(params, mean, std, scale)
    out = net.forward(torch.from_numpy(feat).cuda()).cpu().numpy()
    ref, _ = orc.forward(params, feat, mean, std, scale)
    assert np.linalg.norm(out - ref) <= 2e-3 * np.linalg.norm(ref)


def test_gradient_matches_oracle_and_finite_differences(mods):
    sgs_net, orc = mods
    n = 4096 + 77
    feat, tgt, mean, std, scale = _problem(n, 2)
    params = sgs_net.init_params(4)
    net = sgs_net.SgsNet()
    net.set(params, mean, std, scale)
    g, loss = net.gradient(torch.from_numpy(feat).cuda(), torch.from_numpy(tgt).cuda())
    lq, gq = orc.loss_and_grad(params, feat, tgt, mean, std, scale, quantized=True)
    assert abs(loss - lq) <= 1e-3 * lq
    for k, (o, sh) in orc.OFF.items():
        sl = slice(o, o + int(np.prod(sh)))
        assert np.linalg.norm(g[sl] - gq[sl]) <= 1e-2 * np.linalg.norm(gq[sl]), k
    # the rounded gradient is close to the exact FP64 gradient
    _, g64 = orc.loss_and_grad(params, feat, tgt, mean, std, scale, quantized=False)
    assert np.linalg.norm(g - g64) <= 5e-2 * np.linalg.norm(g64)


def test_training_reduces_loss(mods):
    sgs_net, _ = mods
    n = 65536
    feat, tgt, mean, std, scale = _problem(n, 5)
    net = sgs_net.SgsNet()
    net.set(sgs_net.init_params(6), mean, std, scale)
    f, t = torch.from_numpy(feat).cuda(), torch.from_numpy(tgt).cuda()
    losses = [net.train_step(f, t, lr=3e-3) for _ in range(300)]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.05 * losses[0], (losses[0], losses[-1])
