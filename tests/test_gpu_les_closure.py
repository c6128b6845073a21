"""les_model_type 6: the learned closure inside the channel substep.

Checks: the closure features the substep hands to the network equal a numpy
evaluation from the same state (FP32 storage: 1e-6 relative); with every
point outside the training range the substep is the AMD substep (1e-13);
with no range limit nu_t / kappa_t inside the channel are the network's
outputs on those features (1e-6, FP64 and FP32 fields); and a run with the closure stays finite
and divergence free.
"""
import numpy as np
import pytest

from _util import STATE, channel_state, config0_params, gradients_at_gy, grid_for, rel_l2, seed_pair

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def Channel():
    from diablo3_b200.channel import Channel
    return Channel


def les_params(model=5, **kw):
    base = dict(nx=32, ny=33, nz=32, use_les=1, create_new_flow=0, les_model_type=model, kick=0.05, re=5000.0)
    base.update(kw)
    return config0_params(**base)


def _net(seed=1, scale=1e-4):
    from diablo3_b200 import sgs_net
    net = sgs_net.SgsNet()
    mean = np.zeros(16, np.float32)
    std = np.ones(16, np.float32)
    std[12:15] = 0.1
    net.set(sgs_net.init_params(seed) * 0.3, mean, std, np.array([scale, scale], np.float32))
    return net


def test_closure_features_match_numpy(oracle_mod, Channel):
    p = les_params()
    gy = grid_for(p)
    o, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=31)
    c = {f: o.cplx(f).copy() for f in (0, 1, 2, 4)}
    met = {k: o.metric(i, p.ny + 2) for i, k in enumerate(("gy", "gyf", "dy", "dyf"))}
    kx = o.metric(4, p.nxp)[: p.nkx + 1]
    kz = o.metric(5, 2 * p.nkz + 1)
    G, gt = gradients_at_gy(p, c, met, kx, kz)
    _, _, feat = ch.les_eval(5, features=True)
    dx, dz = p.lx / p.nx, p.lz / p.nz
    for j in range(3, p.ny):
        ref = np.empty((p.nz, p.nx, 16))
        for i in range(3):
            for k in range(3):
                ref[..., 3 * i + k] = G[i, k, j]
        ref[..., 9:12] = np.moveaxis(gt[:, j], 0, -1)
        ref[..., 12], ref[..., 13], ref[..., 14] = 3 * dx, 2 * met["dy"][j], 3 * dz
        ref[..., 15] = gt[1, j]
        err = np.abs(feat[j] - ref).max(axis=(0, 1))
        scale = np.abs(ref).max(axis=(0, 1)) + 1e-30
        assert np.all(err <= 1e-6 * scale + 1e-30), (j, err / scale)


def test_closure_outside_range_is_amd(oracle_mod, Channel):
    p5, p6 = les_params(5), les_params(6)
    gy = grid_for(p5)
    o, ch5 = seed_pair(oracle_mod.Oracle, Channel, p5, gy, seed=32)
    ch6 = Channel(p6, gy)
    ch6.upload_state(ch5.download_state())
    net = _net()
    net.set_range(np.full(16, 1e30, np.float32), np.full(16, 2e30, np.float32))   # nothing in range
    ch6.set_sgs_net(net)
    ch5.step(5)
    ch6.step(5)
    a, b = channel_state(ch5, p5), channel_state(ch6, p6)
    # the same AMD arithmetic in two instantiations of the closure walk, whose
    # multiply-adds the compiler may contract differently: last-bit
    # differences, which cp (the running sum of phi / h) grows the most
    for f in STATE:
        assert rel_l2(b[f], a[f]) <= 1e-12, f


@pytest.mark.parametrize("prec", [0, 1])
def test_closure_nu_is_network_output(oracle_mod, Channel, prec):
    # the substep's inference forms the features from the FP64 (prec 0) or
    # FP32 (prec 1) physical fields itself; the reference is the network on
    # the features the AMD kernel's feature mode writes from the same fields
    p = les_params(6, precision=prec)
    gy = grid_for(p)
    _, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=33)
    net = _net(2)
    ch.set_sgs_net(net)
    nu, ka, feat = ch.les_eval(6, features=True)
    out = net.forward(torch.from_numpy(feat.reshape(-1, 16)).cuda()).cpu().numpy()
    out = out.reshape(p.ny + 2, p.nz, p.nx, 2)
    for j in range(3, p.ny):
        for q, fld in ((0, nu), (1, ka)):
            ref = out[j, :, :, q]
            got = fld[j, : p.nz, : p.nx]
            assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max(), (j, q)
    for j in (1, 2, p.ny, p.ny + 1):
        assert np.all(nu[j] == 0.0) and np.all(ka[j] == 0.0)


def test_closure_run_finite_and_divergence_free(oracle_mod, Channel):
    p = les_params(6)
    gy = grid_for(p)
    _, ch = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=34)
    ch.set_sgs_net(_net(3))
    ch.step(10)
    st = channel_state(ch, p)
    assert all(np.all(np.isfinite(st[f])) for f in STATE)
    assert ch.divergence() <= 1e-12
    nu, _ = ch.les_eval(6)
    assert np.all(nu >= 0.0) and nu.max() > 0.0
