"""Autotuner (db_autotune): the launch shapes it picks change only how the
work is split over CTAs, never the arithmetic, so a tuned context must step
bit-identically to an untuned one from the same state (FP64 DNS, mixed
precision, and LES with the per-column Thomas)."""
import numpy as np
import pytest

from _util import STATE, config0_params, grid_for, seed_pair

pytestmark = pytest.mark.gpu

NU_T = 9


@pytest.mark.parametrize("case", ["dns_fp64", "dns_mixed", "les_fp64", "les_mixed"])
def test_autotuned_steps_bit_identical(oracle_mod, case):
    from diablo3_b200.channel import Channel
    kw = dict(nx=64, ny=65, nz=64, kick=0.05)
    if case.startswith("les"):
        kw.update(use_les=1, create_new_flow=0, les_model_type=5, re=5000.0)
    if case.endswith("mixed"):
        kw.update(precision=1)
    p = config0_params(**kw)
    gy = grid_for(p)
    o, ref = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=5)
    tuned = Channel(p, gy)
    tuned.upload_state({fid: o.cplx(fid).copy() for fid in STATE})
    report = tuned.autotune()
    assert "chosen:" in report and "x-pass" in report and "z-pass" in report, report
    if case.startswith("les"):
        assert "LES Thomas" in report, report
    ref.step(4)
    tuned.step(4)
    a, b = ref.download_state(), tuned.download_state()
    for fid in STATE:
        assert np.array_equal(a[fid], b[fid]), fid
    if case.startswith("les"):
        assert np.array_equal(ref.download_field(NU_T), tuned.download_field(NU_T))
    ref.close()
    tuned.close()


@pytest.mark.parametrize("case", ["amd_fp64", "amd_mixed", "learned_fp64"])
def test_closure_walk_chunks_bit_identical(oracle_mod, case):
    """The LES closure's column walk split into 1, 2, 3 or 8 wall-normal
    chunks (each chunk rebuilds the carried values from the row before it)
    stores exactly what one walk stores: the steps agree bit for bit."""
    from diablo3_b200 import sgs_net
    from diablo3_b200.channel import Channel
    kw = dict(nx=32, ny=65, nz=32, kick=0.05, use_les=1, create_new_flow=0, les_model_type=5, re=5000.0)
    if case == "amd_mixed":
        kw.update(precision=1)
    if case == "learned_fp64":
        kw.update(les_model_type=6)
    p = config0_params(**kw)
    gy = grid_for(p)
    net = None
    if case == "learned_fp64":
        net = sgs_net.SgsNet()
        std = np.ones(16, np.float32)
        std[12:15] = 0.1
        net.set(sgs_net.init_params(3) * 0.3, np.zeros(16, np.float32), std, np.array([1e-4, 1e-4], np.float32))
    o, base = seed_pair(oracle_mod.Oracle, Channel, p, gy, seed=9)
    start = {fid: o.cplx(fid).copy() for fid in STATE}
    results = []
    for chunks in (1, 2, 3, 8):
        ch = Channel(p, gy)
        if net is not None:
            ch.set_sgs_net(net)
        ch.upload_state(start)
        ch.set_tuning([0, 0, 0, 0, 0, chunks])
        assert ch.tuning()[5] == chunks
        ch.step(3)
        results.append((ch.download_state(), ch.download_field(NU_T)))
        ch.close()
    a_state, a_nu = results[0]
    assert np.abs(a_nu).max() > 0.0
    for b_state, b_nu in results[1:]:
        for fid in STATE:
            assert np.array_equal(a_state[fid], b_state[fid]), fid
        assert np.array_equal(a_nu, b_nu)
    base.close()
    if net is not None:
        net.close()
