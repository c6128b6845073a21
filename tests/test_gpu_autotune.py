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
