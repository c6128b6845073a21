"""A full RK step reads U, V, W, TH and P only.

The RK history CF is rebuilt in a step's first substep before anything
reads it (for/solver.f90:413 reads it only for rk_step > 1, :487 assigns
it), so a step from a state whose CF fields hold arbitrary values gives the
same result, bit for bit, as a step from the true CF.  Checked on the FP64,
mixed and LES (AMD) paths: two contexts run the same two steps, the second
then gets random CF fields, and after one more step, and again after two
more, the five fields are identical (CF itself keeps the random values on
the boundary planes, which the step neither reads nor writes).  The
end-to-end bench leg relies on this: it moves those five fields each way
per step.
"""
import numpy as np
import pytest

from _util import channel_state, config0_params, grid_for

pytestmark = pytest.mark.gpu

STEP_FIELDS = (0, 1, 2, 3, 4)   # cu1 cu2 cu3 cp cth
CF_FIELDS = (5, 6, 7, 8)        # cf1 cf2 cf3 cfth


@pytest.mark.parametrize("kind", ["fp64", "mixed", "les"])
def test_full_step_does_not_read_cf(kind):
    from diablo3_b200.channel import Channel
    kw = dict(nx=32, ny=33, nz=32, precision=1 if kind == "mixed" else 0)
    if kind == "les":
        kw.update(use_les=1, create_new_flow=0, les_model_type=5, kick=0.05, re=5000.0)
    p = config0_params(**kw)
    gy = grid_for(p)
    a, b = Channel(p, gy), Channel(p, gy)
    for ch in (a, b):
        ch.init_flow(seed=4)
        ch.step(2)
    sa0 = channel_state(a, p)
    assert all(np.abs(sa0[f]).max() > 0 for f in CF_FIELDS)   # a real history to lose
    rng = np.random.default_rng(11)
    for f in CF_FIELDS:
        shape = b.new_spectral().shape
        b.upload_field(f, rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    for n in (1, 2):
        a.step(n)
        b.step(n)
        sa, sb = channel_state(a, p), channel_state(b, p)
        for f in STEP_FIELDS:
            assert np.array_equal(sa[f], sb[f]), (n, f)
    assert a.status().flags == b.status().flags == 0
    a.close()
    b.close()
