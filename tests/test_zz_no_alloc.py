"""db_rem_div_static: divergence removal for callers that cannot allocate.

Callers whose device memory belongs to another allocator (CUDA Fortran or
OpenACC pools) or that must not allocate inside their time loop pass their
own device arrays; the entry point's working memory is a fixed static device
array.  This file is named to be collected last.  It checks, on two calls in
a row with different inputs (so the second call runs on scratch the first
one left behind), that the result matches the context-based db_rem_div to
the same 1e-12 relative tolerance as the other rem_div parity test, and on
the first call of the small grid the CPU oracle's rem_div_chan as well.  The
second grid is tall enough that one call runs the chunk loop six times.
"""
import ctypes

import numpy as np
import pytest

from _util import config0_params, grid_for, rel_l2, significant

pytestmark = pytest.mark.gpu


def _field(ch, p, rng, scale):
    """A non-solenoidal spectral velocity field in the reference layout."""
    a = ch.new_spectral()
    sl = (slice(None), slice(0, 2 * p.nkz + 1), slice(0, p.nkx + 1))
    a[sl] = scale * (rng.standard_normal(a[sl].shape) + 1j * rng.standard_normal(a[sl].shape))
    return a


@pytest.mark.parametrize("ny", [65, 2049])
def test_rem_div_static_matches_rem_div_twice(oracle_mod, ny):
    # ny = 2049: the static scratch holds 169 columns per launch, so the 946
    # (kx, kz) columns take six launches of the chunk loop
    import torch

    from diablo3_b200 import lib as L
    from diablo3_b200.channel import Channel

    p = config0_params(nx=64, ny=ny, nz=64)
    gy = grid_for(p)
    rng = np.random.default_rng(2024)
    with Channel(p, gy) as ch:
        for call in range(2):
            u = [_field(ch, p, rng, 10.0 ** -call) for _ in range(3)]
            # reference result: the context-based entry point
            ch.upload_state({0: u[0], 1: u[1], 2: u[2]})
            ch.rem_div_chan()
            ref = ch.download_state()
            # caller-owned device arrays (allocated by the test, not the entry point)
            dev = [torch.from_numpy(x.view(np.float64).copy()).cuda() for x in u]
            torch.cuda.synchronize()
            rc = L.load().db_rem_div_static(ctypes.byref(ch.p), L.dptr(gy),
                                            ctypes.c_void_p(dev[0].data_ptr()),
                                            ctypes.c_void_p(dev[1].data_ptr()),
                                            ctypes.c_void_p(dev[2].data_ptr()), None)
            assert rc == 0
            torch.cuda.synchronize()
            got = [dev[f].cpu().numpy().view(np.complex128).reshape(u[f].shape) for f in range(3)]
            for f in range(3):
                err = rel_l2(significant(p, got[f]), significant(p, ref[f]))
                assert err < 1e-12, (call, f, err)
            if ny == 65 and call == 0:
                # and directly against the oracle's rem_div_chan
                o = oracle_mod.Oracle(p, gy)
                for f in range(3):
                    o.cplx(f)[...] = u[f]
                o.rem_div()
                for f in range(3):
                    err = rel_l2(significant(p, got[f]), significant(p, o.cplx(f)))
                    assert err < 1e-12, ("oracle", f, err)
                o.close()


def test_rem_div_static_rejects_oversized_grid():
    from diablo3_b200 import lib as L

    p = config0_params(nx=16, ny=20000, nz=16)
    gy = np.linspace(-1.0, 1.0, p.ny + 1)
    rc = L.load().db_rem_div_static(ctypes.byref(p), L.dptr(gy), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                    ctypes.c_void_p(16), None)
    assert rc == 3  # DB_ERR_SIZE, before any device work
