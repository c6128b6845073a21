"""Device-resident transforms (db_fft_xz_to_fourier_dev / _physical_dev) on
device arrays in the reference layout, against the host-array forms on the
same fields: bit-identical on FP64 and mixed-precision contexts, the padding
of the physical layout left as it was in both."""
import numpy as np
import pytest

from _util import config0_params, grid_for

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("prec", [0, 1])
def test_device_transforms_match_host_forms(prec):
    from diablo3_b200.channel import Channel
    p = config0_params(nx=32, ny=33, nz=32, precision=prec)
    ch = Channel(p, grid_for(p))
    rng = np.random.default_rng(7)
    phys = rng.standard_normal(ch.new_real().shape)   # padding holds values too
    # forward
    spec_host = ch.fft_xz_to_fourier(phys.copy()).copy()
    d = torch.from_numpy(phys.copy()).cuda()
    torch.cuda.synchronize()
    ch.fft_xz_to_fourier_dev(d)
    torch.cuda.synchronize()
    spec_dev = d.cpu().numpy().reshape(-1).view(np.complex128).reshape(spec_host.shape)
    assert np.array_equal(spec_dev, spec_host)
    # inverse, from a spectral array whose unretained entries hold values
    # (both forms ignore them)
    spec = spec_host.copy()
    nkx, nkzp = p.nx // 3, 2 * (p.nz // 3) + 1
    spec[:, :, nkx + 1:] = rng.standard_normal(spec[:, :, nkx + 1:].shape)
    spec[:, nkzp:, :] = rng.standard_normal(spec[:, nkzp:, :].shape)
    phys_host = ch.fft_xz_to_physical(spec.copy()).copy()
    d2 = torch.from_numpy(spec.copy()).cuda()
    torch.cuda.synchronize()
    ch.fft_xz_to_physical_dev(d2)
    torch.cuda.synchronize()
    phys_dev = d2.cpu().numpy().reshape(-1).view(np.float64).reshape(phys_host.shape)
    assert np.array_equal(phys_dev, phys_host)
    # the forward transform of the band-limited result gives the same modes
    d3 = torch.from_numpy(phys_dev.copy()).cuda()
    torch.cuda.synchronize()
    ch.fft_xz_to_fourier_dev(d3)
    torch.cuda.synchronize()
    again = d3.cpu().numpy().reshape(-1).view(np.complex128).reshape(spec_host.shape)
    tol = 1e-12 if prec == 0 else 1e-5
    assert np.abs(again - spec_host).max() <= tol * np.abs(spec_host).max()
    ch.close()
