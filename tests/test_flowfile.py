"""The reference-layout flow file on the host (no GPU): the u2 moves between
GY and GYF points (g2gf / gf2g, for/tools.f90:255-318), the FP64 host
transforms with the reference's normalisation and truncation, the dataset
layout of WriteHDF5 (for/phdf5.f90:918-1197) through a stand-in channel, and
files that are not flow files, are cut short, changed, or of another
resolution."""
import numpy as np
import pytest

from diablo3_b200 import flowfile
from diablo3_b200 import lib as L
from diablo3_b200.params import make_params


def _p():
    return make_params(nx=16, ny=9, nz=16, delta_t=1e-3)


def test_g2gf_gf2g():
    rng = np.random.default_rng(1)
    ny = 9
    v = rng.standard_normal((ny + 2, 4, 5))
    w = flowfile.g2gf(v, ny)
    # GYF row y holds the mean of GY rows y, y+1 with the wall rows copied in
    assert np.allclose(w[3], 0.5 * (v[3] + v[4]))
    assert np.allclose(w[1], v[2]) and np.allclose(w[ny], v[ny])
    back = flowfile.gf2g(w, ny)
    # interior rows return; the wall rows take the zero-mass-flux values
    assert np.allclose(back[2: ny + 1], v[2: ny + 1], atol=1e-14)
    assert np.allclose(back[1], -back[2]) and np.allclose(back[ny + 1], -back[ny])


def test_host_transforms_round_trip():
    p = _p()
    rng = np.random.default_rng(2)
    u = rng.standard_normal((p.ny + 2, p.nz, p.nx))
    c = flowfile.to_fourier(p, u)
    # a band-limited field (the retained modes of u) comes back exactly
    ub = flowfile.to_physical(p, c)
    assert np.allclose(flowfile.to_fourier(p, ub), c, atol=1e-14)
    # normalisation: the (0,0) mode is the plane mean
    assert np.allclose(c[:, 0, 0].real, u.mean(axis=(1, 2)))


class Stub:
    def __init__(self):
        self.p = _p()
        rng = np.random.default_rng(3)
        self.state = {}
        for f in L.STATE_FIELDS:
            u = rng.standard_normal((self.p.ny + 2, self.p.nz, self.p.nx))
            self.state[f] = flowfile.to_fourier(self.p, u)

    def status(self):
        s = L.DbStatus()
        s.time, s.time_step, s.delta_t = 2.5, 17, 1e-3
        return s

    def download_state(self):
        return self.state


def test_dataset_layout(tmp_path):
    ch = Stub()
    p = ch.p
    path = str(tmp_path / "end.flow")
    flowfile.write_flow(ch, path, save_flow_time=3.0, save_stats_time=2.75, save_movie_time=2.9)
    hdr, d = flowfile.read_file(path)
    assert hdr["Resolution"] == [p.nx, p.ny, p.nz]
    assert hdr["Timestep"] == {"Time": 2.5, "Save_Flow_Time": 3.0, "Save_Stats_Time": 2.75,
                               "Save_Movie_Time": 2.9, "Time_Step": 17}
    assert set(d) == {"U", "W", "V", "TH1", "P"}
    u1 = flowfile.to_physical(p, ch.state[L.CU1])
    u2 = flowfile.to_physical(p, ch.state[L.CU2])
    # U(x, y, z) = u1(x, z, y) for y = 1..Nyp: a C array [z][y][x]
    assert d["U"].shape == (p.nz, p.ny, p.nx)
    assert np.allclose(d["U"][5, 2, 7], u1[3, 5, 7])
    # W is u2 at the GYF points
    w = 0.5 * (u2[4] + u2[5])
    assert np.allclose(d["W"][:, 3, :], w)
    flowfile.write_flow(ch, path, save_pressure=False)
    assert "P" not in flowfile.read_file(path)[1]


def test_damaged_and_foreign_files(tmp_path):
    ch = Stub()
    path = str(tmp_path / "x.flow")
    flowfile.write_flow(ch, path)
    data = open(path, "rb").read()
    with open(path, "wb") as f:
        f.write(data[:-10])
    with pytest.raises(flowfile.FlowFileError, match="truncated"):
        flowfile.read_file(path)
    bad = bytearray(data)
    bad[-8] ^= 1
    with open(path, "wb") as f:
        f.write(bytes(bad))
    with pytest.raises(flowfile.FlowFileError, match="CRC"):
        flowfile.read_file(path)
    with open(path, "wb") as f:
        f.write(b"DIABLOB3" + data[8:])
    with pytest.raises(flowfile.FlowFileError, match="not a flow file"):
        flowfile.read_file(path)
    with open(path, "wb") as f:
        f.write(data)
    q = make_params(nx=32, ny=9, nz=16)
    with pytest.raises(flowfile.FlowFileError, match="resolution"):
        flowfile.read_flow(path, q, np.linspace(-1, 1, q.ny + 1))
