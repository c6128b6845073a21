"""Pinning the CPU oracle (no GPU): the reference has no golden vectors, so
the oracle is checked against independent known answers."""
import math

import numpy as np
import pytest

from _util import config0_params, gradients_at_gy, grid_for, rel_l2, significant


@pytest.mark.parametrize("n", [8, 16, 64, 512])
def test_fft_matches_long_double_dft_and_numpy(oracle_mod, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    f = oracle_mod.fft_c2c(x, -1)
    assert rel_l2(f, oracle_mod.dft_c2c_ld(x, -1)) < 1e-14
    assert rel_l2(f, np.fft.fft(x)) < 1e-14
    b = oracle_mod.fft_c2c(x, +1)
    assert rel_l2(b, np.fft.ifft(x) * n) < 1e-14


def test_fft_xz_to_fourier_matches_numpy_rfft2(oracle_mod):
    p = config0_params(nx=32, ny=9, nz=16)
    o = oracle_mod.Oracle(p, grid_for(p))
    rng = np.random.default_rng(0)
    phys = rng.standard_normal((p.ny + 2, p.nz + 2, p.nx + 2))
    buf = phys.copy()
    o.fft_to_fourier(buf.reshape(-1))
    c = buf.reshape(-1).view(np.complex128).reshape(p.ny + 2, p.nz + 2, p.nxp + 1)
    ref = np.fft.rfft2(phys[:, :p.nz, :p.nx], axes=(1, 2)) / (p.nx * p.nz)
    nkx, nkz = p.nkx, p.nkz
    packed = np.concatenate([ref[:, :nkz + 1, :nkx + 1], ref[:, p.nz - nkz:, :nkx + 1]], axis=1)
    assert rel_l2(significant(p, c), packed) < 1e-14


def test_round_trip_on_dealiased_field_and_dc_imag_ignored(oracle_mod):
    p = config0_params(nx=32, ny=5, nz=32)
    o = oracle_mod.Oracle(p, grid_for(p))
    rng = np.random.default_rng(1)
    c = np.zeros((p.ny + 2, p.nz + 2, p.nxp + 1), dtype=np.complex128)
    sl = (slice(None), slice(0, 2 * p.nkz + 1), slice(0, p.nkx + 1))
    c[sl] = rng.standard_normal(c[sl].shape) + 1j * rng.standard_normal(c[sl].shape)
    # a real field needs a Hermitian kx = 0 column: make it so
    col = c[:, : 2 * p.nkz + 1, 0]
    kz = np.r_[0:p.nkz + 1, -p.nkz:0]
    for a, k in enumerate(kz):
        if k < 0:
            col[:, a] = np.conj(col[:, list(kz).index(-k)])
    col[:, 0] = col[:, 0].real
    c0 = c.copy()
    phys = c.copy()
    o.fft_to_physical(phys.view(np.float64).reshape(-1))
    back = phys.view(np.float64).copy()
    o.fft_to_fourier(back.reshape(-1))
    cb = back.reshape(-1).view(np.complex128).reshape(c.shape)
    assert rel_l2(significant(p, cb), significant(p, c0)) < 1e-14
    # FFTW's c2r ignores Im of the DC mode: adding one changes nothing
    c2 = c0.copy()
    c2[:, 0, 0] += 1j * 3.0
    p2 = c2.copy()
    o.fft_to_physical(p2.view(np.float64).reshape(-1))
    r1 = phys.view(np.float64).reshape(p.ny + 2, p.nz + 2, p.nx + 2)[:, :p.nz, :p.nx]
    r2 = p2.view(np.float64).reshape(p.ny + 2, p.nz + 2, p.nx + 2)[:, :p.nz, :p.nx]
    assert np.array_equal(r1, r2)


def test_thomas_matches_dense_lu(oracle_mod):
    rng = np.random.default_rng(3)
    ny, inx = 20, 7
    n = ny + 2
    a = rng.uniform(-1, 0, (n, inx))
    c = rng.uniform(-1, 0, (n, inx))
    b = 3.0 + rng.uniform(0, 1, (n, inx))
    g = rng.standard_normal((n, inx))
    x = oracle_mod.thomas_real(a, b, c, g, ny, inx)
    for i in range(inx):
        M = np.diag(b[:, i]) + np.diag(a[1:, i], -1) + np.diag(c[:-1, i], 1)
        assert rel_l2(x[:, i], np.linalg.solve(M, g[:, i])) < 1e-14


def _div(p, o, dyf):
    cu1, cu2, cu3 = o.cplx(0), o.cplx(1), o.cplx(2)
    kx = o.metric(4, p.nxp)[: p.nkx + 1]
    kz = o.metric(5, 2 * p.nkz + 1)
    m = 0.0
    for j in range(2, p.ny):
        d = (1j * kx[None, :] * cu1[j, : 2 * p.nkz + 1, : p.nkx + 1]
             + (cu2[j + 1] - cu2[j])[: 2 * p.nkz + 1, : p.nkx + 1] / dyf[j]
             + 1j * kz[:, None] * cu3[j, : 2 * p.nkz + 1, : p.nkx + 1])
        m = max(m, float(np.abs(d).max()))
    return m


def test_rem_div_removes_divergence(oracle_mod):
    p = config0_params(nx=32, ny=17, nz=32)
    gy = grid_for(p)
    o = oracle_mod.Oracle(p, gy)
    rng = np.random.default_rng(4)
    for f in (0, 1, 2):
        c = o.cplx(f)
        sl = (slice(None), slice(0, 2 * p.nkz + 1), slice(0, p.nkx + 1))
        c[sl] = rng.standard_normal(c[sl].shape) + 1j * rng.standard_normal(c[sl].shape)
    dyf = o.metric(3, p.ny + 2)
    assert _div(p, o, dyf) > 1.0
    o.rem_div()
    assert _div(p, o, dyf) < 1e-12


def test_stokes_mode_matches_independent_propagator(oracle_mod):
    """A spanwise velocity u3 = A(y) cos(kx x) has no nonlinear term, no
    divergence and (with rotation and gravity off) obeys the discrete
    RKW3 + CN heat equation.  Propagate it with dense numpy matrices built
    from the scheme's definition and compare with the oracle."""
    p = config0_params(nx=16, ny=17, nz=16, ic_type=3, flavor_front=0, ro=1e300, grav_y=0.0,
                       kick=0.0, re=50.0, delta_t=2e-3, w_bc_ymin=0, w_bc_ymax=0,
                       u_bc_ymin=0, u_bc_ymax=0)
    gy = grid_for(p)
    o = oracle_mod.Oracle(p, gy)
    nyp = p.ny
    ymet = {k: o.metric(i, nyp + 2) for i, k in enumerate(("gy", "gyf", "dy", "dyf"))}
    dy, dyf = ymet["dy"], ymet["dyf"]
    kxv = o.metric(4, p.nxp)[1]
    # mode kx index 1, kz = 0: cu3(1, 0, j) = A_j
    A = np.zeros(nyp + 2)
    A[2:nyp] = np.sin(np.linspace(0, math.pi, nyp - 2))
    c = o.cplx(2)
    c[:, 0, 1] = A
    nu, hb = 1.0 / p.re, p.delta_t * np.array([8, 2, 5]) / 15.0
    beta_b, zeta_b = [1.0, 25 / 8, 9 / 4], [0.0, -17 / 8, -5 / 4]
    js, je = 2, nyp - 1   # u Dirichlet both walls
    # L: explicit vertical operator at rows js..je (solver.f90:856-858)
    L = np.zeros((nyp + 2, nyp + 2))
    for j in range(js, je + 1):
        L[j, j + 1] += 1.0 / dy[j + 1] / dyf[j]
        L[j, j] -= (1.0 / dy[j + 1] + 1.0 / dy[j]) / dyf[j]
        L[j, j - 1] += 1.0 / dy[j] / dyf[j]
    u, cf = A.astype(complex), np.zeros(nyp + 2, complex)
    for _step in range(3):
        for rk in range(3):
            t1 = 0.5 * nu * hb[rk]
            cf_new = -nu * kxv ** 2 * u
            r = u + (zeta_b[rk] * hb[rk] * cf if rk else 0) + beta_b[rk] * hb[rk] * cf_new
            r = r + t1 * (L @ u)
            M = np.eye(nyp + 2) - t1 * L
            for j in (0, 1, nyp, nyp + 1):     # Dirichlet rows (apply_BC_3_*)
                M[j, :] = 0
                M[j, j] = 1
                r[j] = 0.0
            u_new = np.linalg.solve(M, r)
            keep = np.zeros(nyp + 2, bool)
            keep[js - 1: je + 2] = True
            u = np.where(keep, u_new, u)
            cf = cf_new
    for _ in range(3):
        o.step()
    got = o.cplx(2)[:, 0, 1]
    assert rel_l2(got[1:nyp + 1], u[1:nyp + 1]) < 1e-13
    assert np.abs(o.cplx(0)).max() < 1e-300 + 1e-30  # u1 stays zero


def test_thermal_wind_rest_state_is_steady(oracle_mod):
    """Infinite front (IC 4) without perturbation and with walls that do not
    force the perturbation (w Dirichlet at both walls; a Neumann w wall would
    carry input_chan's compensation -dV/dy and drive a boundary layer): the
    background is in thermal-wind balance inside the solver, so u stays 0 and
    th unchanged."""
    p = config0_params(nx=16, ny=17, nz=16, kick=0.0, w_bc_ymax=0, u_bc_ymax=1)
    gy = grid_for(p)
    from diablo3_b200.ic import initial_fields
    o = oracle_mod.Oracle(p, gy)
    o.init_from_physical(*initial_fields(p, gy, seed=0))
    th0 = significant(p, o.cplx(4)).copy()
    for _ in range(5):
        o.step()
    for f in (0, 1, 2):
        assert np.abs(significant(p, o.cplx(f))).max() < 1e-14
    assert rel_l2(significant(p, o.cplx(4)), th0) < 1e-14


def _amd_fixture(oracle_mod, **kw):
    from diablo3_b200.ic import initial_fields
    p = config0_params(nx=32, ny=33, nz=16, use_les=1, create_new_flow=0, les_model_type=5,
                       kick=0.05, re=5000.0, **kw)
    gy = grid_for(p)
    o = oracle_mod.Oracle(p, gy)
    o.init_from_physical(*initial_fields(p, gy, seed=11))
    c = {f: o.cplx(f).copy() for f in (0, 1, 2, 4)}
    met = {k: o.metric(i, p.ny + 2) for i, k in enumerate(("gy", "gyf", "dy", "dyf"))}
    kx = o.metric(4, p.nxp)[: p.nkx + 1]
    kz = o.metric(5, 2 * p.nkz + 1)
    o.rk_substep(1)
    return p, o, c, met, kx, kz


def _filter_widths(p, met):
    dx, dz = p.lx / p.nx, p.lz / p.nz
    return 3.0 * dx, 2.0 * met["dy"], 3.0 * dz


def test_amd_eddy_viscosity_matches_tensor_form(oracle_mod):
    """nu_t of the AMD model (les_model_type 5) from the oracle's
    element-wise restatement equals the closed tensor form
    C^2 max(0, -tr(S^3) + tr(S W^2)) / |D|^2 * 3 / sum_k delta_k^-2 with
    D_ij = (delta_j / delta_i) du_i/dx_j, S, W its symmetric and
    antisymmetric parts, evaluated here with numpy at GY rows."""
    p, o, c, met, kx, kz = _amd_fixture(oracle_mod)
    G, _ = gradients_at_gy(p, c, met, kx, kz)
    dxs, dys, dzs = _filter_widths(p, met)
    ny = p.ny
    rows = range(3, ny)   # rows 1, 2, ny, ny+1 are the zeroed wall rows
    nut = o.real(9)[:, : p.nz, : p.nx]
    assert np.all(nut >= 0.0)
    for j in (1, 2, ny, ny + 1):
        assert np.all(nut[j] == 0.0)
    worst = 0.0
    for j in rows:
        delta = np.array([dxs, dys[j], dzs])
        D = G[:, :, j] * (delta[None, :] / delta[:, None])[:, :, None, None]
        S = 0.5 * (D + D.transpose(1, 0, 2, 3))
        W = 0.5 * (D - D.transpose(1, 0, 2, 3))
        S3 = np.einsum("ijzx,jkzx,kizx->zx", S, S, S)
        SW2 = np.einsum("ijzx,jkzx,kizx->zx", S, W, W)
        num = -S3 + SW2
        den = np.einsum("ijzx,ijzx->zx", D, D)
        v = np.where(num > 0, num / den, 0.0)
        ref = 0.2887 ** 2 * 3.0 / (1 / dxs ** 2 + 1 / dys[j] ** 2 + 1 / dzs ** 2) * v
        worst = max(worst, float(np.abs(nut[j] - ref).max()))
    scale = float(nut.max())
    assert scale > 0.0
    assert worst < 1e-11 * scale


def test_amd_eddy_diffusivity_matches_tensor_form(oracle_mod):
    """kappa_t of the scalar AMD model equals
    C^2 max(0, -g^T G Delta^2 g) / |Delta g|^2 * 3 / sum_k delta_k^-2
    (G the velocity gradient, g the scalar gradient, Delta = diag(delta))."""
    p, o, c, met, kx, kz = _amd_fixture(oracle_mod)
    G, g = gradients_at_gy(p, c, met, kx, kz)
    dxs, dys, dzs = _filter_widths(p, met)
    ny = p.ny
    kt = o.real(10)[:, : p.nz, : p.nx]
    assert np.all(kt >= 0.0)
    worst = 0.0
    for j in range(3, ny):
        d2 = np.array([dxs, dys[j], dzs]) ** 2
        gj = g[:, j]
        num = -np.einsum("izx,ikzx,k,kzx->zx", gj, G[:, :, j], d2, gj)
        den = np.einsum("k,kzx->zx", d2, gj * gj)
        v = np.where(num > 0, num / den, 0.0)
        ref = 0.2887 ** 2 * 3.0 / (1 / dxs ** 2 + 1 / dys[j] ** 2 + 1 / dzs ** 2) * v
        worst = max(worst, float(np.abs(kt[j] - ref).max()))
    scale = float(kt.max())
    assert scale > 0.0
    assert worst < 1e-11 * scale


def test_mlp_oracle_gradient_matches_central_differences():
    """The FP64 (unrounded) MLP oracle's analytic gradient against central
    differences of its loss, on a few parameters of every block."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import mlp_oracle as mo
    rng = np.random.default_rng(0)
    n = 64
    feat = rng.standard_normal((n, 16))
    tgt = rng.random((n, 2)) * 1e-3
    mean, std, scale = np.zeros(16), np.ones(16), np.array([1e-3, 1e-3])
    params = rng.standard_normal(mo.NPARAMS) * 0.2
    _, g = mo.loss_and_grad(params, feat, tgt, mean, std, scale, quantized=False)
    for k, (o, sh) in mo.OFF.items():
        for idx in rng.choice(int(np.prod(sh)), min(3, int(np.prod(sh))), replace=False):
            i = o + int(idx)
            h = 1e-6
            pp, pm = params.copy(), params.copy()
            pp[i] += h
            pm[i] -= h
            lp, _ = mo.loss_and_grad(pp, feat, tgt, mean, std, scale, quantized=False)
            lm, _ = mo.loss_and_grad(pm, feat, tgt, mean, std, scale, quantized=False)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 * max(1e-8, abs(g[i])) + 1e-12, (k, i, fd, g[i])


def test_amd_from_features_is_model_5(oracle_mod):
    """The yardstick of the learned closure, AMD evaluated on closure
    features (diablo3_b200.sgs_train), gives the oracle's model-5 nu_t and
    kappa_t at the interior GY rows."""
    from diablo3_b200.sgs_train import amd_from_features
    p, o, c, met, kx, kz = _amd_fixture(oracle_mod)
    G, g = gradients_at_gy(p, c, met, kx, kz)
    dxs, dys, dzs = _filter_widths(p, met)
    for j in range(3, p.ny):
        f = np.empty((p.nz * p.nx, 16))
        for i in range(3):
            for k in range(3):
                f[:, 3 * i + k] = G[i, k, j].reshape(-1)
        f[:, 9:12] = g[:, j].reshape(3, -1).T
        f[:, 12], f[:, 13], f[:, 14] = dxs, dys[j], dzs
        f[:, 15] = g[1, j].reshape(-1)
        nu, ka = amd_from_features(f)
        ref_nu = o.real(9)[j, : p.nz, : p.nx].reshape(-1)
        ref_ka = o.real(10)[j, : p.nz, : p.nx].reshape(-1)
        assert np.abs(nu - ref_nu).max() <= 1e-11 * max(ref_nu.max(), 1e-30)
        assert np.abs(ka - ref_ka).max() <= 1e-11 * max(ref_ka.max(), 1e-30)
