// k_substep.cu -- the RKW3 + Crank-Nicolson substep (rk_chan_1,
// for/solver.f90:366-1273) as fused B200 kernels, FP64.
//
//  k_products   : 11 nonlinear products of u1,u2,u3,th in physical space
//                 (solver.f90:655-815, 914-956) fused with their forward
//                 x-FFTs; x-derivatives (i kx) applied in the x-half space so
//                 only 8 x-half fields leave the kernel.
//  k_zpass_rhs  : forward z-FFT of those 8 fields, the spectral linear terms
//                 (viscous, Coriolis, buoyancy, background-front advection,
//                 thermal-wind advection: solver.f90:396-609, 35-111), the RK
//                 combination cr = cu + zeta h cf_old - h grad p + beta h cf
//                 (solver.f90:396-456, 824-838, 966-973), and the inverse
//                 z-FFT of cr.
//  k_tri_coef   : the four implicit systems' rows incl. BC rows
//                 (solver.f90:1012-1233, 1901-2324), LU-factored once per
//                 substep (all (x,z) columns share them without LES).
//  k_thomas     : per (x,z) column, explicit CN term + Thomas sweeps for
//                 th, u2, u1, u3 (solver.f90:850-870, 981-989, 1691-1852).
//  k_rem_div    : per (kx,kz) column, divergence, complex Thomas, projection
//                 and pressure update (solver.f90:1302-1379, 1261-1267).
//  k_courant    : CFL reduction and dt scheduling (flow.f90:746-857).
#include <math.h>

#include "db_kernels.cuh"
#include "fft_smem.cuh"

namespace db {

constexpr int ZPAD_S = 1;

__device__ __forceinline__ bool in_rng(int j, int a, int b) { return j >= a && j <= b; }

// X_a (part 0) or X_b (part 1) at mode m of the complex FFT of a + i b
template <int N>
__device__ __forceinline__ double2 sep(const double2* z, int m, int part) {
  double2 zm = z[m], zn = cconj(z[(N - m) & (N - 1)]);
  if (part == 0) return make_double2(0.5 * (zm.x + zn.x), 0.5 * (zm.y + zn.y));
  return make_double2(0.5 * (zm.y - zn.y), -0.5 * (zm.x - zn.x));
}

// ---------------------------------------------------------------------------
// nonlinear products + forward x-FFT.  One CTA per (z, j) row, 6 sequences:
//  seq0 (u1 u3 | u1 u1)        seq1 (u3 u3 | <u1> u2)    seq2 (<u3> u2 | Dy u1u2)
//  seq3 (Dy u3u2 | Dy u2u2)    seq4 (th u1 | th u3)      seq5 (Dy th u2 | 0)
// Outputs (x-half), o = 0..7:
//  N1 = ikx X(u1u1) + X(Dy u1u2)   M1 = X(u1u3)
//  N3 = ikx X(u1u3) + X(Dy u3u2)   M3 = X(u3u3)
//  N2 = ikx X(<u1>u2) + X(Dy u2u2) M2 = X(<u3>u2)
//  NT = ikx X(th u1) + X(Dy th u2) MT = X(th u3)
// so that cf_e -= Z(N_e) + ikz Z(M_e) after the z-pass.
template <int N>
__global__ void __launch_bounds__(6 * (N / 8)) k_products(State s, Geom g) {
  extern __shared__ double2 sm[];
  constexpr int T = N / 8;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int z = blockIdx.x, j = blockIdx.y;
  const bool r1 = in_rng(j, g.jstart, g.jend);
  const bool r2 = in_rng(j, 2, g.ny);
  const bool rt = in_rng(j, g.jstart_th, g.jend_th);
  const long long hrow = (long long)j * g.hp + (long long)z * g.kxs;
  if (!(r1 || r2 || rt)) {
    for (int idx = threadIdx.x; idx < 8 * g.kxs; idx += blockDim.x)
      s.xh[idx / g.kxs][hrow + idx % g.kxs] = make_double2(0.0, 0.0);
    return;
  }
  double2* buf = sm + seq * (N + ZPAD_S);
  const long long o0 = (long long)j * g.pp + (long long)z * g.nx;
  const long long om = o0 - g.pp, op = o0 + g.pp;
  const double dyj = g.dy[j], dyfj = g.dyf[j];
  const double dyfjm = (j >= 1) ? g.dyf[j - 1] : 0.0;
#pragma unroll 2
  for (int m = 0; m < 8; ++m) {
    const int x = lane + m * T;
    double a = 0.0, b = 0.0;
    switch (seq) {
      case 0:
        if (r1) {
          double u1 = s.u1[o0 + x], u3 = s.u3[o0 + x];
          a = u3 * u1;
          b = u1 * u1;
        }
        break;
      case 1:
        if (r1) {
          double u3 = s.u3[o0 + x];
          a = u3 * u3;
        }
        if (r2) b = ((dyfj * s.u1[o0 + x] + dyfjm * s.u1[om + x]) / (2. * dyj)) * s.u2[o0 + x];
        break;
      case 2:
        if (r2) a = ((dyfj * s.u3[o0 + x] + dyfjm * s.u3[om + x]) / (2. * dyj)) * s.u2[o0 + x];
        if (r1) {
          double u1p = s.u1[op + x], u1 = s.u1[o0 + x], u1m = s.u1[om + x];
          double u2p = s.u2[op + x], u2 = s.u2[o0 + x];
          b = (u1p * u2p + u1 * u2p - u1 * u2 - u1m * u2) / (2.0 * dyfj);
        }
        break;
      case 3:
        if (r1) {
          double u3p = s.u3[op + x], u3 = s.u3[o0 + x], u3m = s.u3[om + x];
          double u2p = s.u2[op + x], u2 = s.u2[o0 + x];
          a = (u3p * u2p + u3 * u2p - u3 * u2 - u3m * u2) / (2.0 * dyfj);
        }
        if (r2) {
          double u2 = s.u2[o0 + x];
          double p = u2 + s.u2[op + x], q = u2 + s.u2[om + x];
          b = (0.25 * (p * p) - 0.25 * (q * q)) / dyj;
        }
        break;
      case 4:
        if (rt) {
          double th = s.th[o0 + x];
          a = th * s.u1[o0 + x];
          b = th * s.u3[o0 + x];
        }
        break;
      default:
        if (rt) {
          double thp = s.th[op + x], th = s.th[o0 + x], thm = s.th[om + x];
          double u2p = s.u2[op + x], u2 = s.u2[o0 + x];
          a = (thp * u2p + th * u2p - th * u2 - thm * u2) / (2.0 * dyfj);
        }
        break;
    }
    buf[x] = make_double2(a, b);
  }
  __syncthreads();
  fft_inplace<N, -1>(buf, lane, true, g.twx);
  // combine into the 8 x-half outputs, scaled by 1/Nx
  const double sc = 1.0 / (double)N;
  const int P = N + ZPAD_S;
  for (int idx = threadIdx.x; idx < 8 * g.kxs; idx += blockDim.x) {
    const int o = idx / g.kxs, mm = idx % g.kxs;
    double2 v = make_double2(0.0, 0.0);
    if (mm <= g.nkx) {
      const double k = g.kx[mm];
      double2 dx = make_double2(0.0, 0.0), pl = make_double2(0.0, 0.0);
      bool ok = true;
      switch (o) {
        case 0: ok = r1; dx = sep<N>(sm + 0 * P, mm, 1); pl = sep<N>(sm + 2 * P, mm, 1); break;
        case 1: ok = r1; pl = sep<N>(sm + 0 * P, mm, 0); break;
        case 2: ok = r1; dx = sep<N>(sm + 0 * P, mm, 0); pl = sep<N>(sm + 3 * P, mm, 0); break;
        case 3: ok = r1; pl = sep<N>(sm + 1 * P, mm, 0); break;
        case 4: ok = r2; dx = sep<N>(sm + 1 * P, mm, 1); pl = sep<N>(sm + 3 * P, mm, 1); break;
        case 5: ok = r2; pl = sep<N>(sm + 2 * P, mm, 0); break;
        case 6: ok = rt; dx = sep<N>(sm + 4 * P, mm, 0); pl = sep<N>(sm + 5 * P, mm, 0); break;
        default: ok = rt; pl = sep<N>(sm + 4 * P, mm, 1); break;
      }
      if (ok) v = make_double2((pl.x - k * dx.y) * sc, (pl.y + k * dx.x) * sc);
    }
    s.xh[o][hrow + mm] = v;
  }
}

// ---------------------------------------------------------------------------
// z-pass of the nonlinear terms + spectral RHS + inverse z-pass of cr.
// One CTA = KT kx columns of plane j; 2 KT sequences (N_e, M_e).
// Equation e: 0 -> u1, 1 -> u3, 2 -> u2, 3 -> th.  x-half inputs: xh[2e],
// xh[2e+1]; the inverse-transformed cr_e overwrites xh[2e].
template <int N>
__global__ void __launch_bounds__(2 * KT * (N / 8)) k_zpass_rhs(State s, Geom g, Phys ph, int rk) {
  extern __shared__ double2 sm[];
  constexpr int T = N / 8;
  constexpr int P = N + ZPAD_S;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int kx0 = blockIdx.x * KT, j = blockIdx.y;
  const double hb = s.sc->h_bar[rk];
  const double temp3 = zeta_bar(rk) * hb, temp4 = hb, temp5 = beta_bar(rk) * hb;
  const double nu = ph.nu, f = ph.ro_inv / ph.delta;
  const double tw = ph.delta / ph.ro_inv;  // delta / Ro_inv
  const long long sp0 = (long long)j * g.sp + kx0;
  constexpr int MAXIT = 3;  // ceil(KT * nkzp / blockDim) <= 3 since nkzp <= 2N/3 + 1
  for (int e = 0; e < 4; ++e) {
    const int jlo = (e == 2) ? 2 : (e == 3 ? g.jstart_th : g.jstart);
    const int jhi = (e == 2) ? g.ny : (e == 3 ? g.jend_th : g.jend);
    double2* xin_n = s.xh[2 * e];
    double2* xin_m = s.xh[2 * e + 1];
    const long long h0 = (long long)j * g.hp + kx0;
    if (!in_rng(j, jlo, jhi)) {
      for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x)
        xin_n[h0 + (long long)(idx / KT) * g.kxs + idx % KT] = make_double2(0.0, 0.0);
      continue;
    }
    for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x) {
      int zz = idx / KT, kl = idx % KT;
      long long a = h0 + (long long)zz * g.kxs + kl;
      sm[kl * P + zz] = xin_n[a];
      sm[(KT + kl) * P + zz] = xin_m[a];
    }
    __syncthreads();
    fft_inplace<N, -1>(sm + seq * P, lane, true, g.twz);
    // spectral RHS for every packed (kzp, kl) of the tile
    double2 crv[MAXIT];
    const double inz = 1.0 / (double)N;
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
      const int idx = threadIdx.x + it * blockDim.x;
      crv[it] = make_double2(0.0, 0.0);
      if (idx >= KT * g.nkzp) continue;
      const int kzp = idx / KT, kl = idx % KT, kx = kx0 + kl;
      const int zz = (kzp <= g.nkz) ? kzp : kzp + N - g.nkzp;
      const double kxv = g.kx[kx], kzv = g.kz[kzp];
      const double2 zn = sm[kl * P + zz], zm = sm[(KT + kl) * P + zz];
      // NL = (Z(N) + i kz Z(M)) / Nz
      const double2 nl = make_double2((zn.x - kzv * zm.y) * inz, (zn.y + kzv * zm.x) * inz);
      const long long a = sp0 + (long long)kzp * g.kxs + kl;
      const double kk = pow(kxv * kxv + kzv * kzv, ph.beta);
      double2 cf, cr;
      if (e == 0 || e == 1) {
        const double2 cu1 = s.cu1[a], cu3 = s.cu3[a], cth = s.cth[a], cp = s.cp[a];
        const double2 v2 = make_double2(0.5 * (s.cu2[a].x + s.cu2[a + g.sp].x),
                                        0.5 * (s.cu2[a].y + s.cu2[a + g.sp].y));
        const double2 cu = (e == 0) ? cu1 : cu3;
        cf = cscale(cu, -nu * kk);
        if (e == 0) {
          cf = cadd(cf, cscale(cu3, f));
          cf = cadd(cf, cscale(cth, ph.grav_x));
        } else {
          cf = csub(cf, cscale(cu1, f));
          cf = cadd(cf, cscale(cth, ph.grav_z));
        }
        if (ph.front_tw) {
          const double y = g.gyf[j] - 0.5 * ph.ly;
          const double ax = ph.dthdx * y * tw;          // multiplies ikz
          const double az = -1.0 * ph.dthdz * y * tw;   // multiplies ikx
          const double2 t1 = cmul_i(cu, 1.0);           // i cu
          cf = csub(cf, cscale(t1, ax * kzv));
          cf = csub(cf, cscale(t1, az * kxv));
          const double c2 = (e == 0) ? (-1.0 * ph.dthdz * tw) : (ph.dthdx * tw);
          cf = csub(cf, cscale(v2, c2));
        }
        cf = csub(cf, nl);
        const double kd = (e == 0) ? kxv : kzv;
        cr = cu;
        if (rk > 0) cr = cadd(cr, cscale((e == 0) ? s.cf1[a] : s.cf3[a], temp3));
        cr = csub(cr, cscale(cmul_i(cp, 1.0), temp4 * kd));
        if (e == 0 && kx == 0 && kzp == 0) {
          if (ph.f_type == 1) cr.x -= temp4 * ph.px0;
          if (ph.f_type == 2) cr.x -= temp4 * (ph.px0 + ph.amp_omega0 * cos(ph.omega0 * s.sc->time));
        }
        cr = cadd(cr, cscale(cf, temp5));
        if (e == 0) s.cf1[a] = cf; else s.cf3[a] = cf;
      } else if (e == 2) {
        const double2 cu2 = s.cu2[a];
        cf = cscale(cu2, -nu * kk);
        if (!(kx == 0 && kzp == 0)) {
          const double2 t0 = s.cth[a], tm = s.cth[a - g.sp];
          const double w = ph.grav_y / (2.0 * g.dy[j]);
          cf = cadd(cf, make_double2(w * (t0.x * g.dyf[j - 1] + tm.x * g.dyf[j]),
                                     w * (t0.y * g.dyf[j - 1] + tm.y * g.dyf[j])));
        }
        if (ph.front_tw) {
          const double y = g.gy[j] - 0.5 * ph.ly;
          const double2 t1 = cmul_i(cu2, 1.0);
          cf = csub(cf, cscale(t1, ph.dthdx * y * tw * kzv));
          cf = csub(cf, cscale(t1, -1.0 * ph.dthdz * y * tw * kxv));
        }
        cf = csub(cf, nl);
        cr = cu2;
        if (rk > 0) cr = cadd(cr, cscale(s.cf2[a], temp3));
        const double2 dp = csub(s.cp[a], s.cp[a - g.sp]);
        cr = csub(cr, cscale(dp, temp4 / g.dy[j]));
        cr = cadd(cr, cscale(cf, temp5));
        s.cf2[a] = cf;
      } else {
        const double2 cth = s.cth[a];
        cf = cscale(cth, -(nu / ph.pr) * kk);
        cf = csub(cf, cscale(s.cu1[a], ph.dthdx));
        cf = csub(cf, cscale(s.cu3[a], ph.dthdz));
        if (ph.front_tw) {
          const double y = g.gyf[j] - 0.5 * ph.ly;
          const double2 t1 = cmul_i(cth, 1.0);
          cf = csub(cf, cscale(t1, tw * ph.dthdx * y * kzv));
          cf = csub(cf, cscale(t1, tw * (-1.0) * ph.dthdz * y * kxv));
        }
        cf = csub(cf, nl);
        cr = cth;
        if (rk > 0) cr = cadd(cr, cscale(s.cfth[a], temp3));
        cr = cadd(cr, cscale(cf, temp5));
        s.cfth[a] = cf;
      }
      crv[it] = cr;
    }
    __syncthreads();
    // unpack cr into the second half (zero the de-aliased rows) and invert
    for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x) {
      int zz = idx / KT, kl = idx % KT;
      int kzp = (zz <= g.nkz) ? zz : (zz >= N - g.nkz ? zz - N + g.nkzp : -1);
      if (kzp < 0) sm[(KT + kl) * P + zz] = make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
      const int idx = threadIdx.x + it * blockDim.x;
      if (idx >= KT * g.nkzp) continue;
      const int kzp = idx / KT, kl = idx % KT;
      const int zz = (kzp <= g.nkz) ? kzp : kzp + N - g.nkzp;
      sm[(KT + kl) * P + zz] = crv[it];
    }
    __syncthreads();
    fft_inplace<N, +1>(sm + (KT + seq) * P, lane, seq < KT, g.twz);
    for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x) {
      int zz = idx / KT, kl = idx % KT;
      xin_n[h0 + (long long)zz * g.kxs + kl] = sm[(KT + kl) * P + zz];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// implicit systems: rows of the four equations (th, u2, u1, u3) -> tri[eq*np + j]
__global__ void k_tri_coef(Geom g, Phys ph, TriRow* tri, DevScalars* sc, int rk) {
  const int eq = threadIdx.x;  // 0..3
  if (eq >= 4) return;
  const int np = g.np, Nyp = g.ny;
  TriRow* R = tri + eq * np;
  const double temp1 = 0.5 * ph.nu * sc->h_bar[rk];
  const double tv = temp1 * ph.nu_v_scale;
  const double tth = temp1 / ph.pr * ph.nu_v_scale;
  for (int j = 0; j < np; ++j) {
    R[j].l = 0.0; R[j].d = 1.0; R[j].u = 0.0; R[j].bc = 0.0;
    R[j].is_bc = 1; R[j].interior = 0; R[j].cn_lo = 0.0; R[j].cn_hi = 0.0;
  }
  const double* dy = g.dy;
  const double* dyf = g.dyf;
  auto setr = [&](int j, double l, double d, double u, double v) {
    R[j].l = l; R[j].d = d; R[j].u = u; R[j].bc = v; R[j].is_bc = 1; R[j].interior = 0;
  };
  if (eq == 0 || eq == 2 || eq == 3) {
    const int lo = (eq == 0) ? g.jstart_th : g.jstart;
    const int hi = (eq == 0) ? g.jend_th : g.jend;
    for (int j = lo; j <= hi; ++j) {
      if (eq == 0) {  // solver.f90:1023-1026
        R[j].l = -(tth) / (dy[j] * dyf[j]);
        R[j].d = 1. + (tth) / (dy[j + 1] * dyf[j]) + (tth) / (dy[j] * dyf[j]);
        R[j].u = -(tth) / (dy[j + 1] * dyf[j]);
        R[j].cn_hi = (tth) / dyf[j] / dy[j + 1];
        R[j].cn_lo = (tth) / dyf[j] / dy[j];
      } else {        // solver.f90:1140-1143, 1196-1199
        R[j].l = -tv / (dy[j] * dyf[j]);
        R[j].d = 1. - tv * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]));
        R[j].u = -tv / (dy[j + 1] * dyf[j]);
        R[j].cn_hi = tv / dyf[j] / dy[j + 1];
        R[j].cn_lo = tv / dyf[j] / dy[j];
      }
      R[j].is_bc = 0; R[j].interior = 1;
    }
    // apply_BC_th/1/3 lower and upper (solver.f90:1901-1982, 2066-2232)
    const int bl = (eq == 0) ? BC_TH_MIN : (eq == 2 ? BC_U_MIN : BC_W_MIN);
    const int bh = (eq == 0) ? BC_TH_MAX : (eq == 2 ? BC_U_MAX : BC_W_MAX);
    double cmax = ph.bc_c1[bh];
    if (eq == 3 && ph.bc_type[BC_W_MAX] == 1) {
      if (ph.f_type == 4)
        sc->w_bc_ymax_c1_transient = ph.bc_c1[BC_W_MAX] + ph.amp_omega0 *
            sin(ph.omega0 * (ph.ro_inv / ph.delta * sc->time - ph.force_start));
      cmax = sc->w_bc_ymax_c1_transient;
    }
    if (ph.bc_type[bl] == 0) {
      setr(0, 0., 1., 0., 0.);
      setr(1, 0., 1., 0., ph.bc_c1[bl]);
    } else {
      setr(0, 0., 1., 0., 0.);
      setr(1, 0., -1., 1., dy[2] * ph.bc_c1[bl]);
    }
    if (ph.bc_type[bh] == 0) {
      setr(Nyp + 1, 0., 1., 0., 0.);
      setr(Nyp, 0., 1., 0., cmax);
    } else {
      setr(Nyp, -1., 1., 0., dy[Nyp] * cmax);
      setr(Nyp + 1, 0., 1., 0., 0.);
    }
  } else {  // u2, solver.f90:1085-1088 and apply_BC_2_* (1987-2061)
    for (int j = 2; j <= Nyp; ++j) {
      R[j].l = -tv / (dyf[j - 1] * dy[j]);
      R[j].d = 1. + tv / (dyf[j] * dy[j]) + tv / (dyf[j - 1] * dy[j]);
      R[j].u = -tv / (dyf[j] * dy[j]);
      R[j].cn_hi = tv / dy[j] / dyf[j];
      R[j].cn_lo = tv / dy[j] / dyf[j - 1];
      R[j].is_bc = 0; R[j].interior = 1;
    }
    if (ph.bc_type[BC_V_MIN] == 0) {
      setr(1, 0., 1., 0., ph.bc_c1[BC_V_MIN]);
      setr(2, 0., 1., 0., ph.bc_c1[BC_V_MIN]);
    } else {
      setr(1, 0., -1., 1., dyf[1] * ph.bc_c1[BC_V_MIN]);
    }
    setr(0, 0., 1., 0., 0.);
    if (ph.bc_type[BC_V_MAX] == 0) {
      setr(Nyp + 1, 0., 1., 0., ph.bc_c1[BC_V_MAX]);
      setr(Nyp, 0., 1., 0., ph.bc_c1[BC_V_MAX]);
    } else {
      setr(Nyp + 1, -1., 1., 0., dyf[Nyp] * ph.bc_c1[BC_V_MAX]);
    }
  }
  // Thomas forward elimination of the matrix (thomas_forward_real_mpi with
  // one rank: rows 1..Nyp+1, solver.f90:1731-1757)
  double bprev = R[0].d;
  R[0].ap = 0.0;
  R[0].ibp = 1.0 / bprev;
  for (int j = 1; j < np; ++j) {
    const double a = -R[j].l / bprev;
    const double b = R[j].d + a * R[j - 1].u;
    R[j].ap = a;
    R[j].ibp = 1.0 / b;
    bprev = b;
  }
}

// per-column Thomas for the four equations, one thread per (x, z)
__global__ void __launch_bounds__(128) k_thomas(State s, Geom g) {
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= g.pp) return;
  const int np = g.np, Nyp = g.ny;
  const long long pp = g.pp;
  for (int eq = 0; eq < 4; ++eq) {
    const TriRow* R = s.tri + eq * np;
    double* u = (eq == 0) ? s.th : (eq == 1 ? s.u2 : (eq == 2 ? s.u1 : s.u3));
    const double* r = (eq == 0) ? s.rth : (eq == 1 ? s.r2 : (eq == 2 ? s.r1 : s.r3));
    u += col;
    r += col;
    // rows written back (solver.f90:1056, 1115, 1171, 1227)
    const int lo = (eq == 0) ? g.jstart_th - 1 : (eq == 1 ? 1 : g.jstart - 1);
    const int hi = (eq == 0) ? g.jend_th + 1 : (eq == 1 ? Nyp + 1 : g.jend + 1);
    double um = 0.0, uc = u[0], gprev = 0.0, g0 = 0.0, glast = 0.0;
    for (int j = 0; j < np; ++j) {
      const double un = (j + 1 < np) ? u[(long long)(j + 1) * pp] : 0.0;
      const TriRow row = R[j];
      double vec;
      if (row.is_bc) vec = row.bc;
      else vec = r[(long long)j * pp] + (row.cn_hi * (un - uc) - row.cn_lo * (uc - um));
      const double gj = (j == 0) ? vec : vec + row.ap * gprev;
      if (j >= lo && j <= hi) u[(long long)j * pp] = gj;
      if (j == 0) g0 = gj;
      glast = gj;
      gprev = gj;
      um = uc;
      uc = un;
    }
    double xn = glast * R[np - 1].ibp;
    if (np - 1 >= lo && np - 1 <= hi) u[(long long)(np - 1) * pp] = xn;
    for (int j = np - 2; j >= 0; --j) {
      const double gj = (j >= lo && j <= hi) ? u[(long long)j * pp] : (j == 0 ? g0 : 0.0);
      const double x = (gj - R[j].u * xn) * R[j].ibp;
      if (j >= lo && j <= hi) u[(long long)j * pp] = x;
      xn = x;
    }
  }
}

// ---------------------------------------------------------------------------
// rem_div factors: per (kx, kzp) column, rows 1..Nyp of the Poisson system
// (solver.f90:1326-1333 with apply_BC_rem_div_mpi 2341-2368), forward
// eliminated once: pfac[j] = (a'_j, 1/b'_j).
__global__ void k_pfac(Geom g, double2* pfac) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  if (kx > g.nkx) return;
  const int Nyp = g.ny;
  const double kx2 = g.kx[kx] * g.kx[kx], kz2 = g.kz[kzp] * g.kz[kzp];
  const bool zero_mode = (kx == 0 && kzp == 0);
  auto row = [&](int j, double& l, double& d, double& u) {
    if (j == 1) { l = 0.; d = 1.; u = zero_mode ? 0. : -1.; return; }
    if (j == Nyp) { l = 1.; d = -1.; u = 0.; return; }
    l = 1. / (g.dy[j] * g.dyf[j]);
    d = -kx2 - kz2 - 1. / (g.dy[j + 1] * g.dyf[j]) - 1. / (g.dy[j] * g.dyf[j]);
    u = 1. / (g.dy[j + 1] * g.dyf[j]);
  };
  double l, d, u, lp, dp, up;
  row(1, lp, dp, up);
  double bprev = dp;
  pfac[(long long)1 * g.sp + (long long)kzp * g.kxs + kx] = make_double2(0.0, 1.0 / dp);
  for (int j = 2; j <= Nyp; ++j) {
    row(j, l, d, u);
    const double a = -l / bprev;
    const double b = d + a * up;
    pfac[(long long)j * g.sp + (long long)kzp * g.kxs + kx] = make_double2(a, 1.0 / b);
    bprev = b;
    up = u;
  }
}

// divergence removal + pressure update, one thread per (kx, kzp) column
__global__ void __launch_bounds__(128) k_rem_div(State s, Geom g, int rk, int update_cp) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  if (kx > g.nkx) return;
  const int Nyp = g.ny;
  const long long c0 = (long long)kzp * g.kxs + kx, sp = g.sp;
  const double kxv = g.kx[kx], kzv = g.kz[kzp];
  const bool zero_mode = (kx == 0 && kzp == 0);
  // forward sweep: g_1 = 0 (BC row), g_j = rhs_j + a'_j g_{j-1}; rhs_Nyp = 0
  double2 gp = make_double2(0.0, 0.0);
  s.phi_g[1 * sp + c0] = gp;
  double2 u2c = s.cu2[2 * sp + c0];
  for (int j = 2; j <= Nyp; ++j) {
    const double2 pf = s.pfac[j * sp + c0];
    double2 rhs = make_double2(0.0, 0.0);
    const double2 u2n = s.cu2[(long long)(j + 1) * sp + c0];
    if (j < Nyp) {
      const double2 a1 = s.cu1[j * sp + c0], a3 = s.cu3[j * sp + c0];
      const double idf = 1.0 / g.dyf[j];
      rhs = make_double2(-kxv * a1.y + (u2n.x - u2c.x) * idf - kzv * a3.y,
                         kxv * a1.x + (u2n.y - u2c.y) * idf + kzv * a3.x);
    }
    gp = make_double2(rhs.x + pf.x * gp.x, rhs.y + pf.x * gp.y);
    s.phi_g[j * sp + c0] = gp;
    u2c = u2n;
  }
  // backward sweep with the projection (solver.f90:1361-1376) and cp update
  const double itemp4 = 1.0 / s.sc->h_bar[rk];
  double2 phin = make_double2(0.0, 0.0);
  for (int j = Nyp; j >= 1; --j) {
    const double2 pf = s.pfac[j * sp + c0];
    const double2 gj = s.phi_g[j * sp + c0];
    double cj;
    if (j == Nyp) cj = 0.0;
    else if (j == 1) cj = zero_mode ? 0.0 : -1.0;
    else cj = 1.0 / (g.dy[j + 1] * g.dyf[j]);
    const double2 phi = (j == Nyp) ? make_double2(gj.x * pf.y, gj.y * pf.y)
                                   : make_double2((gj.x - cj * phin.x) * pf.y, (gj.y - cj * phin.y) * pf.y);
    const long long a = j * sp + c0;
    double2 v1 = s.cu1[a], v3 = s.cu3[a];
    v1.x += kxv * phi.y; v1.y -= kxv * phi.x;   // cu1 -= i kx phi
    v3.x += kzv * phi.y; v3.y -= kzv * phi.x;   // cu3 -= i kz phi
    s.cu1[a] = v1;
    s.cu3[a] = v3;
    if (j + 1 <= Nyp) {  // cu2(j+1) -= (phi(j+1) - phi(j)) / dy(j+1)
      const long long b = (long long)(j + 1) * sp + c0;
      const double w = 1.0 / g.dy[j + 1];
      double2 v2 = s.cu2[b];
      v2.x -= (phin.x - phi.x) * w;
      v2.y -= (phin.y - phi.y) * w;
      s.cu2[b] = v2;
    }
    if (update_cp && j >= g.jstart && j <= g.jend) {
      double2 p = s.cp[a];
      p.x += phi.x * itemp4;
      p.y += phi.y * itemp4;
      s.cp[a] = p;
    }
    phin = phi;
  }
}

// ---------------------------------------------------------------------------
// courant: CFL minimum over the physical velocity (flow.f90:781-808)
__device__ __forceinline__ unsigned long long dbits(double v) { return (unsigned long long)__double_as_longlong(v); }

__global__ void __launch_bounds__(256) k_courant_reduce(State s, Geom g, Phys ph, CflCtl ctl) {
  DevScalars* sc = s.sc;
  if (!ctl.force && !(ctl.variable_dt && (sc->time_step % ctl.update_dt) == 0)) return;
  const long long n = (long long)g.pp;
  const int jlo = ph.front ? g.jstart : 1, jhi = ph.front ? g.jend : g.ny;
  const long long total = (long long)(jhi - jlo + 1) * n;
  const double f = ph.ro_inv / ph.delta;
  double dmin = __longlong_as_double(0x7ff0000000000000LL);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int j = jlo + (int)(idx / n);
    const long long p = (long long)j * n + idx % n;
    double dx, dyv, dz;
    if (ph.front) {
      dx = ctl.cfl * ph.dx / fabs(s.u1[p] - ph.dthdz * g.gyf[j] / f);
      dyv = ctl.cfl * g.dy[j] / fabs(s.u2[p]);
      dz = ctl.cfl * ph.dz / fabs(s.u3[p] + (1.0 / f) * ph.dthdx * (g.gyf[j] - 0.5 * ph.ly));
    } else {
      dx = ctl.cfl * ph.dx / fabs(s.u1[p]);
      dyv = ctl.cfl * g.dy[j] / fabs(s.u2[p]);
      dz = ctl.cfl * ph.dz / fabs(s.u3[p]);
    }
    dmin = fmin(dmin, fmin(dx, fmin(dyv, dz)));
    if (!isfinite(s.u1[p]) || !isfinite(s.u2[p]) || !isfinite(s.u3[p])) atomicOr(&sc->flags, 1);
  }
  for (int o = 16; o > 0; o >>= 1) dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dmin;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) dmin = fmin(dmin, red[w]);
    if (dmin >= 0.0) atomicMin(&sc->dt_min_bits, dbits(dmin));
  }
}

__global__ void k_courant_final(DevScalars* sc, Phys ph, CflCtl ctl) {
  if (!ctl.force && !(ctl.variable_dt && (sc->time_step % ctl.update_dt) == 0)) return;
  // flow.f90:758-773 (0.1 is a single-precision literal)
  double dt = 1.0;
  dt = fmin(dt, 0.5 * pow(fmin(ph.dx, ph.dz), 2.0 * ph.beta) / ph.nu);
  dt = fmin(dt, dt * ph.nu / (ph.nu / ph.pr));
  if (ph.ro_inv != 0.0) dt = fmin(dt, 2.0 * ph.pi_ref / fabs(ph.ro_inv / ph.delta) / 20.0);
  {
    const double nmax = sqrt(fabs(ph.bc_c1[BC_TH_MIN]));
    dt = fmin(dt, (double)0.1f * 2.0 * ph.pi_ref / nmax);
  }
  dt = fmin(dt, __longlong_as_double((long long)sc->dt_min_bits));
  sc->dt_min_bits = dbits(__longlong_as_double(0x7ff0000000000000LL));
  // flow.f90:812-854
  double delta_t;
  if (dt <= 0) { delta_t = 0.00001; sc->flags |= 2; }
  else if (dt >= 1000.) { delta_t = 1000.0; sc->flags |= 4; }
  else delta_t = dt;
  const double tl = ctl.time_limit, t = sc->time;
  const double next = fmin(fmin(tl, sc->save_stats_time - t), fmin(sc->save_flow_time - t, tl - t));
  const double r_max = (double)(1.0f - 0.025f);
  if (next < dt) delta_t = next + 1.e-14;
  else if (next < (1. + r_max) * dt) delta_t = 1. / (1. + r_max) * next;
  else delta_t = dt;
  if (delta_t < 1.e-10) sc->flags |= 8;
  // rk_chan_1 froze temp1..temp5 at its start (solver.f90:385-389): the new
  // dt takes effect after the substep's projection and pressure update
  sc->dt_next = delta_t;
  sc->dt_pending = 1;
}

// flow.f90:852-854, applied once the substep that called courant is done
__global__ void k_apply_dt(DevScalars* sc) {
  if (!sc->dt_pending) return;
  const double delta_t = sc->dt_next;
  sc->delta_t = delta_t;
  sc->h_bar[0] = delta_t * (8.0 / 15.0);
  sc->h_bar[1] = delta_t * (2.0 / 15.0);
  sc->h_bar[2] = delta_t * (5.0 / 15.0);
  sc->dt_pending = 0;
}

__global__ void k_step_begin(DevScalars* sc) { sc->time_step += 1; }
__global__ void k_step_end(DevScalars* sc) { sc->time += sc->delta_t; }

// max |div| at GYF rows 2..Nyp-1 (the rows rem_div zeroes)
__global__ void k_divergence(State s, Geom g) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  double m = 0.0;
  if (kx <= g.nkx) {
    const long long c0 = (long long)kzp * g.kxs + kx, sp = g.sp;
    const double kxv = g.kx[kx], kzv = g.kz[kzp];
    for (int j = 2; j <= g.ny - 1; ++j) {
      const double2 a1 = s.cu1[j * sp + c0], a3 = s.cu3[j * sp + c0];
      const double2 b = s.cu2[j * sp + c0], c = s.cu2[(j + 1) * sp + c0];
      const double idf = 1.0 / g.dyf[j];
      const double re = -kxv * a1.y + (c.x - b.x) * idf - kzv * a3.y;
      const double im = kxv * a1.x + (c.y - b.y) * idf + kzv * a3.x;
      m = fmax(m, sqrt(re * re + im * im));
    }
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax((unsigned long long*)&s.sc->max_div, dbits(m));
}

// apply_BC_vel_mpi_post on the spectral velocity (flow.f90:1161-1360)
__global__ void k_bc_vel_post(State s, Geom g, Phys ph) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  if (kx > g.nkx) return;
  const long long c0 = (long long)kzp * g.kxs + kx, sp = g.sp;
  const int Nyp = g.ny;
  const bool m0 = (kx == 0 && kzp == 0);
  const double2 Z = make_double2(0.0, 0.0);
  auto R = [&](double v) { return make_double2(v, 0.0); };
  double2 *cu1 = s.cu1 + c0, *cu2 = s.cu2 + c0, *cu3 = s.cu3 + c0;
  // lower
  if (ph.bc_type[BC_U_MIN] == 0) {
    cu1[0] = Z; cu1[sp] = Z;
    if (m0) { cu1[sp] = R(ph.bc_c1[BC_U_MIN]); cu1[0] = R(ph.bc_c1[BC_U_MIN]); }
  } else {
    cu1[sp] = cu1[2 * sp]; cu1[0] = cu1[sp];
    if (m0) {
      cu1[sp] = csub(cu1[2 * sp], R(g.dy[2] * ph.bc_c1[BC_U_MIN]));
      cu1[0] = csub(cu1[sp], R(g.dy[1] * ph.bc_c1[BC_U_MIN]));
    }
  }
  if (ph.bc_type[BC_W_MIN] == 0) {
    cu3[0] = Z; cu3[sp] = Z;
    if (m0) { cu3[sp] = R(ph.bc_c1[BC_W_MIN]); cu3[0] = R(ph.bc_c1[BC_W_MIN]); }
  } else {
    cu3[sp] = cu3[2 * sp]; cu3[0] = cu3[sp];
    if (m0) {
      cu3[sp] = csub(cu3[2 * sp], R(g.dy[2] * ph.bc_c1[BC_W_MIN]));
      cu3[0] = csub(cu3[sp], R(g.dy[1] * ph.bc_c1[BC_W_MIN]));
    }
  }
  if (ph.bc_type[BC_V_MIN] == 0) {
    cu2[sp] = csub(R(2.0 * ph.bc_c1[BC_V_MIN]), cu2[2 * sp]);
    cu2[0] = cu2[sp];
  } else {
    cu2[sp] = cu2[2 * sp]; cu2[0] = cu2[sp];
    if (m0) {
      cu2[sp] = csub(cu2[2 * sp], R(g.dyf[1] * ph.bc_c1[BC_V_MIN]));
      cu2[0] = csub(cu2[sp], R(g.dyf[1] * ph.bc_c1[BC_V_MIN]));
    }
  }
  // upper
  const long long N0 = (long long)Nyp * sp, N1 = (long long)(Nyp + 1) * sp, Nm = (long long)(Nyp - 1) * sp;
  if (ph.bc_type[BC_U_MAX] == 0) {
    cu1[N0] = Z; cu1[N1] = Z;
    if (m0) { cu1[N0] = R(ph.bc_c1[BC_U_MAX]); cu1[N1] = R(ph.bc_c1[BC_U_MAX]); }
  } else {
    cu1[N0] = cu1[Nm]; cu1[N1] = cu1[N0];
    if (m0) {
      cu1[N0] = cadd(cu1[Nm], R(g.dy[Nyp] * ph.bc_c1[BC_U_MAX]));
      cu1[N1] = cadd(cu1[N0], R(g.dy[Nyp] * ph.bc_c1[BC_U_MAX]));
    }
  }
  if (ph.bc_type[BC_W_MAX] == 0) {
    cu3[N0] = Z; cu3[N1] = Z;
    if (m0) { cu3[N0] = R(ph.bc_c1[BC_W_MAX]); cu3[N1] = Z; }
  } else {
    cu3[N0] = cu3[Nm]; cu3[N1] = cu3[N0];
    if (m0) {
      double wt = ph.bc_c1[BC_W_MAX];
      if (ph.f_type == 4)
        wt = ph.bc_c1[BC_W_MAX] + ph.amp_omega0 * sin(ph.omega0 * (ph.ro_inv / ph.delta * s.sc->time - ph.force_start));
      cu3[N0] = cadd(cu3[Nm], R(g.dy[Nyp] * wt));
      cu3[N1] = cadd(cu3[N0], R(g.dy[Nyp] * wt));
    }
  }
  if (ph.bc_type[BC_V_MAX] == 0) {
    if (m0) cu2[N1] = csub(R(2.0 * ph.bc_c1[BC_V_MAX]), cu2[N0]);
  } else {
    cu2[N0] = cu2[Nm]; cu2[N1] = cu2[N0];
    if (m0) cu2[N1] = cadd(cu2[N0], R(g.dy[Nyp] * ph.bc_c1[BC_V_MAX]));
  }
}

// ---------------------------------------------------------------------------
// launchers

template <int N>
static void go_products(const Geom& g, const State& s, cudaStream_t st) {
  size_t smem = (size_t)6 * (N + ZPAD_S) * sizeof(double2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_products<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_products<N><<<dim3(g.nz, g.np), 6 * (N / 8), smem, st>>>(s, g);
}
template <int N>
static void go_zpass(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st) {
  size_t smem = (size_t)2 * KT * (N + ZPAD_S) * sizeof(double2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_zpass_rhs<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_zpass_rhs<N><<<dim3(g.kxs / KT, g.np), 2 * KT * (N / 8), smem, st>>>(s, g, ph, rk);
}

#define DB_DISPATCH_N2(n, FN, ...)                  \
  switch (n) {                                      \
    case 16: FN<16>(__VA_ARGS__); break;            \
    case 32: FN<32>(__VA_ARGS__); break;            \
    case 64: FN<64>(__VA_ARGS__); break;            \
    case 128: FN<128>(__VA_ARGS__); break;          \
    case 256: FN<256>(__VA_ARGS__); break;          \
    case 512: FN<512>(__VA_ARGS__); break;          \
    case 1024: FN<1024>(__VA_ARGS__); break;        \
    default: return cudaErrorInvalidValue;          \
  }

cudaError_t launch_products(const Geom& g, const State& s, cudaStream_t st) {
  DB_DISPATCH_N2(g.nx, go_products, g, s, st);
  return cudaGetLastError();
}
cudaError_t launch_zpass_rhs(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st) {
  DB_DISPATCH_N2(g.nz, go_zpass, g, ph, s, rk, st);
  return cudaGetLastError();
}
cudaError_t launch_tri_coef(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st) {
  k_tri_coef<<<1, 32, 0, st>>>(g, ph, s.tri, s.sc, rk);
  return cudaGetLastError();
}
cudaError_t launch_thomas(const Geom& g, const State& s, cudaStream_t st) {
  long long n = g.pp;
  k_thomas<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(s, g);
  return cudaGetLastError();
}
cudaError_t launch_courant(const Geom& g, const Phys& ph, const State& s, CflCtl ctl, cudaStream_t st) {
  k_courant_reduce<<<148 * 8, 256, 0, st>>>(s, g, ph, ctl);
  k_courant_final<<<1, 1, 0, st>>>(s.sc, ph, ctl);
  return cudaGetLastError();
}
cudaError_t launch_rem_div(const Geom& g, const State& s, int rk, int update_cp, cudaStream_t st) {
  k_rem_div<<<dim3((g.nkx + 1 + 127) / 128, g.nkzp), 128, 0, st>>>(s, g, rk, update_cp);
  return cudaGetLastError();
}
cudaError_t launch_pfac(const Geom& g, const State& s, cudaStream_t st) {
  k_pfac<<<dim3((g.nkx + 1 + 127) / 128, g.nkzp), 128, 0, st>>>(g, s.pfac);
  return cudaGetLastError();
}
cudaError_t launch_apply_dt(DevScalars* sc, cudaStream_t st) {
  k_apply_dt<<<1, 1, 0, st>>>(sc);
  return cudaGetLastError();
}
cudaError_t launch_step_begin(DevScalars* sc, cudaStream_t st) {
  k_step_begin<<<1, 1, 0, st>>>(sc);
  return cudaGetLastError();
}
cudaError_t launch_step_end(DevScalars* sc, cudaStream_t st) {
  k_step_end<<<1, 1, 0, st>>>(sc);
  return cudaGetLastError();
}
cudaError_t launch_divergence(const Geom& g, const State& s, cudaStream_t st) {
  k_divergence<<<dim3((g.nkx + 1 + 127) / 128, g.nkzp), 128, 0, st>>>(s, g);
  return cudaGetLastError();
}
cudaError_t launch_bc_vel_post(const Geom& g, const Phys& ph, const State& s, cudaStream_t st) {
  k_bc_vel_post<<<dim3((g.nkx + 1 + 127) / 128, g.nkzp), 128, 0, st>>>(s, g, ph);
  return cudaGetLastError();
}

}  // namespace db
