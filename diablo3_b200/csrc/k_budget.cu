// k_budget.cu -- the energy-budget statistics of save_stats_chan that need
// the mean flow as a function of x (for/diagnostics.f90: compute_TKE
// 1254-1360, compute_TKE_Production 1366-1520, compute_MKE_diss 1097-1250,
// compute_Vorticity 1525-1730, compute_BPE 1733-1856), in FP64 on both
// precision paths.
//
// The means follow compute_averages (676-800): with homogeneousX the x-z
// mean of each plane (the (0,0) mode) at every x; otherwise the z-mean of
// each x line.  The z-lines are read from FP64 physical copies of u1, u2,
// u3 (inverse transforms of the FP64 state into scratch); the x-derivatives
// of the z-means come from the kz = 0 row of the spectral state (the
// reference transforms i kx cr(kx, 0, j) to physical space), evaluated per
// x as a direct sum over the retained kx.  One CTA per plane, threads over x.
// The vorticity rms is a plane sum of squared spectral combinations, taken
// by Parseval over the retained modes; the BPE histogram runs over the
// physical buoyancy with its background gradient added.
#include <math.h>

#include "db_kernels.cuh"

namespace db {

enum BudRow {
  BU_TKE, BU_UU_DUDX, BU_WU_DWDX, BU_VU_DVDX, BU_VV_DVDY, BU_UV_DUDY, BU_WV_DWDY, BU_EPS_M,
  BU_OMX, BU_OMY, BU_OMZ, NBUD
};

// z-means of u1, u2, u3 per (plane, x) into mxy[f][j][x] (x-z means with homx)
__global__ void __launch_bounds__(256) k_zmeans(const __grid_constant__ State s, Geom g,
                                                const __grid_constant__ FieldSet phys, int homx, double* mxy) {
  const int j = blockIdx.x, np = g.np, nx = g.nx, nz = g.nz;
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    for (int f = 0; f < 3; ++f) {
      double m;
      if (homx) {
        const double2* cu = f == 0 ? s.cu1 : (f == 1 ? s.cu2 : s.cu3);
        m = cu[(long long)j * g.sp].x;
      } else {
        const double* u = (const double*)phys.p[f] + (long long)j * g.pp + x;
        m = 0.0;
        for (int z = 0; z < nz; ++z) m += u[(long long)z * nx];
        m /= (double)nz;
      }
      mxy[((long long)f * np + j) * nx + x] = m;
    }
  }
}

// d/dx of the z-mean of field cu at plane j, point x: the kz = 0 row i kx
// cu(kx, 0, j) to physical space (inverse transform, unnormalised)
__device__ __forceinline__ double ddx_zmean(const double2* cu, const Geom& g, int j, int x) {
  const double2* row = cu + (long long)j * g.sp;
  double acc = 0.0;
  for (int kx = 1; kx <= g.nkx; ++kx) {
    double sn, cs;
    sincospi(2.0 * (double)kx * (double)x / (double)g.nx, &sn, &cs);
    const double2 c = row[kx];
    const double k = g.kx[kx];
    // 2 Re(i k c e^{i th}) = -2 k (c.x sin + c.y cos)
    acc += -2.0 * k * (c.x * sn + c.y * cs);
  }
  return acc;
}

__global__ void __launch_bounds__(256) k_budget(const __grid_constant__ State s, Geom g, Phys ph,
                                                const __grid_constant__ FieldSet phys, int homx, const double* mxy,
                                                double* out) {
  const int j = blockIdx.x, np = g.np, nx = g.nx, nz = g.nz, Nyp = g.ny;
  const long long pp = g.pp;
  const double* U1 = (const double*)phys.p[0];
  const double* U2 = (const double*)phys.p[1];
  const double* U3 = (const double*)phys.p[2];
  auto M = [&](int f, int jj, int x) { return mxy[((long long)f * np + jj) * nx + x]; };
  const bool gyf = (j >= 1 && j <= Nyp), gyr = (j >= 2 && j <= Nyp);
  const double tws = ph.front_tw ? (ph.delta / ph.ro_inv) * ph.dthdx : 0.0;   // thermal-wind shear
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // TKE, 6 production terms, epsilon_m
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    if (!gyf) break;
    // z-line statistics of the fluctuations about the means (compute_TKE,
    // compute_TKE_Production)
    const double m1 = M(0, j, x), m2 = M(1, j, x), m3 = M(2, j, x);
    double uu = 0, vv = 0, ww = 0, uw = 0, uv = 0, wv = 0;
    const double m1m = j >= 1 ? M(0, j - 1, x) : 0.0, m3m = j >= 1 ? M(2, j - 1, x) : 0.0;
    for (int z = 0; z < nz; ++z) {
      const long long o = (long long)j * pp + (long long)z * nx + x;
      const double a1 = U1[o] - m1, a2 = U2[o] - m2, a3 = U3[o] - m3;
      uu += a1 * a1;
      vv += a2 * a2;
      ww += a3 * a3;
      uw += a1 * a3;
      if (gyr) {
        const double b1 = U1[o - pp] - m1m, b3 = U3[o - pp] - m3m;
        uv += (g.dyf[j - 1] * a1 + g.dyf[j] * b1) / (2.0 * g.dy[j]) * a2;
        wv += (g.dyf[j - 1] * a3 + g.dyf[j] * b3) / (2.0 * g.dy[j]) * a2;
      }
    }
    const double inz = 1.0 / (double)nz;
    uu *= inz; vv *= inz; ww *= inz; uw *= inz; uv *= inz; wv *= inz;
    acc[0] += 0.5 * (uu + vv + ww);
    // mean-flow gradients (compute_MKE_diss): x-derivatives of the z-means
    // (zero with homogeneousX, where the reference skips compute_MKE_diss)
    const double dudx = homx ? 0.0 : ddx_zmean(s.cu1, g, j, x);
    const double dvdx = homx ? 0.0 : ddx_zmean(s.cu2, g, j, x);
    const double dwdx = homx ? 0.0 : ddx_zmean(s.cu3, g, j, x);
    acc[1] += uu * dudx;   // uu_dudx (GYF)
    acc[2] += uw * dwdx;   // wu_dwdx (GYF)
    if (gyr) {
      const double dvdy = (M(1, j + 1, x) - M(1, j - 1, x)) / (g.gy[j + 1] - g.gy[j - 1]);
      const double dudy = (m1 - m1m) / g.dy[j];
      const double dwdy = (m3 - m3m) / g.dy[j] + tws;
      acc[3] += uv * dvdx;   // vu_dvdx (GY)
      acc[4] += dvdy * vv;   // vv_dvdy
      acc[5] += dudy * uv;   // uv_dudy
      acc[6] += dwdy * wv;   // wv_dwdy
      if (!homx) acc[7] += dudy * dudy + dvdy * dvdy + dwdy * dwdy;
    }
    if (!homx) {
      // the x-derivative terms of epsilon_m: du/dx, dw/dx at GYF rows j, j-1
      // interpolated as squares, dv/dx at row j (compute_MKE_diss)
      const double dudxm = ddx_zmean(s.cu1, g, j - 1, x), dwdxm = ddx_zmean(s.cu3, g, j - 1, x);
      const double w0 = g.dyf[j - 1] / (2.0 * g.dy[j]), w1 = g.dyf[j] / (2.0 * g.dy[j]);
      acc[7] += w0 * dudx * dudx + w1 * dudxm * dudxm + dvdx * dvdx + w0 * dwdx * dwdx + w1 * dwdxm * dwdxm;
    }
  }
  __shared__ double red[8][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k][threadIdx.x];
    v /= (double)nx;
    if (threadIdx.x == 7) v *= ph.nu;
    out[(long long)threadIdx.x * np + j] = v;
  }
}

// rms vorticity of plane j (compute_Vorticity) by Parseval over the
// retained modes; omega_x carries the thermal-wind shear in its mean
__global__ void __launch_bounds__(256) k_vorticity(const __grid_constant__ State s, Geom g, Phys ph, double* out) {
  const int j = blockIdx.x, np = g.np, Nyp = g.ny;
  const long long sp = g.sp;
  const int nk = g.nkx + 1, nmodes = g.nkzp * nk;
  double ax = 0.0, ay = 0.0, az = 0.0;
  const bool in = (j >= 1 && j <= Nyp);
  const double tws = ph.front_tw ? (ph.delta / ph.ro_inv) * ph.dthdx : 0.0;
  for (int m = threadIdx.x; in && m < nmodes; m += blockDim.x) {
    const int kzp = m / nk, kx = m % nk;
    const long long a = (long long)j * sp + (long long)kzp * g.kxs + kx;
    const double w = kx == 0 ? 1.0 : 2.0;
    const double kxv = g.kx[kx], kzv = g.kz[kzp];
    const double i2f = 1.0 / (2.0 * g.dyf[j]);
    const double2 u1 = s.cu1[a], u3 = s.cu3[a];
    const double2 u1p = s.cu1[a + sp], u1m = s.cu1[a - sp], u3p = s.cu3[a + sp], u3m = s.cu3[a - sp];
    const double2 v = make_double2(0.5 * (s.cu2[a + sp].x + s.cu2[a].x), 0.5 * (s.cu2[a + sp].y + s.cu2[a].y));
    // omega_x = i kz <u2> - d u3 / dy, omega_y = i kx u3 - i kz u1,
    // omega_z = d u1 / dy - i kx <u2>
    double2 ox = make_double2(-kzv * v.y - (u3p.x - u3m.x) * i2f, kzv * v.x - (u3p.y - u3m.y) * i2f);
    if (kx == 0 && kzp == 0) ox.x -= tws;
    const double2 oy = make_double2(-kxv * u3.y + kzv * u1.y, kxv * u3.x - kzv * u1.x);
    const double2 oz = make_double2((u1p.x - u1m.x) * i2f + kxv * v.y, (u1p.y - u1m.y) * i2f - kxv * v.x);
    ax += w * (ox.x * ox.x + ox.y * ox.y);
    ay += w * (oy.x * oy.x + oy.y * oy.y);
    az += w * (oz.x * oz.x + oz.y * oz.y);
  }
  __shared__ double red[8][3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double v3[3] = {ax, ay, az};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double v = v3[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k][threadIdx.x];
    out[(long long)(BU_OMX + threadIdx.x) * np + j] = sqrt(v);
  }
}

// PDF of the buoyancy with its background gradient (compute_BPE): weights
// dyf(j) over the planes jstart_th..jend_th, into nbin bins; constant bins
// over +-1.1 dTHdX Lx/2 with homogeneousX, else cos-spaced over +-Ro_inv
// With fbin, also the dyf-weighted sum of a field per bin
// (Bin_Ystar_and_Write, diagnostics.f90:1859-1950): kind 0 the field f0,
// kind 1 the kinetic energy 0.5 (f0^2 + f1^2 + f2^2) of the physical u1, u2,
// u3 at each point.
__global__ void __launch_bounds__(256) k_bpe_pdf(const double* th, Geom g, Phys ph, int homx, int nbin, double* pdf,
                                                 double* fbin, int kind, const double* f0, const double* f1,
                                                 const double* f2) {
  extern __shared__ double hist[];
  double* hf = hist + nbin;
  for (int b = threadIdx.x; b < nbin; b += blockDim.x) {
    hist[b] = 0.0;
    if (fbin) hf[b] = 0.0;
  }
  __syncthreads();
  const int j = g.jstart_th + blockIdx.y;
  const double dyfj = g.dyf[j];
  const double thmin = homx ? -ph.dthdx * 0.5 * ph.lx * 1.1 : -ph.ro_inv;
  const double thmax = homx ? ph.dthdx * 0.5 * ph.lx * 1.1 : ph.ro_inv;
  const double dth = (thmax - thmin) / nbin + 1.e-14;
  const double pi = ph.pi_ref;   // the reference's pi (for/fft.f90:147)
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.pp; p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % g.nx);
    const double gx = x * (ph.lx / g.nx);
    const double b = th[(long long)j * g.pp + p] + ph.dthdx * (gx - 0.5 * ph.lx);
    int bin;
    if (homx) {
      bin = min((int)((b - thmin) / dth), nbin - 1);
    } else {
      const double c = -fmin(fmax(b, thmin), thmax) / (ph.ro_inv + 1.e-14);
      bin = min((int)(acos(c) * nbin / pi), nbin - 1);
    }
    if (bin >= 0) {
      atomicAdd(&hist[bin], dyfj);
      if (fbin) {
        const long long q = (long long)j * g.pp + p;
        const double v = kind == 1 ? 0.5 * (f0[q] * f0[q] + f1[q] * f1[q] + f2[q] * f2[q]) : f0[q];
        atomicAdd(&hf[bin], v * dyfj);
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbin; b += blockDim.x) {
    if (hist[b] != 0.0) atomicAdd(&pdf[b], hist[b]);
    if (fbin && hf[b] != 0.0) atomicAdd(&fbin[b], hf[b]);
  }
}

// The LES statistics: the plane means of nu_t and kappa_t that les_chan and
// les_chan_th write under flag_save_LES (for/les.f90:909-935, 1404-1430),
// and compute_TKE_diss_les's eps_sgs2 (for/diagnostics.f90:2057-2118), the
// implicitly stepped part of the SGS dissipation: at GY row j (2..Nyp) the
// u1, u3 terms u_i d/dy(nu_t du_i/dy), formed at the GYF rows j and j - 1
// and averaged onto GY, plus the u2 term at GY with nu_t averaged onto GYF.
// FP64 physical u1, u2, u3 (phys.p[0..2]); nu_t, kappa_t at the context's
// precision R.  One CTA per plane, FP64 sums; out[3][np], zero where a row
// is not defined.
template <typename R>
__global__ void __launch_bounds__(256) k_les_stats(const __grid_constant__ State s, Geom g,
                                                   const __grid_constant__ FieldSet phys, double* out) {
  const int j = blockIdx.x, np = g.np, Nyp = g.ny;
  const long long pp = g.pp;   // Nx * Nz points per plane
  const R* nut = (const R*)s.nu_t;
  const R* kat = (const R*)s.kappa_t;
  const double* U1 = (const double*)phys.p[0];
  const double* U2 = (const double*)phys.p[1];
  const double* U3 = (const double*)phys.p[2];
  const bool eps = (j >= 2 && j <= Nyp);
  // s1 of compute_TKE_diss_les at GYF row jj (1..Nyp), point c of the plane
  auto s1 = [&](int jj, long long c) -> double {
    const long long o = (long long)jj * pp + c;
    const double n0 = (double)nut[o], n1 = (double)nut[o + pp];
    const double dyp = g.dy[jj + 1], dy0 = g.dy[jj], dyfj = g.dyf[jj];
    const double t1 = (n1 * (U1[o + pp] - U1[o]) / dyp - n0 * (U1[o] - U1[o - pp]) / dy0) / dyfj;
    const double t3 = (n1 * (U3[o + pp] - U3[o]) / dyp - n0 * (U3[o] - U3[o - pp]) / dy0) / dyfj;
    return U1[o] * t1 + U3[o] * t3;
  };
  double acc[3] = {0.0, 0.0, 0.0};
  for (long long c = threadIdx.x; c < pp; c += blockDim.x) {
    const long long o = (long long)j * pp + c;
    acc[0] += (double)nut[o];
    acc[1] += (double)kat[o];
    if (eps) {
      const double nj = (double)nut[o], njp = (double)nut[o + pp], njm = (double)nut[o - pp];
      const double t2 = (0.5 * (nj + njp) * (U2[o + pp] - U2[o]) / g.dyf[j] -
                         0.5 * (nj + njm) * (U2[o] - U2[o - pp]) / g.dyf[j - 1]) / g.dy[j];
      acc[2] += 0.5 * (s1(j, c) + s1(j - 1, c)) + U2[o] * t2;
    }
  }
  __shared__ double red[8][3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k][threadIdx.x];
    out[(long long)threadIdx.x * np + j] = (threadIdx.x < 2 || eps) ? v / (double)pp : 0.0;
  }
}

cudaError_t launch_les_stats(const Geom& g, const State& s, FieldSet phys, double* out, cudaStream_t st) {
  if (!s.nu_t || !s.kappa_t) return cudaErrorInvalidValue;
  if (g.prec) k_les_stats<float><<<g.np, 256, 0, st>>>(s, g, phys, out);
  else k_les_stats<double><<<g.np, 256, 0, st>>>(s, g, phys, out);
  return cudaGetLastError();
}

cudaError_t launch_budget(const Geom& g, const Phys& ph, const State& s, FieldSet phys, int homx, double* mxy,
                          double* out, cudaStream_t st) {
  k_zmeans<<<g.np, 256, 0, st>>>(s, g, phys, homx, mxy);
  k_budget<<<g.np, 256, 0, st>>>(s, g, ph, phys, homx, mxy, out);
  k_vorticity<<<g.np, 256, 0, st>>>(s, g, ph, out);
  return cudaGetLastError();
}

cudaError_t launch_bpe_pdf(const Geom& g, const Phys& ph, const double* th, int homx, int nbin, double* pdf,
                           cudaStream_t st, double* fbin, int kind, const double* f0, const double* f1,
                           const double* f2) {
  const int nj = g.jend_th - g.jstart_th + 1;
  if (nj < 1 || nbin < 1) return cudaErrorInvalidValue;
  const size_t smem = (size_t)nbin * sizeof(double) * (fbin ? 2 : 1);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_bpe_pdf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_bpe_pdf<<<dim3(8, nj), 256, smem, st>>>(th, g, ph, homx, nbin, pdf, fbin, kind, f0, f1, f2);
  return cudaGetLastError();
}

}  // namespace db
