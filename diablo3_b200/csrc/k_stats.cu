// k_stats.cu -- the mean / energy-budget profiles of save_stats_chan
// (for/diagnostics.f90:3-480, compute_TKE 1270-1330, compute_TKE_diss
// 804-1020, TKE production 1385-1425), in FP64 from the FP64 spectral
// state on both precision paths.
//
// Every statistic is a horizontal average of a product of two fields at
// one plane, so by Parseval it is a sum over the retained Fourier modes:
//   <f g>_xz = sum_modes w Re(f^ conj(g^)),  w = 1 (kx = 0), 2 (kx > 0),
// the half-spectrum storage holding each kx > 0 mode for its conjugate
// too.  Fluctuations are the modes outside the averaging set: without the
// (0,0) mode for an x-homogeneous flow, without every kz = 0 mode when the
// reference averages over z only (fronts, IC_Type 5..8: homogeneousX false,
// for/parameters.f90:282-286).  One CTA per plane j.
#include "db_kernels.cuh"

namespace db {

// rows of the output, [stat][Nyp+2]
enum StatRow {
  ST_UME, ST_VME, ST_WME, ST_THME,   // means (u1, u3, th at GYF; u2 at GY)
  ST_UU, ST_VV, ST_WW, ST_TT,        // fluctuation variances (vv at GY)
  ST_UV, ST_WV,                      // <u1'u2'>, <u3'u2'> at GY (j >= 2), u interpolated with dyf weights
  ST_UW,                             // <u1'u3'> at GYF
  ST_THV,                            // <th' (u2'(j) + u2'(j+1))/2> at GYF
  ST_EPS,                            // sum of the 9 squared fluctuation gradients at GY (j = 2..Nyp), not times nu
  ST_GTH,                            // <|grad th|^2> at GYF without the background gradient
  NSTAT
};

__device__ __forceinline__ double mag2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double redot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

__global__ void __launch_bounds__(256) k_stats(const __grid_constant__ State s, Geom g, int homx, double* out) {
  const int j = blockIdx.x, np = g.np, Nyp = g.ny;
  const long long sp = g.sp;
  const int nk = g.nkx + 1, nmodes = g.nkzp * nk;
  double acc[NSTAT];
#pragma unroll
  for (int q = 0; q < NSTAT; ++q) acc[q] = 0.0;
  const double2 Z = make_double2(0.0, 0.0);
  const bool gy_ok = (j >= 2 && j <= Nyp);      // GY rows with both neighbours
  const bool gyf_ok = (j >= 1 && j <= Nyp);
  const double idy = gy_ok ? 1.0 / g.dy[j] : 0.0;
  const double wlo = gy_ok ? g.dyf[j - 1] / (2.0 * g.dy[j]) : 0.0;   // weight of row j
  const double whi = gy_ok ? g.dyf[j] / (2.0 * g.dy[j]) : 0.0;       // weight of row j - 1
  const double i2gy = gy_ok ? 1.0 / (g.gy[j + 1] - g.gy[j - 1]) : 0.0;
  const double i2gyf = gyf_ok ? 1.0 / (g.gyf[j + 1] - g.gyf[j - 1]) : 0.0;
  for (int m = threadIdx.x; m < nmodes; m += blockDim.x) {
    const int kzp = m / nk, kx = m % nk;
    const long long a = (long long)j * sp + (long long)kzp * g.kxs + kx;
    const double w = kx == 0 ? 1.0 : 2.0;
    const bool fluct = homx ? !(kx == 0 && kzp == 0) : (kzp != 0);
    const double kx2 = g.kx[kx] * g.kx[kx], kz2 = g.kz[kzp] * g.kz[kzp];
    const double2 u1 = s.cu1[a], u2 = s.cu2[a], u3 = s.cu3[a], th = s.cth[a];
    const double2 u1m = j >= 1 ? s.cu1[a - sp] : Z, u3m = j >= 1 ? s.cu3[a - sp] : Z;
    const double2 u2m = j >= 1 ? s.cu2[a - sp] : Z, u2p = j + 1 < np ? s.cu2[a + sp] : Z;
    const double2 thm = j >= 1 ? s.cth[a - sp] : Z, thp = j + 1 < np ? s.cth[a + sp] : Z;
    if (kx == 0 && kzp == 0) {
      acc[ST_UME] = u1.x; acc[ST_VME] = u2.x; acc[ST_WME] = u3.x; acc[ST_THME] = th.x;
    }
    if (gyf_ok) {   // |grad th|^2 over every mode (the mean gradient included)
      const double2 dth = make_double2((thp.x - thm.x) * i2gyf, (thp.y - thm.y) * i2gyf);
      acc[ST_GTH] += w * ((kx2 + kz2) * mag2(th) + mag2(dth));
    }
    if (!fluct) continue;
    acc[ST_UU] += w * mag2(u1);
    acc[ST_VV] += w * mag2(u2);
    acc[ST_WW] += w * mag2(u3);
    acc[ST_TT] += w * mag2(th);
    acc[ST_UW] += w * redot(u1, u3);
    if (gyf_ok) {
      const double2 vf = make_double2(0.5 * (u2.x + u2p.x), 0.5 * (u2.y + u2p.y));
      acc[ST_THV] += w * redot(th, vf);
    }
    if (gy_ok) {
      const double2 u1g = make_double2(wlo * u1.x + whi * u1m.x, wlo * u1.y + whi * u1m.y);
      const double2 u3g = make_double2(wlo * u3.x + whi * u3m.x, wlo * u3.y + whi * u3m.y);
      acc[ST_UV] += w * redot(u1g, u2);
      acc[ST_WV] += w * redot(u3g, u2);
      // x and z derivatives (GYF rows interpolated to GY as squares), then
      // the y-differences of the fluctuations (compute_TKE_diss)
      const double s1 = wlo * mag2(u1) + whi * mag2(u1m), s3 = wlo * mag2(u3) + whi * mag2(u3m);
      double e = (kx2 + kz2) * (s1 + s3 + mag2(u2));
      const double2 d1 = make_double2((u1.x - u1m.x) * idy, (u1.y - u1m.y) * idy);
      const double2 d3 = make_double2((u3.x - u3m.x) * idy, (u3.y - u3m.y) * idy);
      const double2 d2 = make_double2((u2p.x - u2m.x) * i2gy, (u2p.y - u2m.y) * i2gy);
      e += mag2(d1) + mag2(d3) + mag2(d2);
      acc[ST_EPS] += w * e;
    }
  }
  // CTA reduction (the mean rows come from the one thread that owns mode (0,0))
  __shared__ double red[8][NSTAT];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NSTAT; ++q) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < NSTAT) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k][threadIdx.x];
    out[(long long)threadIdx.x * np + j] = v;
  }
}

cudaError_t launch_stats(const Geom& g, const State& s, int homx, double* out, cudaStream_t st) {
  k_stats<<<g.np, 256, 0, st>>>(s, g, homx, out);
  return cudaGetLastError();
}

}  // namespace db
