// k_sgs_data.cu -- training data of the learned SGS closure from a resolved
// (DNS) state: a box filter of fx x fy x fz fine cells around every point of
// the coarse (LES) grid's GY rows, the exact subgrid stress and flux of that
// filter, and eddy coefficients fitted to them by least squares.
//
// Coarse grid: every fx-th x point, every fz-th z point, and in y the
// coarse grid of the same stretching with (NY - 1) / fy cells between its
// walls; its GY face k lies next to fine face J = fy (k - 1) (within a
// fraction of a fine cell for the create_grid.m stretchings).  The box
// around coarse face k spans fine cells J - fy/2 .. J + fy/2 - 1 in y and
// fx x fz points in x, z, weighted by the cell heights dyf (a volume
// average; the x, z spacing is uniform).
// Fields are taken at fine cell centres (u2 averaged from its two faces).
//   ubar_i, thbar, tau_ij = bar(u_i u_j) - ubar_i ubar_j,
//   q_i = bar(u_i th) - ubar_i thbar, Gbar_ij = bar(du_i/dx_j), gbar = bar(grad th)
//   S = sym(Gbar), tau^d = tau - tr(tau)/3 I
//   nu_t = max(0, -tau^d : S / (2 S : S)),  kappa_t = max(0, -q . gbar / |gbar|^2)
// Features (closure order): Gbar (i-major), gbar, 3 dx_c, 2 dy_c(k), 3 dz_c,
// gbar_y.  Output rows: coarse faces k = 3 .. NYc - 1, where the closure's
// nu_t is not the wall value 0 (ghost_les_mpi, for/les.f90:2229-2244).
#include "db_kernels.cuh"

namespace db {

struct SgsData {
  int fx, fy, fz;         // filter (coarsening) factors
  int nxc, nzc, nyc;      // coarse sizes (code NY of the coarse grid: nyc)
  int kmin, kmax;         // coarse GY faces written (3 .. nyc - 1)
  double dxc3, dzc3;      // 3 dx_c, 3 dz_c
  const double* dyc2;     // 2 dy_c(k), k = 0 .. nyc+1
  float* feat;            // [points][16]
  float* target;          // [points][2]
};

template <typename R>
__global__ void __launch_bounds__(128) k_sgs_targets(const __grid_constant__ State s, Geom g, SgsData d) {
  const int xc = blockIdx.x * blockDim.x + threadIdx.x;
  const int zc = blockIdx.y;
  const int k = d.kmin + blockIdx.z;
  if (xc >= d.nxc || k > d.kmax) return;
  const long long pp = g.pp;
  const R* U1 = (const R*)s.u1;
  const R* U2 = (const R*)s.u2;
  const R* U3 = (const R*)s.u3;
  const R* TH = (const R*)s.th;
  const R* GX[4] = {(const R*)s.gx[0], (const R*)s.gx[1], (const R*)s.gx[2], (const R*)s.gx[3]};
  const R* GZ[4] = {(const R*)s.gz[0], (const R*)s.gz[1], (const R*)s.gz[2], (const R*)s.gz[3]};
  const int J = d.fy * (k - 1);
  double W = 0, su[3] = {0, 0, 0}, sth = 0, suu[6] = {0, 0, 0, 0, 0, 0}, sut[3] = {0, 0, 0};
  double sG[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, sg[3] = {0, 0, 0};
  for (int jc = J - d.fy / 2; jc <= J + d.fy / 2 - 1; ++jc) {
    const double w = g.dyf[jc];
    const double iyc = 1.0 / (g.gyf[jc + 1] - g.gyf[jc - 1]);
    const double idf = 1.0 / g.dyf[jc];
    for (int dz = 0; dz < d.fz; ++dz) {
      const int z = zc * d.fz + dz;
      for (int dx = 0; dx < d.fx; ++dx) {
        const int x = xc * d.fx + dx;
        const long long c = (long long)jc * pp + (long long)z * g.nx + x;
        const double u1 = U1[c], u3 = U3[c], th = TH[c];
        const double u2 = 0.5 * ((double)U2[c] + (double)U2[c + pp]);
        double G[9], gt[3];
        G[0] = GX[0][c];
        G[1] = ((double)U1[c + pp] - (double)U1[c - pp]) * iyc;
        G[2] = GZ[0][c];
        G[3] = 0.5 * ((double)GX[1][c] + (double)GX[1][c + pp]);
        G[4] = ((double)U2[c + pp] - (double)U2[c]) * idf;
        G[5] = 0.5 * ((double)GZ[1][c] + (double)GZ[1][c + pp]);
        G[6] = GX[2][c];
        G[7] = ((double)U3[c + pp] - (double)U3[c - pp]) * iyc;
        G[8] = GZ[2][c];
        gt[0] = GX[3][c];
        gt[1] = ((double)TH[c + pp] - (double)TH[c - pp]) * iyc;
        gt[2] = GZ[3][c];
        W += w;
        su[0] += w * u1; su[1] += w * u2; su[2] += w * u3; sth += w * th;
        suu[0] += w * u1 * u1; suu[1] += w * u2 * u2; suu[2] += w * u3 * u3;
        suu[3] += w * u1 * u2; suu[4] += w * u1 * u3; suu[5] += w * u2 * u3;
        sut[0] += w * u1 * th; sut[1] += w * u2 * th; sut[2] += w * u3 * th;
#pragma unroll
        for (int i = 0; i < 9; ++i) sG[i] += w * G[i];
#pragma unroll
        for (int i = 0; i < 3; ++i) sg[i] += w * gt[i];
      }
    }
  }
  const double iW = 1.0 / W;
  double ub[3], tb = sth * iW, Gb[9], gb[3];
  for (int i = 0; i < 3; ++i) ub[i] = su[i] * iW;
  for (int i = 0; i < 9; ++i) Gb[i] = sG[i] * iW;
  for (int i = 0; i < 3; ++i) gb[i] = sg[i] * iW;
  // tau (11 22 33 12 13 23), deviatoric part, q
  double t11 = suu[0] * iW - ub[0] * ub[0], t22 = suu[1] * iW - ub[1] * ub[1], t33 = suu[2] * iW - ub[2] * ub[2];
  const double t12 = suu[3] * iW - ub[0] * ub[1], t13 = suu[4] * iW - ub[0] * ub[2], t23 = suu[5] * iW - ub[1] * ub[2];
  const double tr = (t11 + t22 + t33) / 3.0;
  t11 -= tr; t22 -= tr; t33 -= tr;
  const double q1 = sut[0] * iW - ub[0] * tb, q2 = sut[1] * iW - ub[1] * tb, q3 = sut[2] * iW - ub[2] * tb;
  const double S11 = Gb[0], S22 = Gb[4], S33 = Gb[8];
  const double S12 = 0.5 * (Gb[1] + Gb[3]), S13 = 0.5 * (Gb[2] + Gb[6]), S23 = 0.5 * (Gb[5] + Gb[7]);
  const double SS = S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
  const double TS = t11 * S11 + t22 * S22 + t33 * S33 + 2.0 * (t12 * S12 + t13 * S13 + t23 * S23);
  const double gg = gb[0] * gb[0] + gb[1] * gb[1] + gb[2] * gb[2];
  const double qg = q1 * gb[0] + q2 * gb[1] + q3 * gb[2];
  const double nu = SS > 0.0 ? fmax(0.0, -TS / (2.0 * SS)) : 0.0;
  const double ka = gg > 0.0 ? fmax(0.0, -qg / gg) : 0.0;
  const long long pt = ((long long)(k - d.kmin) * d.nzc + zc) * d.nxc + xc;
  float* f = d.feat + pt * 16;
  for (int i = 0; i < 9; ++i) f[i] = (float)Gb[i];
  f[9] = (float)gb[0]; f[10] = (float)gb[1]; f[11] = (float)gb[2];
  f[12] = (float)d.dxc3; f[13] = (float)d.dyc2[k]; f[14] = (float)d.dzc3; f[15] = (float)gb[1];
  d.target[pt * 2] = (float)nu;
  d.target[pt * 2 + 1] = (float)ka;
}

cudaError_t launch_sgs_targets(const Geom& g, const State& s, const SgsData& d, cudaStream_t st) {
  const int bx = d.nxc < 128 ? d.nxc : 128;
  const dim3 grid((d.nxc + bx - 1) / bx, d.nzc, d.kmax - d.kmin + 1);
  if (g.prec) k_sgs_targets<float><<<grid, bx, 0, st>>>(s, g, d);
  else k_sgs_targets<double><<<grid, bx, 0, st>>>(s, g, d);
  return cudaGetLastError();
}

}  // namespace db
