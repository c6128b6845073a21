// les_feat.cuh -- the 16 input features of the learned SGS closure at one
// point of a GY row (include/diablo_b200.h gives the order), shared by the
// column-walking LES kernel (k_les.cu: feature output and the training-range
// check) and the fused feature + inference kernel (k_mlp.cu), so that every
// path sees bit-identical features.  The two-point interpolations from the
// GYF rows j - 1, j to GY row j are written as explicit fma so the rounding
// does not depend on how the compiler contracts each call site.
#pragma once

#include "db_kernels.cuh"
#include "mlp.cuh"

namespace db {

constexpr double BETA_SGS = 3.0;   // filter width / grid spacing (les.f90:43)

// velocity/scalar gradient values a GY row's features need: x and z
// derivatives at the GYF rows j (a*) and j - 1 (f*), the y-differences at GY
// row j (d*y) and du2/dy at the GYF rows j (c2y) and j - 1 (f2y)
template <typename R>
struct LesFeatIn {
  R a1x, f1x, a1z, f1z, a2x, a2z, a3x, f3x, a3z, f3z, atx, ftx, atz, ftz;
  R d1y, d3y, dty, c2y, f2y;
};

// GYF(j-1), GYF(j) -> GY(j) with weights wa (row j), wb (row j - 1)
template <typename R>
__device__ __forceinline__ R gy_interp(R aj, R fjm, R wa, R wb) {
  return fma(aj, wa, fjm * wb);
}

// dxs, dzs: the x, z filter widths; dly: the GY row's y filter width
template <typename R>
__device__ __forceinline__ void les_features(const LesFeatIn<R>& v, R wa, R wb, R dxs, R dly, R dzs, float* fv) {
  fv[0] = (float)gy_interp(v.a1x, v.f1x, wa, wb);
  fv[1] = (float)v.d1y;
  fv[2] = (float)gy_interp(v.a1z, v.f1z, wa, wb);
  fv[3] = (float)v.a2x;
  fv[4] = (float)gy_interp(v.c2y, v.f2y, wa, wb);
  fv[5] = (float)v.a2z;
  fv[6] = (float)gy_interp(v.a3x, v.f3x, wa, wb);
  fv[7] = (float)v.d3y;
  fv[8] = (float)gy_interp(v.a3z, v.f3z, wa, wb);
  fv[9] = (float)gy_interp(v.atx, v.ftx, wa, wb);
  fv[10] = (float)v.dty;
  fv[11] = (float)gy_interp(v.atz, v.ftz, wa, wb);
  fv[12] = (float)dxs;
  fv[13] = (float)dly;
  fv[14] = (float)dzs;
  fv[15] = (float)v.dty;
}

// Features of GY row j (1 <= j <= Nyp + 1) at column col read straight from
// the physical fields (point-parallel form of the column walk in k_les_amd):
// rows j - 1 and j of every field, u2 also at row j + 1 when j <= Nyp.
template <typename R>
__device__ __forceinline__ void les_features_at(const LesFeatSrc& s, int j, long long col, float* fv) {
  const long long o = (long long)j * s.pp + col, om = o - s.pp;
  const R* const* G = reinterpret_cast<const R* const*>(s.f);   // u1 u2 u3 th, d/dx x4, d/dz x4
  LesFeatIn<R> v;
  v.a1x = G[4][o]; v.f1x = G[4][om];
  v.a1z = G[8][o]; v.f1z = G[8][om];
  v.a2x = G[5][o]; v.a2z = G[9][o];
  v.a3x = G[6][o]; v.f3x = G[6][om];
  v.a3z = G[10][o]; v.f3z = G[10][om];
  v.atx = G[7][o]; v.ftx = G[7][om];
  v.atz = G[11][o]; v.ftz = G[11][om];
  const LesRow& lr = s.lrow[j];
  // ydiff: y-differences of fluctuations plus those of the plane means when
  // the fields hold fluctuations, formed as the column walk forms them
  const double* pm = s.mean;
  const int np = s.ny + 2;
  v.d1y = ydiff<R>(G[0][o], G[0][om], pm, 0, np, j, j - 1, lr.idy);
  v.d3y = ydiff<R>(G[2][o], G[2][om], pm, 2, np, j, j - 1, lr.idy);
  v.dty = ydiff<R>(G[3][o], G[3][om], pm, 3, np, j, j - 1, lr.idy);
  const R u2j = G[1][o];
  v.c2y = (j <= s.ny) ? ydiff<R>(G[1][o + s.pp], u2j, pm, 1, np, j + 1, j, lr.idyf) : (R)0;
  v.f2y = ydiff<R>(u2j, G[1][om], pm, 1, np, j, j - 1, s.lrow[j - 1].idyf);
  les_features<R>(v, (R)lr.wa, (R)lr.wb, (R)s.dxs, (R)lr.dys_y, (R)s.dzs, fv);
}

}  // namespace db
