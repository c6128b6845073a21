// db_bc.cuh -- boundary conditions on the spectral ghost rows, one
// (kx, kzp) column at a time.  A column's rows 0, 1, 2, Nyp-1, Nyp, Nyp+1
// are held in a GhostCol; the BC routines only ever write rows 0, 1, Nyp
// and Nyp+1.
#pragma once

#include "db_kernels.cuh"
#include "cplx_dft.cuh"

namespace db {

enum { G_0 = 0, G_1, G_2, G_M, G_N, G_N1 };   // rows 0, 1, 2, Nyp-1, Nyp, Nyp+1

struct GhostCol {
  double2 v[6];
};

__device__ __forceinline__ long long ghost_row(int q, int Nyp) {
  return q <= G_2 ? q : (long long)(Nyp - 1 + (q - G_M));
}

__device__ __forceinline__ void load_col(GhostCol& c, const double2* col, long long sp, int Nyp) {
#pragma unroll
  for (int q = 0; q < 6; ++q) c.v[q] = col[ghost_row(q, Nyp) * sp];
}

// write rows 0, 1, Nyp, Nyp+1 back into a state column
__device__ __forceinline__ void store_ghosts(const GhostCol& c, double2* col, long long sp, int Nyp) {
  col[0] = c.v[G_0];
  col[sp] = c.v[G_1];
  col[(long long)Nyp * sp] = c.v[G_N];
  col[(long long)(Nyp + 1) * sp] = c.v[G_N1];
}

// apply_BC_vel_mpi_post on one column of the velocity (flow.f90:1161-1360);
// m0: the (0, 0) mode; time: the clock the f_type 4 wall forcing reads
__device__ __forceinline__ void bc_vel_post(GhostCol& u1, GhostCol& u2, GhostCol& u3, const Geom& g, const Phys& ph,
                                            bool m0, double time) {
  const int Nyp = g.ny;
  const double2 Z = make_double2(0.0, 0.0);
  auto R = [](double v) { return make_double2(v, 0.0); };
  // lower
  if (ph.bc_type[BC_U_MIN] == 0) {
    u1.v[G_0] = Z; u1.v[G_1] = Z;
    if (m0) { u1.v[G_1] = R(ph.bc_c1[BC_U_MIN]); u1.v[G_0] = R(ph.bc_c1[BC_U_MIN]); }
  } else {
    u1.v[G_1] = u1.v[G_2]; u1.v[G_0] = u1.v[G_1];
    if (m0) {
      u1.v[G_1] = csub(u1.v[G_2], R(g.dy[2] * ph.bc_c1[BC_U_MIN]));
      u1.v[G_0] = csub(u1.v[G_1], R(g.dy[1] * ph.bc_c1[BC_U_MIN]));
    }
  }
  if (ph.bc_type[BC_W_MIN] == 0) {
    u3.v[G_0] = Z; u3.v[G_1] = Z;
    if (m0) { u3.v[G_1] = R(ph.bc_c1[BC_W_MIN]); u3.v[G_0] = R(ph.bc_c1[BC_W_MIN]); }
  } else {
    u3.v[G_1] = u3.v[G_2]; u3.v[G_0] = u3.v[G_1];
    if (m0) {
      u3.v[G_1] = csub(u3.v[G_2], R(g.dy[2] * ph.bc_c1[BC_W_MIN]));
      u3.v[G_0] = csub(u3.v[G_1], R(g.dy[1] * ph.bc_c1[BC_W_MIN]));
    }
  }
  if (ph.bc_type[BC_V_MIN] == 0) {
    u2.v[G_1] = csub(R(2.0 * ph.bc_c1[BC_V_MIN]), u2.v[G_2]);
    u2.v[G_0] = u2.v[G_1];
  } else {
    u2.v[G_1] = u2.v[G_2]; u2.v[G_0] = u2.v[G_1];
    if (m0) {
      u2.v[G_1] = csub(u2.v[G_2], R(g.dyf[1] * ph.bc_c1[BC_V_MIN]));
      u2.v[G_0] = csub(u2.v[G_1], R(g.dyf[1] * ph.bc_c1[BC_V_MIN]));
    }
  }
  // upper
  if (ph.bc_type[BC_U_MAX] == 0) {
    u1.v[G_N] = Z; u1.v[G_N1] = Z;
    if (m0) { u1.v[G_N] = R(ph.bc_c1[BC_U_MAX]); u1.v[G_N1] = R(ph.bc_c1[BC_U_MAX]); }
  } else {
    u1.v[G_N] = u1.v[G_M]; u1.v[G_N1] = u1.v[G_N];
    if (m0) {
      u1.v[G_N] = cadd(u1.v[G_M], R(g.dy[Nyp] * ph.bc_c1[BC_U_MAX]));
      u1.v[G_N1] = cadd(u1.v[G_N], R(g.dy[Nyp] * ph.bc_c1[BC_U_MAX]));
    }
  }
  if (ph.bc_type[BC_W_MAX] == 0) {
    u3.v[G_N] = Z; u3.v[G_N1] = Z;
    if (m0) { u3.v[G_N] = R(ph.bc_c1[BC_W_MAX]); u3.v[G_N1] = Z; }
  } else {
    u3.v[G_N] = u3.v[G_M]; u3.v[G_N1] = u3.v[G_N];
    if (m0) {
      double wt = ph.bc_c1[BC_W_MAX];
      if (ph.f_type == 4)
        wt = ph.bc_c1[BC_W_MAX] + ph.amp_omega0 * sin(ph.omega0 * (ph.ro_inv / ph.delta * time - ph.force_start));
      u3.v[G_N] = cadd(u3.v[G_M], R(g.dy[Nyp] * wt));
      u3.v[G_N1] = cadd(u3.v[G_N], R(g.dy[Nyp] * wt));
    }
  }
  if (ph.bc_type[BC_V_MAX] == 0) {
    if (m0) u2.v[G_N1] = csub(R(2.0 * ph.bc_c1[BC_V_MAX]), u2.v[G_N]);
  } else {
    u2.v[G_N] = u2.v[G_M]; u2.v[G_N1] = u2.v[G_N];
    if (m0) u2.v[G_N1] = cadd(u2.v[G_N], R(g.dy[Nyp] * ph.bc_c1[BC_V_MAX]));
  }
}

// apply_BC_th_mpi_post on one column of the scalar (flow.f90:1596-1689)
__device__ __forceinline__ void bc_th_post(GhostCol& th, const Geom& g, const Phys& ph, bool m0) {
  const int Nyp = g.ny;
  const double2 Z = make_double2(0.0, 0.0);
  auto R = [](double v) { return make_double2(v, 0.0); };
  if (ph.bc_type[BC_TH_MIN] == 0) {
    th.v[G_0] = Z; th.v[G_1] = Z;
    if (m0) { th.v[G_1] = R(ph.bc_c1[BC_TH_MIN]); th.v[G_0] = R(ph.bc_c1[BC_TH_MIN]); }
  } else {
    th.v[G_1] = th.v[G_2]; th.v[G_0] = th.v[G_1];
    if (m0) {
      th.v[G_1] = csub(th.v[G_2], R(g.dy[2] * ph.bc_c1[BC_TH_MIN]));
      th.v[G_0] = csub(th.v[G_1], R(g.dy[1] * ph.bc_c1[BC_TH_MIN]));
    }
  }
  if (ph.bc_type[BC_TH_MAX] == 0) {
    th.v[G_N] = Z; th.v[G_N1] = Z;
    if (m0) { th.v[G_N] = R(ph.bc_c1[BC_TH_MAX]); th.v[G_N1] = R(ph.bc_c1[BC_TH_MAX]); }
  } else {
    th.v[G_N] = th.v[G_M]; th.v[G_N1] = th.v[G_N];
    if (m0) {
      th.v[G_N] = cadd(th.v[G_M], R(g.dy[Nyp] * ph.bc_c1[BC_TH_MAX]));
      th.v[G_N1] = cadd(th.v[G_N], R(g.dy[Nyp] * ph.bc_c1[BC_TH_MAX]));
    }
  }
}

// apply_BC_les and apply_BC_th_les (les.f90:1980-2079): at Neumann walls
// both ghost rows take the first interior row, mean mode included
__device__ __forceinline__ void bc_les(GhostCol& u1, GhostCol& u3, GhostCol& th, const Phys& ph) {
  if (ph.bc_type[BC_U_MAX] == 1) { u1.v[G_N] = u1.v[G_M]; u1.v[G_N1] = u1.v[G_N]; }
  if (ph.bc_type[BC_W_MAX] == 1) { u3.v[G_N] = u3.v[G_M]; u3.v[G_N1] = u3.v[G_N]; }
  if (ph.bc_type[BC_U_MIN] == 1) { u1.v[G_1] = u1.v[G_2]; u1.v[G_0] = u1.v[G_1]; }
  if (ph.bc_type[BC_W_MIN] == 1) { u3.v[G_1] = u3.v[G_2]; u3.v[G_0] = u3.v[G_1]; }
  if (ph.bc_type[BC_TH_MAX] == 1) { th.v[G_N] = th.v[G_M]; th.v[G_N1] = th.v[G_N]; }
  if (ph.bc_type[BC_TH_MIN] == 1) { th.v[G_1] = th.v[G_2]; th.v[G_0] = th.v[G_1]; }
}

}  // namespace db
