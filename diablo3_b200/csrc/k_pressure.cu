// k_pressure.cu -- poisson_p_chan (for/solver.f90:1382-1590): the pressure
// cp from the velocity and the buoyancy, for a restart whose file holds no
// pressure (ReadHDF5 calls it, for/phdf5.f90:1452-1454).
//
//  k_pp_terms : the spectral factors of one term of (dui/dxj)(duj/dxi) at the
//               planes 2..Nyp (the reference's cf1, cf2 before their
//               transforms): term 0..2 the diagonal derivatives du1/dx,
//               du2/dy, du3/dz (squared in physical space), term 3..5 the
//               pairs (du1/dy, du2/dx), (du3/dy, du2/dz), (du1/dz, du3/dx)
//               (2 a b in physical space)
//  k_pp_accum : the physical product of a term added to the sum q
//  k_pp_solve : right-hand side -(Q + d th / dy) (the buoyancy term without
//               the (0,0) mode) and the complex Thomas per (kx, kz) with
//               apply_BC_poisson_mpi's rows (solver.f90:2375-2411); cp at
//               the planes 1..Nyp
// The transforms between are the library's FP64 passes.  The reference
// transforms each product back separately and adds the six in spectral
// space; here they are added in physical space and transformed once (the
// same sum, rounded differently).  FP64 on both precision paths.
#include <math.h>

#include "db_kernels.cuh"

namespace db {

__global__ void __launch_bounds__(256) k_pp_terms(const __grid_constant__ State s, Geom g, int term, double2* w1,
                                                  double2* w2) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (m >= g.nkzp * g.kxs) return;
  const int kzp = m / g.kxs, kx = m % g.kxs;
  const long long a = (long long)j * g.sp + m, sp = g.sp;
  const double2 Z = make_double2(0.0, 0.0);
  if (j < 2 || j > g.ny || kx > g.nkx) {
    w1[a] = Z;
    if (w2) w2[a] = Z;
    return;
  }
  const double kxv = g.kx[kx], kzv = g.kz[kzp];
  auto ik = [](double k, double2 c) { return make_double2(-k * c.y, k * c.x); };
  auto dyc = [&](const double2* f) {   // (f(j+1) - f(j-1)) / (2 dyf(j))
    const double w = 1.0 / (2.0 * g.dyf[j]);
    return make_double2((f[a + sp].x - f[a - sp].x) * w, (f[a + sp].y - f[a - sp].y) * w);
  };
  const double2 v = make_double2(0.5 * (s.cu2[a].x + s.cu2[a + sp].x), 0.5 * (s.cu2[a].y + s.cu2[a + sp].y));
  switch (term) {
    case 0: w1[a] = ik(kxv, s.cu1[a]); break;
    case 1: {
      const double w = 1.0 / g.dyf[j];
      w1[a] = make_double2((s.cu2[a + sp].x - s.cu2[a].x) * w, (s.cu2[a + sp].y - s.cu2[a].y) * w);
      break;
    }
    case 2: w1[a] = ik(kzv, s.cu3[a]); break;
    case 3: w1[a] = dyc(s.cu1); w2[a] = ik(kxv, v); break;
    case 4: w1[a] = dyc(s.cu3); w2[a] = ik(kzv, v); break;
    default: w1[a] = ik(kzv, s.cu1[a]); w2[a] = ik(kxv, s.cu3[a]); break;
  }
}

__global__ void __launch_bounds__(256) k_pp_accum(Geom g, const double* p1, const double* p2, int square,
                                                  double* q) {
  const long long n = (long long)g.np * g.pp;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(i / g.pp);
    if (j < 2 || j > g.ny) continue;
    q[i] += square ? p1[i] * p1[i] : 2.0 * p1[i] * p2[i];
  }
}

// one thread per (kx, kzp); gsc, bsc: the forward sweep's g_j and b'_j
__global__ void __launch_bounds__(128) k_pp_solve(const __grid_constant__ State s, Geom g, const double2* rhs,
                                                  double2* gsc, double* bsc) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  if (kx > g.nkx) return;
  const int Nyp = g.ny;
  const long long c0 = (long long)kzp * g.kxs + kx, sp = g.sp;
  const double kx2 = g.kx[kx] * g.kx[kx], kz2 = g.kz[kzp] * g.kz[kzp];
  const bool m0 = (kx == 0 && kzp == 0);
  // rows 1..Nyp: row 1 and row Nyp from apply_BC_poisson_mpi; the upper
  // coefficient of row Nyp keeps its interior value but couples to no row
  auto row = [&](int j, double& l, double& d, double& u, double2& v) {
    l = 1. / (g.dy[j] * g.dyf[j]);
    d = -kx2 - kz2 - 1. / (g.dy[j + 1] * g.dyf[j]) - 1. / (g.dy[j] * g.dyf[j]);
    u = 1. / (g.dy[j + 1] * g.dyf[j]);
    const long long a = (long long)j * sp + c0;
    double2 r = rhs[a];
    if (!m0) {   // buoyancy: d th / dy at GYF, centred
      const double w = 1.0 / (g.gyf[j + 1] - g.gyf[j - 1]);
      r.x += (s.cth[a + sp].x - s.cth[a - sp].x) * w;
      r.y += (s.cth[a + sp].y - s.cth[a - sp].y) * w;
    }
    v = make_double2(-r.x, -r.y);
    if (j == 1) { l = 0.; d = 1.; u = m0 ? 0. : -1.; v = make_double2(0., 0.); }
    if (j == Nyp) { l = 1.; d = -1.; v = make_double2(0., 0.); }
  };
  double l, d, u, uprev = 0.0, bprev = 1.0;
  double2 v, gp = make_double2(0.0, 0.0);
  for (int j = 1; j <= Nyp; ++j) {
    row(j, l, d, u, v);
    double b = d;
    if (j > 1) {
      const double a = -l / bprev;
      b = d + a * uprev;
      v = make_double2(v.x + a * gp.x, v.y + a * gp.y);
    }
    gsc[(long long)j * sp + c0] = v;
    bsc[(long long)j * sp + c0] = b;
    gp = v;
    bprev = b;
    uprev = u;
  }
  double2 x = make_double2(0.0, 0.0);
  for (int j = Nyp; j >= 1; --j) {
    const long long a = (long long)j * sp + c0;
    const double2 gj = gsc[a];
    const double b = bsc[a];
    double uj = 0.0;
    if (j < Nyp) {
      double lj, dj;
      double2 vj;
      row(j, lj, dj, uj, vj);
    }
    x = make_double2((gj.x - uj * x.x) / b, (gj.y - uj * x.y) / b);
    s.cp[a] = x;
  }
}

cudaError_t launch_pp_terms(const Geom& g, const State& s, int term, double2* w1, double2* w2, cudaStream_t st) {
  k_pp_terms<<<dim3((g.nkzp * g.kxs + 255) / 256, g.np), 256, 0, st>>>(s, g, term, w1, w2);
  return cudaGetLastError();
}
cudaError_t launch_pp_accum(const Geom& g, const double* p1, const double* p2, int square, double* q,
                            cudaStream_t st) {
  k_pp_accum<<<4 * sm_count(), 256, 0, st>>>(g, p1, p2, square, q);
  return cudaGetLastError();
}
cudaError_t launch_pp_solve(const Geom& g, const State& s, const double2* rhs, double2* gsc, double* bsc,
                            cudaStream_t st) {
  k_pp_solve<<<dim3((g.nkx + 1 + 127) / 128, g.nkzp), 128, 0, st>>>(s, g, rhs, gsc, bsc);
  return cudaGetLastError();
}

}  // namespace db
