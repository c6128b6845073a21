// k_les.cu -- LES closure of the channel substep, les_model_type 5:
// anisotropic minimum dissipation (AMD, Verstappen form) for momentum and
// scalar (for/les.f90:3-1068 model-5 branch, 1072-1435, 1443-1746).
//
// The reference builds 26 spectral tensor fields (Sij, SIij, Oij, all nine
// velocity gradients, three scalar gradients), transforms them all to
// physical space, forms the model there and transforms 9 stress/flux fields
// back.  Every one of those fields is a fixed linear combination of
//   u_i, th                      (needed by the substep anyway),
//   d/dx and d/dz of u_i and th  (8 fields),
//   y-differences of u_i, th     (formed pointwise in physical space),
// so here only the 8 x/z derivatives are transformed (as extra outputs of
// the state's inverse transforms, the derivative applied on the way), and
// the divergence of the model stress is folded into the nonlinear-product
// fields before their forward transform: the SGS terms cost no forward FFT.
//
//  k_les_bc     : apply_BC_vel_mpi_post, apply_BC_th_mpi_post, apply_BC_les,
//                 apply_BC_th_les on the spectral ghost rows (les.f90:63-75),
//                 into a side buffer the inverse transforms overlay.
//  k_les_amd    : one thread per (x, z) column walks j; from the gradients it
//                 forms the AMD coefficients at GYF and GY rows (les.f90:
//                 574-719, 1216-1310), nu_t and kappa_t (:783-795, :1347-1358,
//                 ghost_les_mpi with one rank), and the physical-space parts
//                 of the SGS forcing per product slot (:800-900, :1360-1391).
//  k_thomas_les : the CN solves with the eddy viscosity/diffusivity in the
//                 explicit term and the matrix (solver.f90:872-903, 988-1003,
//                 1028-1045, 1088-1105, 1144-1161, 1200-1217): the matrix
//                 differs per (x, z) column, so each thread runs its own
//                 Thomas sweep, with an FP64 scratch for the eliminated
//                 coefficients and batched row loads.
#include <math.h>

#include "../../include/diablo_b200.h"
#include "db_bc.cuh"
#include "db_kernels.cuh"
#include "les_feat.cuh"
#include "umma.cuh"

namespace db {

// ---------------------------------------------------------------------------
// Ghost rows the model sees (les.f90:63-75).  The reference rewrites the
// state's rows 0, 1, Nyp, Nyp+1 here, after the substep has already formed
// cr and cf from the unmodified state (solver.f90:396-609), and the rewrite
// reaches the rest of the substep only through the physical fields.  So the
// rewritten rows go to a side buffer ghost[f][q] (f = cu1, cu2, cu3, cth;
// q = rows 0, 1, Nyp, Nyp+1) that the inverse transforms read in place of
// the state's rows; the final forward transform of the physical fields
// carries them into the new state exactly as in the reference.
__global__ void k_les_bc(const __grid_constant__ State s, Geom g, Phys ph) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  if (kx >= g.kxs) return;
  const long long c0 = (long long)kzp * g.kxs + kx, sp = g.sp;
  const int Nyp = g.ny;
  GhostCol a, b, c, t;
  load_col(a, s.cu1 + c0, sp, Nyp);
  load_col(b, s.cu2 + c0, sp, Nyp);
  load_col(c, s.cu3 + c0, sp, Nyp);
  load_col(t, s.cth + c0, sp, Nyp);
  if (kx <= g.nkx) {
    const bool m0 = (kx == 0 && kzp == 0);
    bc_vel_post(a, b, c, g, ph, m0, s.sc->time);
    bc_th_post(t, g, ph, m0);
    bc_les(a, c, t, ph);
  }
  const GhostCol* f[4] = {&a, &b, &c, &t};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double2* o = s.ghost + (long long)(4 * i) * sp + c0;
    o[0] = f[i]->v[G_0];
    o[sp] = f[i]->v[G_1];
    o[2 * sp] = f[i]->v[G_N];
    o[3 * sp] = f[i]->v[G_N1];
  }
}

// ---------------------------------------------------------------------------
// AMD model

constexpr double C_AMD = 0.2887;     // les.f90:25

// max{0, -(I3 - I4)} / (I1 - I2) of the scaled strain SI and rotation O
// tensors (les.f90:578-619): -tr(SI^3) + tr(SI O^2) over |SI|^2 + |O|^2
template <typename R>
__device__ __forceinline__ R amd_ratio(R s1, R s2, R s3, R s4, R s5, R s6, R o4, R o5, R o6) {
  const R c2 = 2, c3 = 3, c6 = 6;
  const R i3 = s1 * s1 * s1 + s2 * s2 * s2 + s3 * s3 * s3 + c3 * s1 * s4 * s4 + c3 * s1 * s5 * s5 +
               c3 * s2 * s4 * s4 + c3 * s2 * s6 * s6 + c3 * s3 * s5 * s5 + c3 * s3 * s6 * s6 + c6 * s4 * s5 * s6;
  const R v = -i3 - s1 * o4 * o4 - s1 * o5 * o5 - s2 * o4 * o4 - s2 * o6 * o6 - s3 * o5 * o5 - s3 * o6 * o6 -
              c2 * s4 * o5 * o6 + c2 * s5 * o4 * o6 - c2 * s6 * o4 * o5;
  if (v <= (R)0) return (R)0;
  return v / (s1 * s1 + s2 * s2 + s3 * s3 + c2 * s4 * s4 + c2 * o4 * o4 + c2 * s5 * s5 + c2 * o5 * o5 +
              c2 * s6 * s6 + c2 * o6 * o6);
}

// scalar AMD: max{0, -(delta_k^2 du_i/dx_k dth/dx_k dth/dx_i)} / |delta dth|^2
// (les.f90:1222-1249, 1265-1305); arguments are the gradient components
// at one point, dys the y filter width there
template <typename R>
__device__ __forceinline__ R amd_th_ratio(R dxs, R dys, R dzs, R u1x, R u2y, R u3z, R u1y, R u2x, R u1z, R u3x,
                                          R u2z, R u3y, R tx, R ty, R tz) {
  const R v = -(dxs * dxs * u1x * tx * tx + dys * dys * u2y * ty * ty + dzs * dzs * u3z * tz * tz +
                (dys * dys * u1y + dxs * dxs * u2x) * tx * ty + (dzs * dzs * u1z + dxs * dxs * u3x) * tx * tz +
                (dzs * dzs * u2z + dys * dys * u3y) * ty * tz);
  if (v <= (R)0) return (R)0;
  return v / ((dxs * tx) * (dxs * tx) + (dys * ty) * (dys * ty) + (dzs * tz) * (dzs * tz));
}

// filter coefficient -2 C^2 Delta^2 at a row of spacing h (les.f90:756-780)
__device__ __forceinline__ double amd_delta(double dxs, double dzs, double h) {
  return -2.0 * C_AMD * C_AMD * 3.0 / (1.0 / (dxs * dxs) + 1.0 / ((h * 2.0) * (h * 2.0)) + 1.0 / (dzs * dzs));
}

// SGS forcing terms, zero outside the rows where the reference applies each:
//  L0 = dyf-filter * s1 S11            (u1 eq., times i kx)      rows j1..j2
//  L1 = Dy(delta_y tau_12)             (u1 eq., no derivative)   rows j1..j2
//  L2 = dyf-filter * s1 S13            (u1: i kz, u3: i kx)      rows j1..j2
//  L3 = Dy(delta_y tau_23)             (u3 eq., no derivative)   rows j1..j2
//  L4 = dyf-filter * s1 S33            (u3 eq., times i kz)      rows j1..j2
//  L5 = delta_y tau_12 - nu_t du1/dy   (u2 eq., times i kx)      rows 2..Nyp
//  L6 = delta_y tau_23 - nu_t du3/dy   (u2 eq., times i kz)      rows 2..Nyp
//  L7 = dyf-filter/2 * s1_th dth/dx    (th eq., times i kx)      rows jst..jet
//  L8 = dyf-filter/2 * s1_th dth/dz    (th eq., times i kz)      rows jst..jet
// with j1 = jstart, j2 = Nyp - 1 (les.f90:46-49, one rank), tau_12 at GY
// rows = temp (S12 - du1/dy / 2) for j >= 2 and the raw strain at j = 1
// (les.f90:737-748).  Each is added to the nonlinear product it shares a
// derivative with, and the kernel stores the 11 real sequences of every
// plane the LES products kernel transforms (physical [j][z][x], in the
// products' (group, sequence, part) order, stored on the rows where that
// kernel reads them; <.> the GY interpolation, Dy the conservative
// y-difference):
//  les[0] = u1 u1 + L0   les[1] = Dy(u1 u2) + L1   les[2] = u3 u1 + L2
//  les[3] = Dy(u3 u2) + L3   les[4] = u3 u3 + L4                          rows jstart..jend
//  les[5] = <u1> u2 + L5   les[6] = Dy(u2 u2)   les[9] = <u3> u2 + L6     rows 2..Nyp
//  les[7] = th u1 + L7   les[8] = Dy(th u2)   les[10] = th u3 + L8        rows jst..jet
// Plane r needs rows r - 1 .. r + 1, so it is formed with the GYF outputs of
// row r, one iteration after row r + 1 arrived.  R: arithmetic and storage
// type (FP32 on the mixed path).
// MODE 0: AMD.  MODE 1: only the learned closure's 16 features at every GY
// row (include/diablo_b200.h order) into s.sgs_feat[point][16].  MODE 2:
// the closure's nu_t, kappa_t (s.sgs_out[point][2], at GY rows) take the
// place of the AMD coefficients, temp = -2 nu / filter at GY rows and
// s1 = -2 nu_GYF / filter at GYF rows with nu_GYF the mean of the two GY
// neighbours; a point whose features leave the training range
// (s.sgs_range: lo[16], hi[16]) keeps its AMD value.
//
// The walk over j = 1 .. Nyp + 1 is split into gridDim.z chunks run by
// separate threads.  A chunk [ja, jb] starts from the GYF values of row
// ja - 2 and computes row ja - 1 without storing it, which rebuilds exactly
// the values a single walk carries into row ja; it then stores the GY rows
// ja .. jb and the GYF rows ja - 1 .. jb - 1, so the chunks partition every
// output and each stored value is the one a single walk would store.
constexpr int AMD_SLOTS = 4;

template <typename R, int MODE>
__global__ void __launch_bounds__(128, 3) k_les_amd(const __grid_constant__ State s, Geom g, Phys ph) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
  if (x >= g.nx) return;
  const long long pp = g.pp;
  const long long col = (long long)z * g.nx + x;
  const int Nyp = g.ny;
  const int clen = (Nyp + 1 + gridDim.z - 1) / gridDim.z;
  const int ja = 1 + blockIdx.z * clen, jb = min(Nyp + 1, ja + clen - 1);
  if (ja > jb) return;
  const int j0 = ja >= 2 ? ja - 2 : 0;   // row the walk starts from (GYF values only)
  const int jst = g.jstart_th, jet = g.jend_th;
  const int j1 = g.jstart, j2 = Nyp - 1;
  const R h = 0.5;
  const double dxs_d = ph.dx * BETA_SGS, dzs_d = ph.dz * BETA_SGS;
  const R dxs = (R)dxs_d, dzs = (R)dzs_d;
  const R rzx = (R)(dzs_d / dxs_d), rxz = (R)(dxs_d / dzs_d);
  const LesRow* LR = s.lrow;
  const R* u1 = (const R*)s.u1 + col;
  const R* u2 = (const R*)s.u2 + col;
  const R* u3 = (const R*)s.u3 + col;
  const R* th = (const R*)s.th + col;
  const R *g1x = (const R*)s.gx[0] + col, *g2x = (const R*)s.gx[1] + col, *g3x = (const R*)s.gx[2] + col,
          *gtx = (const R*)s.gx[3] + col;
  const R *g1z = (const R*)s.gz[0] + col, *g2z = (const R*)s.gz[1] + col, *g3z = (const R*)s.gz[2] + col,
          *gtz = (const R*)s.gz[3] + col;
  R* o[11];
#pragma unroll
  for (int i = 0; i < 11; ++i) o[i] = (R*)s.les[i] + col;
  R* nut = (R*)s.nu_t + col;
  R* kat = (R*)s.kappa_t + col;
  float* fo = s.sgs_feat;
  const float* mo = s.sgs_out;
  const float* rng = s.sgs_range;
  if (MODE == 1 && ja == 1) {
#pragma unroll
    for (int f = 0; f < 16; ++f) fo[col * 16 + f] = 0.0f;
  }
  R hnu = 0, hka = 0;     // closure values at the previous GY row
  bool hval = false;

  // row j0: GYF values only (GY row 0 does not exist); with_mean: the
  // plane means when the fields hold fluctuations (mixed path)
  // (the products take the full values, the y-differences (ydiff) the
  // fluctuations, suffix _f, and the differences of the means)
  const long long o0 = (long long)j0 * pp;
  const double* pm = (sizeof(R) == sizeof(float)) ? s.pmean : nullptr;   // the split is a mixed-path form
  const int np = g.np;
  R u1m_f = __ldg(u1 + o0), u3m_f = __ldg(u3 + o0), thm_f = __ldg(th + o0), u2c_f = __ldg(u2 + o0 + pp);
  R u1m = with_mean(u1m_f, pm, 0, np, j0), u3m = with_mean(u3m_f, pm, 2, np, j0);
  R thm = with_mean(thm_f, pm, 3, np, j0), u2c = with_mean(u2c_f, pm, 1, np, j0 + 1);
  R f1x = __ldg(g1x + o0), f3z = __ldg(g3z + o0), f1z = __ldg(g1z + o0), f3x = __ldg(g3x + o0);
  R ftx = __ldg(gtx + o0), ftz = __ldg(gtz + o0);
  const R u2m1_f = __ldg(u2 + o0);
  R u2m1 = with_mean(u2m1_f, pm, 1, np, j0);
  R f2y = ydiff<R>(u2c_f, u2m1_f, pm, 1, np, j0 + 1, j0, LR[j0].idyf);
  // rows j - 2 of u1, u3, th and u2 (the products of plane j - 1)
  R u1mm = u1m, u3mm = u3m, thmm = thm, u2m2 = u2m1;
  // previous GY row (r = j - 1) values
  R h1y = 0, h3y = 0, hty = 0, h2x = 0, h2z = 0;
  R hSI4 = 0, hSI6 = 0, hO4 = 0, hO6 = 0, hP4 = 0, hP6 = 0, hdl = 0, hL5 = 0, hL6 = 0;
  if (MODE != 1 && ja == 1) {
    nut[0] = 0;
    kat[0] = 0;
  }

  // the 12 values a row needs come through a ring of AMD_SLOTS shared-memory
  // slots per thread, filled by cp.async AMD_SLOTS - 1 rows ahead: row j's
  // loads were issued while rows j - 3 .. j - 1 were computed
  extern __shared__ __align__(16) unsigned char amd_raw[];
  R* ring = reinterpret_cast<R*>(amd_raw);   // [slot][value][threadIdx.x]
  const int tb = blockDim.x, tx = threadIdx.x;
  const R* srcs[12] = {u1, u3, th, u2 + pp, g1x, g2x, g3x, gtx, g1z, g2z, g3z, gtz};
  auto issue = [&](int jr) {
    if (jr <= jb) {
      R* sl = ring + (jr % AMD_SLOTS) * 12 * tb + tx;
      const long long oj = (long long)jr * pp;
#pragma unroll
      for (int v = 0; v < 12; ++v) {
        if (v == 3 && jr + 1 > Nyp + 1) sl[v * tb] = (R)0;   // u2 above the top ghost plane
        else cp_async<sizeof(R)>(sl + v * tb, srcs[v] + oj);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int jr = 1; jr < AMD_SLOTS; ++jr) issue(j0 + jr);

  for (int j = j0 + 1; j <= jb; ++j) {
    const bool keep = j >= ja;   // row ja - 1 only rebuilds the carried values
    const long long oj = (long long)j * pp;
    issue(j + AMD_SLOTS - 1);
    cp_async_wait<AMD_SLOTS - 1>();
    const R* sl = ring + (j % AMD_SLOTS) * 12 * tb + tx;
    const R u1j_f = sl[0], u3j_f = sl[tb], thj_f = sl[2 * tb], u2n_f = sl[3 * tb];
    const R u1j = with_mean(u1j_f, pm, 0, np, j), u3j = with_mean(u3j_f, pm, 2, np, j);
    const R thj = with_mean(thj_f, pm, 3, np, j);
    const bool top = j + 1 > Nyp + 1;   // u2 above the top ghost plane (zero, no mean)
    const R u2n = top ? u2n_f : with_mean(u2n_f, pm, 1, np, j + 1);
    const R a1x = sl[4 * tb], a2x = sl[5 * tb], a3x = sl[6 * tb], atx = sl[7 * tb];
    const R a1z = sl[8 * tb], a2z = sl[9 * tb], a3z = sl[10 * tb], atz = sl[11 * tb];
    const LesRow lr = LR[j];
    // GY row j: y-derivatives and the tensors that live there
    const R d1y = ydiff<R>(u1j_f, u1m_f, pm, 0, np, j, j - 1, lr.idy);
    const R d3y = ydiff<R>(u3j_f, u3m_f, pm, 2, np, j, j - 1, lr.idy);
    const R dty = ydiff<R>(thj_f, thm_f, pm, 3, np, j, j - 1, lr.idy);
    const R dly = (R)lr.dys_y;
    const R ryx = (R)lr.ryx, rxy = (R)lr.rxy, rzy = (R)lr.rzy, ryz = (R)lr.ryz;
    const R SI4 = h * (d1y * ryx + a2x * rxy);
    const R SI6 = h * (a2z * rzy + d3y * ryz);
    const R O4 = h * (d1y * ryx - a2x * rxy);
    const R O6 = h * (a2z * rzy - d3y * ryz);
    const R S4 = h * (d1y + a2x), S6 = h * (a2z + d3y);
    // GYF row j (d u2/dy there needs u2 at j + 1; row Nyp + 1 is unused)
    const R c2y = (j <= Nyp) ? ydiff<R>(u2n_f, u2c_f, pm, 1, np, j + 1, j, lr.idyf) : (R)0;
    const R delt = (R)lr.dgy;
    R temp = 0, temp_th = 0;
    R nu_m = 0, ka_m = 0;
    bool val = false;
    if (MODE != 0) {
      const LesFeatIn<R> fi{a1x, f1x, a1z, f1z, a2x, a2z, a3x, f3x, a3z, f3z, atx, ftx, atz, ftz,
                            d1y, d3y, dty, c2y, f2y};
      float fv[16];
      les_features<R>(fi, (R)lr.wa, (R)lr.wb, dxs, dly, dzs, fv);
      const long long pt = (oj + col) * 16;
      if (MODE == 1) {
        if (keep) {
#pragma unroll
          for (int f = 0; f < 16; ++f) fo[pt + f] = fv[f];
        }
      } else {
        val = true;
#pragma unroll
        for (int f = 0; f < 16; ++f) val = val && (fv[f] >= rng[f]) && (fv[f] <= rng[16 + f]);
        nu_m = (R)mo[(oj + col) * 2];
        ka_m = (R)mo[(oj + col) * 2 + 1];
      }
    }
    if (MODE == 1) {
      u1m = u1j; u3m = u3j; thm = thj; u2c = u2n;
      u1m_f = u1j_f; u3m_f = u3j_f; thm_f = thj_f; u2c_f = u2n_f;
      f1x = a1x; f3z = a3z; f1z = a1z; f3x = a3x; ftx = atx; ftz = atz; f2y = c2y;
      continue;
    }
    if (j >= 2 && j <= Nyp) {
      const R wa = (R)lr.wa, wb = (R)lr.wb;
#define GYI(A, B) ((A) * wa + (B) * wb)
      const R SI5c = h * (a1z * rzx + a3x * rxz), SI5p = h * (f1z * rzx + f3x * rxz);
      const R O5c = h * (a1z * rzx - a3x * rxz), O5p = h * (f1z * rzx - f3x * rxz);
      temp = amd_ratio<R>(GYI(a1x, f1x), GYI(c2y, f2y), GYI(a3z, f3z), SI4, GYI(SI5c, SI5p), SI6, O4,
                          GYI(O5c, O5p), O6);
      temp_th = amd_th_ratio<R>(dxs, dly, dzs, GYI(a1x, f1x), GYI(c2y, f2y), GYI(a3z, f3z), d1y, a2x,
                                GYI(a1z, f1z), GYI(a3x, f3x), a2z, d3y, GYI(atx, ftx), dty, GYI(atz, ftz));
#undef GYI
      if (MODE == 2 && val) {
        temp = (R)-2 * nu_m / delt;
        temp_th = (R)-2 * ka_m / delt;
      }
    }
    const bool wall = (j <= 2 || j >= Nyp);     // ghost_les_mpi / ghost_les_th_mpi
    const R nu = wall ? (R)0 : -h * delt * temp;
    const R ka = wall ? (R)0 : -h * delt * temp_th;
    const R P4 = (j >= 2) ? temp * (S4 - h * d1y) : S4;
    const R P6 = (j >= 2) ? temp * (S6 - h * d3y) : S6;
    const bool gy2 = (j >= 2 && j <= Nyp);
    const R L5 = gy2 ? delt * P4 - nu * d1y : (R)0;
    const R L6 = gy2 ? delt * P6 - nu * d3y : (R)0;
    if (keep) {
      nut[oj] = nu;
      kat[oj] = ka;
    }

    // GYF row r = j - 1: needs GY rows r and r + 1 = j
    {
      const int r = j - 1;
      const long long orr = (long long)r * pp;
      const LesRow lf = LR[r];
      const R dlf = (R)lf.dgyf, idyfr = (R)lf.idyf;
      R L0 = 0, L1 = 0, L2 = 0, L3 = 0, L4 = 0, L7 = 0, L8 = 0;
      if (r >= j1 && r <= j2) {
        const R s4 = h * (SI4 + hSI4), s6 = h * (SI6 + hSI6);
        const R q4 = h * (O4 + hO4), q6 = h * (O6 + hO6);
        const R s5 = h * (f1z * rzx + f3x * rxz), q5 = h * (f1z * rzx - f3x * rxz);
        R s1 = amd_ratio<R>(f1x, f2y, f3z, s4, s5, s6, q4, q5, q6);
        if (MODE == 2 && val && hval) s1 = -(hnu + nu_m) / dlf;
        L0 = dlf * (s1 * f1x);
        L2 = dlf * (s1 * (h * (f1z + f3x)));
        L4 = dlf * (s1 * f3z);
        L1 = (delt * P4 - hdl * hP4) * idyfr;
        L3 = (delt * P6 - hdl * hP6) * idyfr;
      }
      if (r >= jst && r <= jet) {
        const R dys = (R)lf.dys_f;
        R s1t = amd_th_ratio<R>(dxs, dys, dzs, f1x, f2y, f3z, h * (d1y + h1y), h * (a2x + h2x), f1z, f3x,
                                h * (a2z + h2z), h * (d3y + h3y), ftx, h * (dty + hty), ftz);
        if (MODE == 2 && val && hval) s1t = -(hka + ka_m) / dlf;
        L7 = h * dlf * (s1t * ftx);
        L8 = h * dlf * (s1t * ftz);
      }
      // plane r: rows r - 1, r, r + 1 are u1mm, u1m, u1j (u3, th alike) and
      // u2m2, u2m1, u2c (products as in k_products' prod_ab)
      const bool q1 = in_rng(r, g.jstart, g.jend), q2 = in_rng(r, 2, Nyp), qt = in_rng(r, jst, jet);
      if (keep && q1) {
        const ProdY<R> y(g, r);
        o[0][orr] = u1m * u1m + L0;
        o[1][orr] = (u1j * u2c + u1m * u2c - u1m * u2m1 - u1mm * u2m1) * y.i2dyf + L1;
        o[2][orr] = u3m * u1m + L2;
        o[3][orr] = (u3j * u2c + u3m * u2c - u3m * u2m1 - u3mm * u2m1) * y.i2dyf + L3;
        o[4][orr] = u3m * u3m + L4;
      }
      if (keep && (q2 || qt)) {
        const ProdY<R> y(g, r);
        const R qrt = 0.25;
        const R sp = u2m1 + u2c, sm = u2m1 + u2m2;
        o[5][orr] = q2 ? (y.wj * u1m + y.wjm * u1mm) * u2m1 + hL5 : (R)0;
        o[6][orr] = q2 ? (qrt * (sp * sp) - qrt * (sm * sm)) * y.idy : (R)0;
        o[7][orr] = qt ? thm * u1m + L7 : (R)0;
        o[8][orr] = qt ? (thj * u2c + thm * u2c - thm * u2m1 - thmm * u2m1) * y.i2dyf : (R)0;
        o[9][orr] = q2 ? (y.wj * u3m + y.wjm * u3mm) * u2m1 + hL6 : (R)0;
        o[10][orr] = qt ? thm * u3m + L8 : (R)0;
      }
    }
    // shift
    u1mm = u1m; u3mm = u3m; thmm = thm; u2m2 = u2m1; u2m1 = u2c;
    hL5 = L5; hL6 = L6;
    u1m = u1j; u3m = u3j; thm = thj; u2c = u2n;
    u1m_f = u1j_f; u3m_f = u3j_f; thm_f = thj_f; u2c_f = u2n_f;
    f1x = a1x; f3z = a3z; f1z = a1z; f3x = a3x; ftx = atx; ftz = atz; f2y = c2y;
    h1y = d1y; h3y = d3y; hty = dty; h2x = a2x; h2z = a2z;
    hSI4 = SI4; hSI6 = SI6; hO4 = O4; hO6 = O6; hP4 = P4; hP6 = P6; hdl = delt;
    hnu = nu_m; hka = ka_m; hval = val;
  }
}

// ---------------------------------------------------------------------------
// CN solves with eddy viscosity: one thread per (x, z) column and equation
// (blockIdx.z: th, u2, u1, u3) runs a Thomas sweep (FP64 arithmetic, fields
// stored as R).  The matrix differs per column, so nothing is shared: the
// eliminated upper coefficients u_j / b'_j and right-hand side g_j / b'_j go
// to an FP64 scratch (2 fields per equation) and come back in the backward
// sweep.  Rows are handled in batches of TB whose loads are all issued
// first, so each thread keeps 3 TB loads in flight instead of waiting on
// every row.  On the mixed path the increment u_new - u goes out in FP64
// over the g / b' scratch of its equation (launch_thomas_les_inc gives the
// layout), and u itself is written only when keep_u (the third substep's
// CFL reads it).
constexpr int TB = 8;

template <typename R>
__global__ void __launch_bounds__(128) k_thomas_les(const __grid_constant__ State s, Geom g, int rk, int keep_u) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, eq = blockIdx.z;
  if (x >= g.nx) return;
  const int np = g.np, Nyp = g.ny;
  const long long pp = g.pp, col = (long long)z * g.nx + x;
  const double temp2 = 0.5 * s.sc->h_bar[rk];
  double* cmv = s.tscr + (long long)(2 * eq) * np * pp + col;   // u_j / b'_j
  double* gsv = cmv + (long long)np * pp;                         // g_j / b'_j
  constexpr bool INC = sizeof(R) == sizeof(float);   // r holds increments over u
  {
    const TriRow* Rw = s.tri + eq * np;
    R* u = (R*)((eq == 0) ? s.th : (eq == 1 ? s.u2 : (eq == 2 ? s.u1 : s.u3))) + col;
    R* r = (R*)((eq == 0) ? s.rth : (eq == 1 ? s.r2 : (eq == 2 ? s.r1 : s.r3))) + col;
    const R* nv = (const R*)((eq == 0) ? s.kappa_t : s.nu_t) + col;
    const int lo = (eq == 0) ? g.jstart_th - 1 : (eq == 1 ? 1 : g.jstart - 1);
    const int hi = (eq == 0) ? g.jend_th + 1 : (eq == 1 ? Nyp + 1 : g.jend + 1);
    // plane means of the old u when the fields hold fluctuations (mixed
    // path), added in FP64: the explicit and implicit terms then see the
    // FP32 rounding of the fluctuation only
    const double* pm = s.pmean ? s.pmean + (long long)((eq == 0) ? 3 : (eq == 1 ? 1 : (eq == 2 ? 0 : 2))) * np
                               : nullptr;
    auto old_u = [&](int j) { return (double)u[(long long)j * pp] + (pm ? pm[j] : 0.0); };
    double um = 0.0, uc = old_u(0), nm = 0.0, nc = (double)nv[0];
    double ibprev = 1.0, gprev = 0.0, uprev = 0.0;
    for (int jb = 0; jb < np; jb += TB) {
      double xr[TB], xu[TB], xn[TB];
#pragma unroll
      for (int c = 0; c < TB; ++c) {
        const int j = jb + c;
        xr[c] = (j < np) ? (double)r[(long long)j * pp] : 0.0;
        xu[c] = (j + 1 < np) ? old_u(j + 1) : 0.0;
        xn[c] = (j + 1 < np) ? (double)nv[(long long)(j + 1) * pp] : 0.0;
      }
#pragma unroll
      for (int c = 0; c < TB; ++c) {
        const int j = jb + c;
        if (j >= np) break;
        const TriRow row = Rw[j];
        const double un = xu[c], nn = xn[c];
        double l = row.l, d = row.d, uu = row.u, v = row.bc;
        if (!row.is_bc) {
          // eddy coupling to the rows below / above: nu_t (kappa_t) at GY
          // rows j, j+1, or for u2 averaged to the GYF rows around GY row j
          const double lo_c = (eq != 1 ? nc : nc + nm) * row.ef_lo;
          const double hi_c = (eq != 1 ? nn : nc + nn) * row.ef_hi;
          v = (INC ? xr[c] + uc : xr[c]) + (row.cn_hi * (un - uc) - row.cn_lo * (uc - um)) +
              temp2 * (hi_c * (un - uc) - lo_c * (uc - um));
          l = l - temp2 * lo_c;
          d = d + temp2 * hi_c + temp2 * lo_c;
          uu = uu - temp2 * hi_c;
        }
        double b = d, gg = v;
        if (j > 0) {
          const double a = -l * ibprev;
          b = d + a * uprev;
          gg = v + a * gprev;
        }
        const double ib = 1.0 / b;
        cmv[(long long)j * pp] = uu * ib;
        gsv[(long long)j * pp] = gg * ib;
        ibprev = ib; gprev = gg; uprev = uu;
        um = uc; uc = un; nm = nc; nc = nn;
      }
    }
    double xnext = 0.0;
    bool bad = false;   // a non-finite new state (reported as DB_FLAG_NONFINITE)
    for (int jt = np - 1; jt >= 0; jt -= TB) {
      double xc[TB], xg[TB], xo[TB];
#pragma unroll
      for (int c = 0; c < TB; ++c) {
        const int j = jt - c;
        xc[c] = (j >= 0) ? cmv[(long long)j * pp] : 0.0;
        xg[c] = (j >= 0) ? gsv[(long long)j * pp] : 0.0;
        xo[c] = (INC && j >= 0) ? old_u(j) : 0.0;
      }
#pragma unroll
      for (int c = 0; c < TB; ++c) {
        const int j = jt - c;
        if (j < 0) break;
        const double xv = xg[c] - xc[c] * xnext;
        bad = bad || !(fabs(xv) <= 1.7976931348623157e308);
        const bool stored = (j >= lo && j <= hi);
        if (stored && (!INC || keep_u)) u[(long long)j * pp] = (R)xv;
        // increment for the FP64 forward transforms, over g_j / b'_j (read above)
        if (INC) gsv[(long long)j * pp] = stored ? xv - xo[c] : 0.0;
        xnext = xv;
      }
    }
    if (bad) atomicOr(g.flags, DB_FLAG_NONFINITE);
  }
}

// ---------------------------------------------------------------------------
cudaError_t launch_les_bc(const Geom& g, const Phys& ph, const State& s, cudaStream_t st) {
  k_les_bc<<<dim3((g.kxs + 127) / 128, g.nkzp), 128, 0, st>>>(s, g, ph);
  return cudaGetLastError();
}
cudaError_t launch_les_amd(const Geom& g, const Phys& ph, const State& s, cudaStream_t st, int mode) {
  // wall-normal chunks (tuned, else until about 16 warps per SM walk
  // columns; each chunk at least 8 rows), then columns per CTA: 128, narrowed (to 32 at least)
  // until every SM has two CTAs
  const long long cols = (long long)g.nx * g.nz, want = 512LL * sm_count();
  const int maxch = (g.ny + 1) / 8 > 1 ? (g.ny + 1) / 8 : 1;
  int nch = g.tune_amd_ch > 0 ? g.tune_amd_ch : (int)((want + cols - 1) / cols);
  nch = nch < 1 ? 1 : (nch > maxch ? maxch : nch);
  int bx = g.nx < 128 ? g.nx : 128;
  while (bx > 32 && bx % 2 == 0 && (long long)((g.nx + bx - 1) / bx) * g.nz * nch < 2LL * sm_count()) bx >>= 1;
  const dim3 grid((g.nx + bx - 1) / bx, g.nz, nch);
  const size_t smem = (size_t)AMD_SLOTS * 12 * bx * (g.prec ? sizeof(float) : sizeof(double));
  if (g.prec) {
    if (mode == 1) k_les_amd<float, 1><<<grid, bx, smem, st>>>(s, g, ph);
    else if (mode == 2) k_les_amd<float, 2><<<grid, bx, smem, st>>>(s, g, ph);
    else k_les_amd<float, 0><<<grid, bx, smem, st>>>(s, g, ph);
  } else {
    if (mode == 1) k_les_amd<double, 1><<<grid, bx, smem, st>>>(s, g, ph);
    else if (mode == 2) k_les_amd<double, 2><<<grid, bx, smem, st>>>(s, g, ph);
    else k_les_amd<double, 0><<<grid, bx, smem, st>>>(s, g, ph);
  }
  return cudaGetLastError();
}
// where the mixed path's LES solve leaves its FP64 increments (physical,
// fields u1, u2, u3, th) and the FP64 x-half scratch their forward x-pass
// can use (the other half of each equation's solve scratch)
void thomas_les_inc(const Geom& g, const State& s, double* inc[4], double2* xh64[4]) {
  const int eq_of[4] = {2, 1, 3, 0};   // u1, u2, u3, th -> th, u2, u1, u3 order
  const long long f = (long long)g.np * g.pp;
  for (int i = 0; i < 4; ++i) {
    inc[i] = s.tscr + (2 * eq_of[i] + 1) * f;
    xh64[i] = reinterpret_cast<double2*>(s.tscr + 2 * eq_of[i] * f);
  }
}
cudaError_t launch_thomas_les(const Geom& g, const State& s, int rk, cudaStream_t st, bool keep_u) {
  const int want = (g.tune_les_tb > 0 && g.tune_les_tb <= 128) ? g.tune_les_tb : 128;   // powers of two
  const int bx = g.nx < want ? g.nx : want;
  if (g.prec) k_thomas_les<float><<<dim3(g.nx / bx, g.nz, 4), bx, 0, st>>>(s, g, rk, keep_u ? 1 : 0);
  else k_thomas_les<double><<<dim3(g.nx / bx, g.nz, 4), bx, 0, st>>>(s, g, rk, 1);
  return cudaGetLastError();
}

}  // namespace db
