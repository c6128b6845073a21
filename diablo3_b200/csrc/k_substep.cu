// k_substep.cu -- the RKW3 + Crank-Nicolson substep (rk_chan_1,
// for/solver.f90:366-1273) as fused B200 kernels; arithmetic in FP64, or
// FP32 transforms and products on the mixed path.
//
//  k_products    : 11 nonlinear products of u1,u2,u3,th in physical space
//                  (solver.f90:655-815, 914-956) fused with their forward
//                  x-FFTs; x-derivatives (i kx) applied in the x-half space so
//                  only 8 x-half fields leave the kernel.
//  k_zpass_rhs   : (with LES) forward z-FFT of those 8 fields, the spectral
//                  linear terms (viscous, Coriolis, buoyancy, background-front
//                  advection, thermal-wind advection: solver.f90:396-609,
//                  35-111) and the RK combination cr = cu + zeta h cf_old -
//                  h grad p + beta h cf (solver.f90:396-456, 824-838,
//                  966-973), cr through the inverse z-FFT to the physical solve.
//  k_tri_coef    : the four implicit systems' rows incl. BC rows
//                  (solver.f90:1012-1233, 1901-2324), LU-factored once per
//                  substep (all (x,z) columns share them without LES).
//  k_rhs_cn,     : without LES, after the forward z-FFT of the 8 fields: the
//  k_cn_back       spectral RHS and the CN solves of th, u2, u1, u3 per
//                  retained Fourier mode (explicit CN term + Thomas sweeps,
//                  solver.f90:850-870, 981-989, 1691-1852), FP64.
//  k_rem_div     : per (kx,kz) column, divergence, complex Thomas, projection
//                  and pressure update (solver.f90:1302-1379, 1261-1267).
//  k_courant     : CFL reduction and dt scheduling (flow.f90:746-857).
// The CN solves with eddy viscosity (one matrix per column) are in k_les.cu.
#include <math.h>

#include "../../include/diablo_b200.h"
#include "db_bc.cuh"
#include "db_kernels.cuh"
#include "fft_reg.cuh"
#include "umma.cuh"

namespace db {


// ---------------------------------------------------------------------------
// nonlinear products + forward x-FFT.  One CTA per (z, j) row and group; each
// complex sequence carries two real products a + i b:
//  group 0 (u1 and u3 momentum, rows jstart..jend):
//    s0 = (u1 u1 | Dy u1u2)  s1 = (u1 u3 | Dy u3u2)  s2 = (u3 u3 | 0)
//  group 1 (u2 momentum rows 2..Nyp; scalar rows jstart_th..jend_th):
//    s0 = (<u1> u2 | Dy u2u2)  s1 = (th u1 | Dy th u2)  s2 = (<u3> u2 | th u3)
// Outputs (x-half), o = 0..7 = N1 M1 N3 M3 N2 M2 NT MT with
//  N = ikx X(a) + X(b) of one sequence, M = one part of a sequence:
//  N1 = s0(g0)  M1 = s1.a(g0)  N3 = s1(g0)  M3 = s2.a(g0)
//  N2 = s0(g1)  M2 = s2.a(g1)  NT = s1(g1)  MT = s2.b(g1)
// so that cf_e -= Z(N_e) + ikz Z(M_e) after the z-pass (solver.f90:655-815,
// 914-964; <.> is the interpolation to GY points, Dy the conservative
// y-difference).
template <int N, typename C>
__device__ __forceinline__ C sepp(const C* z, int m, int part) {
  using R = typename RealOf<C>::type;
  const C zm = z[pidx(m)], zn = cconj(z[pidx((N - m) & (N - 1))]);
  if (part == 0) return mkc<C>((R)0.5 * (zm.x + zn.x), (R)0.5 * (zm.y + zn.y));
  return mkc<C>((R)0.5 * (zm.y - zn.y), (R)-0.5 * (zm.x - zn.x));
}

// rows j-1 (m), j, j+1 (p) of u1, u2, u3, th
template <typename R>
struct ProdRows {
  const R *u1m, *u1, *u1p, *u2m, *u2, *u2p, *u3m, *u3, *u3p, *thm, *th, *thp;
};

// the real pair (a, b) sequence `seq` of group `grp` carries at point x
// (the LES substep forms the same products in k_les.cu's column walk)
template <typename R>
__device__ __forceinline__ void prod_ab(const ProdRows<R>& P, int grp, int seq, int x, bool r2, bool rt,
                                        const ProdY<R>& y, R& a, R& b) {
  const R qrt = 0.25;
  a = 0;
  b = 0;
  if (grp == 0) {
    const R u1 = P.u1[x], u3 = P.u3[x];
    if (seq == 0) {
      const R u1p = P.u1p[x], u1m = P.u1m[x];
      const R u2p = P.u2p[x], u2 = P.u2[x];
      a = u1 * u1;
      b = (u1p * u2p + u1 * u2p - u1 * u2 - u1m * u2) * y.i2dyf;
    } else if (seq == 1) {
      const R u3p = P.u3p[x], u3m = P.u3m[x];
      const R u2p = P.u2p[x], u2 = P.u2[x];
      a = u3 * u1;
      b = (u3p * u2p + u3 * u2p - u3 * u2 - u3m * u2) * y.i2dyf;
    } else {
      a = u3 * u3;
    }
  } else {
    const R u2 = P.u2[x];
    if (seq == 0) {
      if (r2) {
        const R u1 = P.u1[x], u1m = P.u1m[x];
        const R pp = u2 + P.u2p[x], qq = u2 + P.u2m[x];
        a = (y.wj * u1 + y.wjm * u1m) * u2;
        b = (qrt * (pp * pp) - qrt * (qq * qq)) * y.idy;
      }
    } else if (seq == 1) {
      if (rt) {
        const R th = P.th[x], thp = P.thp[x], thm = P.thm[x];
        const R u2p = P.u2p[x];
        a = th * P.u1[x];
        b = (thp * u2p + th * u2p - th * u2 - thm * u2) * y.i2dyf;
      }
    } else {
      if (r2) a = (y.wj * P.u3[x] + y.wjm * P.u3m[x]) * u2;
      if (rt) b = P.th[x] * P.u3[x];
    }
  }
}

// outputs of one transformed sequence (in sq, natural order), scaled by
// 1/Nx: an N-type output ikx X(a) + X(b), and for s1 (group 0) / s2 (both
// groups) the parts
template <int N, typename C>
__device__ __forceinline__ void prod_out(C* const* xh, const C* sq, const Geom& g, long long hrow, int grp, int seq,
                                         int lane, bool r2, bool rt) {
  using R = typename RealOf<C>::type;
  constexpr int T = FftShape<N>::T;
  const R sc = (R)(1.0 / (double)N);
  const bool n_out = (seq < 2) ? ((grp == 0) || (seq == 0 ? r2 : rt)) : false;
  const int o_n = (grp == 0) ? (seq == 0 ? 0 : 2) : (seq == 0 ? 4 : 6);
  const C Z = mkc<C>(0, 0);
  for (int mm = lane; mm < g.kxs; mm += T) {
    const bool live = mm <= g.nkx;
    const C A = live ? sepp<N>(sq, mm, 0) : Z;
    const C B = live ? sepp<N>(sq, mm, 1) : Z;
    if (seq < 2) {
      const R k = (R)g.kx[mm];
      xh[o_n][hrow + mm] = n_out ? mkc<C>((B.x - k * A.y) * sc, (B.y + k * A.x) * sc) : Z;
    }
    if (grp == 0 && seq == 1) xh[1][hrow + mm] = mkc<C>(A.x * sc, A.y * sc);       // M1
    if (grp == 0 && seq == 2) xh[3][hrow + mm] = mkc<C>(A.x * sc, A.y * sc);       // M3
    if (grp == 1 && seq == 2) {
      xh[5][hrow + mm] = r2 ? mkc<C>(A.x * sc, A.y * sc) : Z;  // M2
      xh[7][hrow + mm] = rt ? mkc<C>(B.x * sc, B.y * sc) : Z;  // MT
    }
  }
}

// One CTA per (z, j, group), rows read from global memory (Nx > 512).
// Sequences of 128 threads and more: no minimum of resident CTAs, so the
// FFT's registers do not spill.
template <int N, typename R>
__global__ void __launch_bounds__(3 * FftShape<N>::T, FftShape<N>::T >= 128 ? 1 : DB_LB_PROD) k_products(const __grid_constant__ State s, Geom g) {
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int z = blockIdx.x, j = blockIdx.y, grp = blockIdx.z;
  const bool r1 = in_rng(j, g.jstart, g.jend);
  const bool r2 = in_rng(j, 2, g.ny);
  const bool rt = in_rng(j, g.jstart_th, g.jend_th);
  const long long hrow = (long long)j * g.hp + (long long)z * g.kxs;
  C* const* xh = reinterpret_cast<C* const*>(s.xh);
  if ((grp == 0 && !r1) || (grp == 1 && !(r2 || rt))) {
    for (int idx = threadIdx.x; idx < 4 * g.kxs; idx += blockDim.x)
      xh[4 * grp + idx / g.kxs][hrow + idx % g.kxs] = mkc<C>(0, 0);
    return;
  }
  C* sq = sm + seq * padded(N);
  const C* twt = tw_x<R>(g);   // twiddles fetched per pass (fewer live registers)
  const long long o0 = (long long)j * g.pp + (long long)z * g.nx;
  const long long om = o0 - g.pp, op = o0 + g.pp;
  const R* U1 = (const R*)s.u1;
  const R* U2 = (const R*)s.u2;
  const R* U3 = (const R*)s.u3;
  const R* TH = (const R*)s.th;
  const ProdRows<R> P{U1 + om, U1 + o0, U1 + op, U2 + om, U2 + o0, U2 + op,
                      U3 + om, U3 + o0, U3 + op, TH + om, TH + o0, TH + op};
  const ProdY<R> y(g, j);
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) {
    R a, b;
    prod_ab(P, grp, seq, lane + q * T, r2, rt, y, a, b);
    v[q] = mkc<C>(a, b);
  }
  fft_reg_lazy<N, -1>(v, lane, true, sq, twt);
  SEQ_SYNC(N);
#pragma unroll
  for (int q = 0; q < E; ++q) sq[pidx(lane + q * T)] = v[q];
  SEQ_SYNC(N);
  prod_out<N>(xh, sq, g, hrow, grp, seq, lane, r2, rt);
}

// Persistent y-marching form (Nx <= 512).  A work item is a block of zr
// consecutive z rows and a range of planes j; the CTA walks the planes in
// order, keeping the rows j-1, j, j+1 of u1, u2, u3, th in a ring of
// shared-memory slots filled by TMA bulk copies that overlap the FFTs.
//  FP64: four slots; at the start of plane j, plane j+2 goes into the slot
//        plane j-2 occupied.  Two CTAs per SM (the registers of the FP64
//        transform).
//  FP32: three slots; once both groups have read plane j-1 (a CTA barrier
//        after the second group's products), plane j+2 goes into its slot,
//        overlapping the second group's FFT and the next plane's first
//        group.  With an exchange stride of padded(N) - 1 a CTA holds
//        < 76 KB of shared memory, and three CTAs share an SM.
// Thread layout: sequence (zi, seq) = (sidx / 3, sidx % 3).
template <typename R>
constexpr int prod_slots() { return sizeof(R) == sizeof(double) ? 4 : 3; }
constexpr uint32_t PROD_WAIT = 1u << 24;

template <int N>
constexpr int prod_zr() { return FftShape<N>::T >= 64 ? 1 : 64 / FftShape<N>::T; }
// exchange-buffer stride of one sequence: the largest index pidx(N - 1) + 1
template <int N>
constexpr int prod_sq() { return padded(N) - 1; }

// B: member-batched (blockIdx.y = member, its items over gridDim.x CTAs)
template <int N, typename R, bool B = false>
__global__ void __launch_bounds__(192, prod_slots<R>() == 4 ? 2 : 3) k_products_st(const __grid_constant__ State s0, Geom g0, int zr, int nzb,
                                                        int jlen, int nitems, const MemberArgs* __restrict__ tab) {
  const int mb = B ? (int)blockIdx.y : 0;
  const State& s = B ? tab[mb].s : s0;
  const Geom& g = g0;   // the same geometry for every member
  using C = typename CplxOf<R>::type;
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const uint32_t fbytes = (uint32_t)zr * N * sizeof(R);   // one field, zr rows of one plane
  const uint32_t slot_bytes = 4u * fbytes;
  constexpr int SQ = prod_sq<N>();
  constexpr int PROD_SLOTS = prod_slots<R>();
  C* xbuf = reinterpret_cast<C*>(sm_raw + PROD_SLOTS * slot_bytes);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm_raw + PROD_SLOTS * slot_bytes + (size_t)3 * zr * SQ * sizeof(C));
  const int sidx = threadIdx.x / T, lane = threadIdx.x % T;
  const int zi = sidx / 3, seq = sidx % 3;
  C* sq = xbuf + sidx * SQ;
  const C* twt = tw_x<R>(g);
  C* const* xh = reinterpret_cast<C* const*>(s.xh);
  const int np = g.np;
  if (threadIdx.x < PROD_SLOTS) mbar_init(&mbar[threadIdx.x], 1);
  __syncthreads();
  uint32_t par = 0;    // parity of the next completion of each slot
  uint32_t pend = 0;   // slots with a copy issued and not yet waited for
  auto issue = [&](int jr, int z0) {   // plane jr of the four fields into its slot
    const int sl = jr % PROD_SLOTS;
    if (threadIdx.x == 0) {
      fence_async_smem();
      unsigned char* dst = sm_raw + sl * slot_bytes;
      const long long off = (long long)jr * g.pp + (long long)z0 * g.nx;
      mbar_expect_tx(&mbar[sl], slot_bytes);
      bulk_g2s(dst, (const R*)s.u1 + off, fbytes, &mbar[sl]);
      bulk_g2s(dst + fbytes, (const R*)s.u2 + off, fbytes, &mbar[sl]);
      bulk_g2s(dst + 2 * fbytes, (const R*)s.u3 + off, fbytes, &mbar[sl]);
      bulk_g2s(dst + 3 * fbytes, (const R*)s.th + off, fbytes, &mbar[sl]);
    }
    pend |= 1u << sl;
  };
  // a wait that gives up leaves its slot pending (same parity), so the
  // drain below waits for that copy before the CTA leaves
  auto wait_row = [&](int jr) -> bool {
    const int sl = jr % PROD_SLOTS;
    const bool ok = mbar_wait_first(&mbar[sl], (par >> sl) & 1u, g.wait_first, PROD_WAIT);
    if (ok) {
      par ^= 1u << sl;
      pend &= ~(1u << sl);
    }
    return ok;
  };
  auto row = [&](int jr, int f) -> const R* {
    return reinterpret_cast<const R*>(sm_raw + (jr % PROD_SLOTS) * slot_bytes + f * fbytes) + zi * N;
  };
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int zb = it % nzb, jc = it / nzb;
    const int z0 = zb * zr, z = z0 + zi;
    const int jlo = jc * jlen, jhi = min(np - 1, jlo + jlen - 1);
    const int jtop = min(np - 1, jhi + 1);
    __syncthreads();   // every slot is free
    for (int jr = max(0, jlo - 1); jr <= min(jtop, jlo + 1); ++jr) issue(jr, z0);
    for (int j = jlo; j <= jhi; ++j) {
      bool ok = true;
      if (j == jlo) {
        for (int jr = max(0, jlo - 1); jr <= min(jtop, jlo + 1); ++jr) ok = wait_row(jr) && ok;
      } else if (j + 1 <= jtop) {
        ok = wait_row(j + 1);
      }
      if (__syncthreads_and(ok ? 1 : 0) == 0) {   // a copy did not land in time: record, drain (bounded), leave
        if (threadIdx.x == 0) {
          atomicOr(B ? tab[mb].g.flags : g.flags, DB_FLAG_WAIT_TIMEOUT);
          for (int sl = 0; sl < PROD_SLOTS; ++sl)
            if (pend >> sl & 1u) mbar_wait(&mbar[sl], (par >> sl) & 1u, PROD_WAIT);
        }
        return;
      }
      if (PROD_SLOTS == 4 && j + 2 <= jtop) issue(j + 2, z0);   // into the slot of plane j - 2
      const bool r1 = in_rng(j, g.jstart, g.jend);
      const bool r2 = in_rng(j, 2, g.ny);
      const bool rt = in_rng(j, g.jstart_th, g.jend_th);
      const ProdY<R> y(g, j);
      const long long hrow = (long long)j * g.hp + (long long)z * g.kxs;
      for (int grp = 0; grp < 2; ++grp) {
        const bool zero = (grp == 0 && !r1) || (grp == 1 && !(r2 || rt));   // uniform over the CTA
        C v[E];
        if (!zero) {
          const int jm = j >= 1 ? j - 1 : j, jp = j + 1 <= np - 1 ? j + 1 : j;
          const ProdRows<R> P{row(jm, 0), row(j, 0), row(jp, 0), row(jm, 1), row(j, 1), row(jp, 1),
                              row(jm, 2), row(j, 2), row(jp, 2), row(jm, 3), row(j, 3), row(jp, 3)};
#pragma unroll
          for (int q = 0; q < E; ++q) {
            R a, b;
            prod_ab(P, grp, seq, lane + q * T, r2, rt, y, a, b);
            v[q] = mkc<C>(a, b);
          }
        }
        if (PROD_SLOTS == 3 && grp == 1) {   // plane j - 1 is read for the last time: its slot takes plane j + 2
          __syncthreads();
          if (j + 2 <= jtop) issue(j + 2, z0);
        }
        if (zero) {
          const long long hrow0 = (long long)j * g.hp + (long long)z0 * g.kxs;
          const int w = zr * g.kxs;
          for (int idx = threadIdx.x; idx < 4 * w; idx += blockDim.x)
            xh[4 * grp + idx / w][hrow0 + idx % w] = mkc<C>(0, 0);
          continue;
        }
        fft_reg_lazy<N, -1>(v, lane, true, sq, twt);
        SEQ_SYNC(N);
#pragma unroll
        for (int q = 0; q < E; ++q) sq[pidx(lane + q * T)] = v[q];
        SEQ_SYNC(N);
        prod_out<N>(xh, sq, g, hrow, grp, seq, lane, r2, rt);
        SEQ_SYNC(N);   // sq is the next group's exchange buffer
      }
    }
  }
}

// LES substep form: the 11 real sequences of each plane come ready from the
// closure's column walk (product + SGS forcing, k_les.cu, les[0..10] in
// (group, sequence, part) order), so a CTA of zr z rows of one plane and one
// group loads its pairs, transforms and separates; no neighbouring planes.
template <int N, typename R>
__global__ void __launch_bounds__(3 * FftShape<N>::T * prod_zr<N>()) k_products_les(const __grid_constant__ State s,
                                                                                    Geom g, int zr) {
  using C = typename CplxOf<R>::type;
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int sidx = threadIdx.x / T, lane = threadIdx.x % T;
  const int zi = sidx / 3, seq = sidx % 3;
  const int z0 = blockIdx.x * zr, z = z0 + zi, j = blockIdx.y, grp = blockIdx.z;
  const bool r1 = in_rng(j, g.jstart, g.jend);
  const bool r2 = in_rng(j, 2, g.ny);
  const bool rt = in_rng(j, g.jstart_th, g.jend_th);
  C* const* xh = reinterpret_cast<C* const*>(s.xh);
  if ((grp == 0 && !r1) || (grp == 1 && !(r2 || rt))) {   // uniform over the CTA
    const long long hrow0 = (long long)j * g.hp + (long long)z0 * g.kxs;
    const int w = zr * g.kxs;
    for (int idx = threadIdx.x; idx < 4 * w; idx += blockDim.x)
      xh[4 * grp + idx / w][hrow0 + idx % w] = mkc<C>(0, 0);
    return;
  }
  C* sq = reinterpret_cast<C*>(sm_raw) + sidx * padded(N);
  const C* twt = tw_x<R>(g);
  const long long o0 = (long long)j * g.pp + (long long)z * g.nx;
  const int ia = grp == 0 ? 2 * seq : 5 + 2 * seq;   // fields of parts a, b (group 0 sequence 2: b = 0)
  const bool hasb = !(grp == 0 && seq == 2);
  const R* A = (const R*)s.les[ia] + o0;
  const R* B = (const R*)s.les[hasb ? ia + 1 : ia] + o0;
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const int x = lane + q * T;
    v[q] = mkc<C>(A[x], hasb ? B[x] : (R)0);
  }
  fft_reg_lazy<N, -1>(v, lane, true, sq, twt);
  SEQ_SYNC(N);
#pragma unroll
  for (int q = 0; q < E; ++q) sq[pidx(lane + q * T)] = v[q];
  SEQ_SYNC(N);
  prod_out<N>(xh, sq, g, (long long)j * g.hp + (long long)z * g.kxs, grp, seq, lane, r2, rt);
}

// ---------------------------------------------------------------------------
// The spectral RHS at one mode (kx, kzp) of plane j for equation e (0 u1,
// 1 u3, 2 u2, 3 th): the linear terms cf (to be stored), the RK combination
// cr = cu + zeta h cf_old - h grad p + beta h cf (solver.f90:396-609,
// 824-838, 966-973, 35-111).  rhs_load reads the state values equation e
// needs at address a (the others stay zero), rhs_eval combines them, so a
// caller can issue the loads of several planes before their arithmetic.
struct RhsIn {
  double2 own;          // the equation's own field
  double2 cu1, cu3, cth, cp;
  double2 nb2, nbp;     // e 0/1: cu2 of planes j and j+1; e 2: cth and cp of plane j-1
  double2 cfo;          // cf of the previous substep (rk > 0)
};
// a hint that brings the line holding p into L2 (p must be a valid global
// address)
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(p)));
}

__device__ __forceinline__ RhsIn rhs_load(const State& s, const Geom& g, int rk, int e, long long a) {
  const double2 z = make_double2(0.0, 0.0);
  RhsIn v{z, z, z, z, z, z, z, z};
  if (e == 0 || e == 1) {
    v.cu1 = s.cu1[a]; v.cu3 = s.cu3[a]; v.cth = s.cth[a]; v.cp = s.cp[a];
    v.own = (e == 0) ? v.cu1 : v.cu3;
    v.nb2 = s.cu2[a]; v.nbp = s.cu2[a + g.sp];
    if (rk > 0) v.cfo = (e == 0) ? s.cf1[a] : s.cf3[a];
  } else if (e == 2) {
    v.own = s.cu2[a]; v.cth = s.cth[a]; v.cp = s.cp[a];
    v.nb2 = s.cth[a - g.sp]; v.nbp = s.cp[a - g.sp];
    if (rk > 0) v.cfo = s.cf2[a];
  } else {
    v.own = s.cth[a]; v.cu1 = s.cu1[a]; v.cu3 = s.cu3[a];
    if (rk > 0) v.cfo = s.cfth[a];
  }
  return v;
}
__device__ __forceinline__ double2* rhs_cf(const State& s, int e) {
  return (e == 0) ? s.cf1 : (e == 1 ? s.cf3 : (e == 2 ? s.cf2 : s.cfth));
}
// The constants of one mode and substep (the same on every plane):
// temp3..5 = zeta h, h, beta h; the wavenumbers; |k|^(2 beta).
struct RhsK {
  double temp3, temp4, temp5, kxv, kzv, kk;
};
__device__ __forceinline__ RhsK rhs_consts(const State& s, const Geom& g, const Phys& ph, int rk, int kx, int kzp) {
  RhsK c;
  const double hb = s.sc->h_bar[rk];
  c.temp3 = zeta_bar(rk) * hb;
  c.temp4 = hb;
  c.temp5 = beta_bar(rk) * hb;
  c.kxv = g.kx[kx];
  c.kzv = g.kz[kzp];
  const double k2 = c.kxv * c.kxv + c.kzv * c.kzv;
  c.kk = (ph.beta == 1.0) ? k2 : pow(k2, ph.beta);
  return c;
}
// nl = (Z(N) + i kz Z(M)) / Nz, the nonlinear term of the mode; with INC the
// increment cr - own is returned.
template <bool INC>
__device__ __forceinline__ double2 rhs_eval(const State& s, const Geom& g, const Phys& ph, int rk, int e, int j,
                                            int kx, int kzp, double2 nl, const RhsIn& v, const RhsK& c,
                                            double2& cf) {
  const double temp3 = c.temp3, temp4 = c.temp4, temp5 = c.temp5;
  const double nu = ph.nu, f = ph.ro_inv / ph.delta;
  const double tw = ph.delta / ph.ro_inv;  // delta / Ro_inv
  const double kxv = c.kxv, kzv = c.kzv, kk = c.kk;
  double2 cr;
  if (e == 0 || e == 1) {
    const double2 v2 = make_double2(0.5 * (v.nb2.x + v.nbp.x), 0.5 * (v.nb2.y + v.nbp.y));
    const double2 cu = v.own;
    cf = cscale(cu, -nu * kk);
    if (e == 0) {
      cf = cadd(cf, cscale(v.cu3, f));
      cf = cadd(cf, cscale(v.cth, ph.grav_x));
    } else {
      cf = csub(cf, cscale(v.cu1, f));
      cf = cadd(cf, cscale(v.cth, ph.grav_z));
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
    cr = INC ? make_double2(0.0, 0.0) : cu;
    if (rk > 0) cr = cadd(cr, cscale(v.cfo, temp3));
    cr = csub(cr, cscale(cmul_i(v.cp, 1.0), temp4 * kd));
    if (e == 0 && kx == 0 && kzp == 0) {
      if (ph.f_type == 1) cr.x -= temp4 * ph.px0;
      if (ph.f_type == 2) cr.x -= temp4 * (ph.px0 + ph.amp_omega0 * cos(ph.omega0 * s.sc->time));
    }
    cr = cadd(cr, cscale(cf, temp5));
  } else if (e == 2) {
    const double2 cu2 = v.own;
    cf = cscale(cu2, -nu * kk);
    if (!(kx == 0 && kzp == 0)) {
      const double2 t0 = v.cth, tm = v.nb2;
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
    cr = INC ? make_double2(0.0, 0.0) : cu2;
    if (rk > 0) cr = cadd(cr, cscale(v.cfo, temp3));
    const double2 dp = csub(v.cp, v.nbp);
    cr = csub(cr, cscale(dp, temp4 / g.dy[j]));
    cr = cadd(cr, cscale(cf, temp5));
  } else {
    const double2 cth = v.own;
    cf = cscale(cth, -(nu / ph.pr) * kk);
    cf = csub(cf, cscale(v.cu1, ph.dthdx));
    cf = csub(cf, cscale(v.cu3, ph.dthdz));
    if (ph.front_tw) {
      const double y = g.gyf[j] - 0.5 * ph.ly;
      const double2 t1 = cmul_i(cth, 1.0);
      cf = csub(cf, cscale(t1, tw * ph.dthdx * y * kzv));
      cf = csub(cf, cscale(t1, tw * (-1.0) * ph.dthdz * y * kxv));
    }
    cf = csub(cf, nl);
    cr = INC ? make_double2(0.0, 0.0) : cth;
    if (rk > 0) cr = cadd(cr, cscale(v.cfo, temp3));
    cr = cadd(cr, cscale(cf, temp5));
  }
  return cr;
}
// Load, evaluate and store cf at one mode; with INC and a ghost overlay
// the rows whose base the inverse transforms took from the overlay return
// cr - base = (cu - base) + increment.
template <bool INC>
__device__ __forceinline__ double2 rhs_point(const State& s, const Geom& g, const Phys& ph, int rk, int e, int j,
                                             int kx, int kzp, double2 nl, const double2* __restrict__ ghost) {
  const long long a = (long long)j * g.sp + (long long)kzp * g.kxs + kx;
  const RhsIn v = rhs_load(s, g, rk, e, a);
  double2 cf;
  double2 cr = rhs_eval<INC>(s, g, ph, rk, e, j, kx, kzp, nl, v, rhs_consts(s, g, ph, rk, kx, kzp), cf);
  rhs_cf(s, e)[a] = cf;
  if (INC && ghost) {
    const int qg = (j <= 1) ? j : (j >= g.ny ? j - g.ny + 2 : -1);
    if (qg >= 0) {
      const int gf = (e == 0) ? 0 : (e == 1 ? 2 : (e == 2 ? 1 : 3));
      const double2 base = ghost[(long long)(4 * gf + qg) * g.sp + (long long)kzp * g.kxs + kx];
      cr = cadd(cr, csub(v.own, base));
    }
  }
  return cr;
}

// z-pass of the nonlinear terms + spectral RHS + inverse z-pass of cr.
// One CTA = KT kx columns of plane j; thread t owns column t % KT and the
// z-set {lane + q N/8}.  Equation e: 0 -> u1, 1 -> u3, 2 -> u2, 3 -> th;
// x-half inputs xh[2e] (N_e), xh[2e+1] (M_e); cr_e overwrites xh[2e].
template <int N, typename R, bool EFAST>
__global__ void __launch_bounds__(KT * FftShape<N>::T, (N <= 512 ? DB_LB_ZPASS : 1))
    k_zpass_rhs(State s, Geom g, Phys ph, int rk, const double2* __restrict__ ghost) {
  // FP32 work type: write the increment cr - base (base = the state as the
  // inverse transforms saw it), so FP32 rounding scales with the substep's
  // change, not with the field
  constexpr bool INC = sizeof(R) == sizeof(float);
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  // column-fastest mapping: a warp reads KT consecutive kx of 32/KT rows
  const int seq = threadIdx.x % KT, lane = threadIdx.x / KT;
  // EFAST: equation fastest in the grid, so the four CTAs of one column
  // block share their spectral reads (cu, cp, cth) through L2 (faster for
  // the FP64 work type; the FP32 one runs faster with the equation slowest).
  // A compile-time choice: a run-time one cost the FP32 kernel 40%.
  const int j = EFAST ? blockIdx.z : blockIdx.y;
  const int kx = (EFAST ? blockIdx.y : blockIdx.x) * KT + seq;
  const bool active = kx < g.kxs;
  const int kxc = active ? kx : 0;
  // per-column buffers, staggered by one element so the KT columns sharing a
  // warp fall into different shared-memory bank groups
  C* sx = sm + seq * (3 * padded(N) + 1);  // exchange buffers (two)
  C* sx1 = sx + padded(N);
  C* sm_z = sx1 + padded(N);             // Z(M) stash, natural order
#if DB_ZPASS_LAZY
#define ZFFT(SIGN_, V_) fft_reg_lazy<N, SIGN_, true>(V_, lane, active, sx, tw_z<R>(g), sx1)
#else
  Twiddles<N, E, C> twd;
  load_twiddles<N, E>(twd, lane, tw_z<R>(g));
#define ZFFT(SIGN_, V_) fft_reg<N, SIGN_, true>(V_, lane, active, sx, twd, sx1)
#endif
  const double inz = 1.0 / (double)N;
  const long long h0 = (long long)j * g.hp + kxc;
  {
    const int e = EFAST ? blockIdx.x : blockIdx.z;
    const int jlo = (e == 2) ? 2 : (e == 3 ? g.jstart_th : g.jstart);
    const int jhi = (e == 2) ? g.ny : (e == 3 ? g.jend_th : g.jend);
    C* xin_n = (C*)s.xh[2 * e];
    const C* xin_m = (const C*)s.xh[2 * e + 1];
    if (!in_rng(j, jlo, jhi)) {
      if (active)
#pragma unroll
        for (int q = 0; q < E; ++q) xin_n[h0 + (long long)(lane + q * T) * g.kxs] = mkc<C>(0, 0);
      return;
    }
    C vn[E];
    // Z(M) first, parked in shared memory in natural order
#pragma unroll
    for (int q = 0; q < E; ++q)
      vn[q] = active ? __ldg(xin_m + h0 + (long long)(lane + q * T) * g.kxs) : mkc<C>(0, 0);
    ZFFT(-1, vn);
#pragma unroll
    for (int q = 0; q < E; ++q) sm_z[pidx(lane + q * T)] = vn[q];
#pragma unroll
    for (int q = 0; q < E; ++q)
      vn[q] = active ? xin_n[h0 + (long long)(lane + q * T) * g.kxs] : mkc<C>(0, 0);
    __syncthreads();
    ZFFT(-1, vn);
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int zz = lane + q * T;
      const int kzp = (zz <= g.nkz) ? zz : (zz >= N - g.nkz ? zz - N + g.nkzp : -1);
      if (kzp < 0 || !active) {
        vn[q] = mkc<C>(0, 0);
        continue;
      }
      const double kzv = g.kz[kzp];
      // NL = (Z(N) + i kz Z(M)) / Nz, formed in FP64
      const double2 zmq = to_d2(sm_z[pidx(zz)]), zn = to_d2(vn[q]);
      const double2 nl = make_double2((zn.x - kzv * zmq.y) * inz, (zn.y + kzv * zmq.x) * inz);
      double2 cr = rhs_point<INC>(s, g, ph, rk, e, j, kxc, kzp, nl, ghost);
      vn[q] = from_d2<C>(cr);
    }
    __syncthreads();
    ZFFT(+1, vn);
    if (active)
#pragma unroll
      for (int q = 0; q < E; ++q) xin_n[h0 + (long long)(lane + q * T) * g.kxs] = vn[q];
  }
}

// ---------------------------------------------------------------------------
// The same z-pass as three lean stages (the FP64 path; the fused kernel keeps
// 128 registers only by spilling there):
//  forward z-FFT of the eight x-half product fields (k_fwd_z) into spectral
//               scratch: Z(N_e)/Nz in nls[e], Z(M_e)/Nz in nls[4 + e]
//  k_rhs_modes: NL_e = Z(N_e) + i kz Z(M_e) and the spectral RHS mode by mode
//               (rhs_point), cr_e over nls[e] in place, zero on the planes
//               the equation does not solve
//  inverse z-FFT of cr_e into xh[2e] (k_inv_z)
__global__ void __launch_bounds__(256) k_rhs_modes(const __grid_constant__ State s, Geom g, Phys ph, int rk,
                                                   const __grid_constant__ FieldSet nl) {
  // equation fastest in the grid: the four CTAs of one block of modes run
  // together and share the state reads (cu1, cu2, cu3, cth, cp) through L2
  const int m = blockIdx.y * blockDim.x + threadIdx.x;
  const int j = blockIdx.z, e = blockIdx.x;
  if (m >= g.nkzp * g.kxs) return;
  const int kzp = m / g.kxs, kx = m % g.kxs;
  const long long a = (long long)j * g.sp + m;
  double2* p = (double2*)nl.p[e] + a;
  const int jlo = (e == 2) ? 2 : (e == 3 ? g.jstart_th : g.jstart);
  const int jhi = (e == 2) ? g.ny : (e == 3 ? g.jend_th : g.jend);
  if (!in_rng(j, jlo, jhi)) {
    *p = make_double2(0.0, 0.0);
    return;
  }
  const double kzv = g.kz[kzp];
  const double2 zn = *p, zm = ((const double2*)nl.p[4 + e])[a];
  const double2 nlv = make_double2(zn.x - kzv * zm.y, zn.y + kzv * zm.x);
  *p = rhs_point<false>(s, g, ph, rk, e, j, kx, kzp, nlv, nullptr);
}

// ---------------------------------------------------------------------------
// implicit systems: rows of the four equations (th, u2, u1, u3) -> tri[eq*np + j].
// One CTA per equation: rows are filled in parallel in shared memory, the BC
// rows and the forward elimination (a serial recurrence) by one thread.
// B: member-batched (blockIdx.y = member)
template <bool B = false>
__global__ void __launch_bounds__(256) k_tri_coef(Geom g0, Phys ph0, TriRow* tri0, DevScalars* sc0, int rk,
                                                  const MemberArgs* __restrict__ tab) {
  const int mb = B ? (int)blockIdx.y : 0;
  const Geom& g = g0;   // the same geometry for every member
  const Phys& ph = B ? tab[mb].ph : ph0;
  TriRow* tri = B ? tab[mb].s.tri : tri0;
  DevScalars* sc = B ? tab[mb].s.sc : sc0;
  extern __shared__ TriRow Rs[];
  const int eq = blockIdx.x;  // 0..3
  const int np = g.np, Nyp = g.ny;
  const double temp1 = 0.5 * ph.nu * sc->h_bar[rk];
  const double tv = temp1 * ph.nu_v_scale;
  const double tth = temp1 / ph.pr * ph.nu_v_scale;
  const double* dy = g.dy;
  const double* dyf = g.dyf;
  const int lo = (eq == 0) ? g.jstart_th : (eq == 1 ? 2 : g.jstart);
  const int hi = (eq == 0) ? g.jend_th : (eq == 1 ? Nyp : g.jend);
  for (int j = threadIdx.x; j < np; j += blockDim.x) {
    TriRow r;
    r.l = 0.0; r.d = 1.0; r.u = 0.0; r.bc = 0.0; r.ap = 0.0; r.ibp = 1.0;
    r.cn_lo = 0.0; r.cn_hi = 0.0; r.ef_lo = 0.0; r.ef_hi = 0.0;
    r.is_bc = 1; r.interior = 0;
    if (j >= lo && j <= hi) {
      if (eq == 0) {  // solver.f90:1023-1026
        r.l = -(tth) / (dy[j] * dyf[j]);
        r.d = 1. + (tth) / (dy[j + 1] * dyf[j]) + (tth) / (dy[j] * dyf[j]);
        r.u = -(tth) / (dy[j + 1] * dyf[j]);
        r.cn_hi = (tth) / dyf[j] / dy[j + 1];
        r.cn_lo = (tth) / dyf[j] / dy[j];
        r.ef_lo = 1.0 / (dy[j] * dyf[j]);
        r.ef_hi = 1.0 / (dy[j + 1] * dyf[j]);
      } else if (eq == 1) {  // solver.f90:1085-1088
        r.l = -tv / (dyf[j - 1] * dy[j]);
        r.d = 1. + tv / (dyf[j] * dy[j]) + tv / (dyf[j - 1] * dy[j]);
        r.u = -tv / (dyf[j] * dy[j]);
        r.cn_hi = tv / dy[j] / dyf[j];
        r.cn_lo = tv / dy[j] / dyf[j - 1];
        r.ef_lo = 0.5 / (dyf[j - 1] * dy[j]);   // times nu(j) + nu(j-1)
        r.ef_hi = 0.5 / (dyf[j] * dy[j]);       // times nu(j) + nu(j+1)
      } else {        // solver.f90:1140-1143, 1196-1199
        r.l = -tv / (dy[j] * dyf[j]);
        r.d = 1. - tv * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]));
        r.u = -tv / (dy[j + 1] * dyf[j]);
        r.cn_hi = tv / dyf[j] / dy[j + 1];
        r.cn_lo = tv / dyf[j] / dy[j];
        r.ef_lo = 1.0 / (dy[j] * dyf[j]);
        r.ef_hi = 1.0 / (dy[j + 1] * dyf[j]);
      }
      r.is_bc = 0;
      r.interior = 1;
    }
    Rs[j] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    auto setr = [&](int j, double l, double d, double u, double v) {
      Rs[j].l = l; Rs[j].d = d; Rs[j].u = u; Rs[j].bc = v; Rs[j].is_bc = 1; Rs[j].interior = 0;
    };
    if (eq != 1) {
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
    } else {  // apply_BC_2_* (solver.f90:1987-2061)
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
    double bprev = Rs[0].d;
    Rs[0].ap = 0.0;
    Rs[0].ibp = 1.0 / bprev;
    double uprev = Rs[0].u;
    for (int j = 1; j < np; ++j) {
      const double a = -Rs[j].l / bprev;
      const double b = Rs[j].d + a * uprev;
      Rs[j].ap = a;
      Rs[j].ibp = 1.0 / b;
      bprev = b;
      uprev = Rs[j].u;
    }
  }
  __syncthreads();
  TriRow* R = tri + eq * np;
  for (int j = threadIdx.x; j < np; j += blockDim.x) R[j] = Rs[j];
}

// ---------------------------------------------------------------------------
// The CN solves of the substep without LES in spectral space.  Without eddy
// viscosity the four implicit systems (solver.f90:1012-1233) have the same
// matrix in every (x, z) column, and their right-hand side (r plus the
// explicit CN term, solver.f90:850-870, 981-989) is linear in the state,
// so solving every physical column and transforming the result to Fourier
// space (solver.f90:1247-1252) equals solving every retained Fourier mode's
// column: the BC rows carry their constant value in the (0,0) mode and zero
// in every other mode.  The inverse x/z transforms of cr, the physical
// solve and the forward transforms of the new state drop out, and the
// solve runs in FP64 on both work types.  Real and imaginary parts of a
// mode are two real columns of the same real system, with the LU factors
// k_tri_coef shares.
//
// k_rhs_cn: one thread per retained mode walks the planes upward and runs
// the four equations (z-pass order 0 u1, 1 u3, 2 u2, 3 th) together,
// joining the spectral RHS with the forward sweep: NL from the z-pass (or
// its Z(N), Z(M) parts, SPLITZ), cr and cf (stored) by rhs_eval, the
// explicit CN term from
// the old state planes j-1..j+1 and y_j = v_j + a'_j y_{j-1}; y_j
// overwrites NL of plane j.  The planes j-1, j, j+1 of cu1, cu3, cu2, cth
// (the CN explicit terms and the cross terms of the RHS) and cp of planes
// j-1, j stay in registers as the walk moves up, so each state plane is
// loaded once for all four equations (13 loads per plane and mode, 17 with
// SPLITZ), and
// the state is only read (cf apart).  Every mode's thread is resident at
// once (a second wave would walk all planes again with few threads).
// B: member-batched (blockIdx.y = member)
template <bool SPLITZ, bool B = false>
__global__ void __launch_bounds__(32, DB_RHSCN_LB) k_rhs_cn(const __grid_constant__ State s0, Geom g0, Phys ph0, int rk,
                                                            const __grid_constant__ FieldSet nl0,
                                                            const MemberArgs* __restrict__ tab) {
  const int mb = B ? (int)blockIdx.y : 0;
  const State& s = B ? tab[mb].s : s0;
  const Geom& g = g0;   // the same geometry for every member
  const Phys& ph = B ? tab[mb].ph : ph0;
  const FieldSet& nl = B ? tab[mb].fs[FS_NL] : nl0;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= g.sp) return;
  const int np = g.np;
  const long long sp = g.sp;
  const int kzp = m / g.kxs, kx = m % g.kxs;
  const RhsK kc = rhs_consts(s, g, ph, rk, kx, kzp);
  const bool m0 = (m == 0);   // the (0,0) mode carries the BC constants
  // z-pass order 0 u1, 1 u3, 2 u2, 3 th; k_tri_coef order th, u2, u1, u3
  const double2* const U[4] = {s.cu1 + m, s.cu3 + m, s.cu2 + m, s.cth + m};
  const int lo[4] = {g.jstart, g.jstart, 2, g.jstart_th};
  const int hi[4] = {g.jend, g.jend, g.ny, g.jend_th};
  const TriRow* const Rw[4] = {s.tri + 2 * np, s.tri + 3 * np, s.tri + np, s.tri};
  double2 um[4], uc[4], y[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    um[e] = make_double2(0.0, 0.0);
    uc[e] = U[e][0];
    y[e] = make_double2(0.0, 0.0);
  }
  double2 pm = make_double2(0.0, 0.0);   // cp of plane j-1
  for (int j = 0; j < np; ++j) {
    const long long a = (long long)j * sp;
    // the next plane's inputs into L2 while this plane is computed (the
    // stores of y below keep the compiler from hoisting those loads, so
    // without this every plane waits for DRAM)
    if (j + 1 < np) {
      const long long an = a + sp;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (j + 2 < np) prefetch_l2(U[e] + an + sp);
        prefetch_l2((const double2*)nl.p[e] + an + m);
        if (SPLITZ) prefetch_l2((const double2*)nl.p[4 + e] + an + m);
        if (rk > 0) prefetch_l2(rhs_cf(s, e) + an + m);
      }
      prefetch_l2(s.cp + an + m);
    }
    double2 un[4], nlv[4], zmv[4], cfo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const bool rr = in_rng(j, lo[e], hi[e]);
      un[e] = (j + 1 < np) ? U[e][a + sp] : make_double2(0.0, 0.0);
      nlv[e] = rr ? ((const double2*)nl.p[e])[a + m] : make_double2(0.0, 0.0);
      if (SPLITZ) zmv[e] = rr ? ((const double2*)nl.p[4 + e])[a + m] : make_double2(0.0, 0.0);
      cfo[e] = (rr && rk > 0) ? rhs_cf(s, e)[a + m] : make_double2(0.0, 0.0);
    }
    const double2 cpj = s.cp[a + m];
    if (SPLITZ) {   // NL = Z(N) + i kz Z(M), both already scaled by 1/Nz
#pragma unroll
      for (int e = 0; e < 4; ++e)
        nlv[e] = make_double2(nlv[e].x - kc.kzv * zmv[e].y, nlv[e].y + kc.kzv * zmv[e].x);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const TriRow* row = Rw[e] + j;
      double2 cr = make_double2(0.0, 0.0);
      if (in_rng(j, lo[e], hi[e])) {
        RhsIn v;
        v.own = uc[e];
        v.cu1 = uc[0];
        v.cu3 = uc[1];
        v.cth = uc[3];
        v.cp = cpj;
        v.nb2 = (e == 2) ? um[3] : uc[2];   // u2: cth of plane j-1; u1, u3: cu2 of plane j
        v.nbp = (e == 2) ? pm : un[2];      // u2: cp of plane j-1;  u1, u3: cu2 of plane j+1
        v.cfo = cfo[e];
        double2 cf;
        cr = rhs_eval<false>(s, g, ph, rk, e, j, kx, kzp, nlv[e], v, kc, cf);
        rhs_cf(s, e)[a + m] = cf;
      }
      double2 w;
      if (row->is_bc) {
        w = make_double2(m0 ? row->bc : 0.0, 0.0);
      } else {
        w.x = cr.x + (row->cn_hi * (un[e].x - uc[e].x) - row->cn_lo * (uc[e].x - um[e].x));
        w.y = cr.y + (row->cn_hi * (un[e].y - uc[e].y) - row->cn_lo * (uc[e].y - um[e].y));
      }
      if (j == 0) {
        y[e] = w;
      } else {
        y[e].x = w.x + row->ap * y[e].x;
        y[e].y = w.y + row->ap * y[e].y;
      }
      ((double2*)nl.p[e])[a + m] = y[e];
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      um[e] = uc[e];
      uc[e] = un[e];
    }
    pm = cpj;
  }
}

// k_cn_back: back substitution per real column (2 sp doubles per plane)
// and equation (blockIdx.y, k_tri_coef order th, u2, u1, u3) from the y
// values k_rhs_cn left in the scratch, batches of TB planes loaded first;
// the new state is written on the planes the reference's solve stores,
// the others keep their values.  A non-finite new state is reported as
// DB_FLAG_NONFINITE.
// B: member-batched (blockIdx.z = member)
template <bool B = false>
__global__ void __launch_bounds__(128) k_cn_back(const __grid_constant__ State s0, Geom g0,
                                                 const __grid_constant__ FieldSet nl0, const MemberArgs* __restrict__ tab) {
  const int mb = B ? (int)blockIdx.z : 0;
  const State& s = B ? tab[mb].s : s0;
  const Geom& g = g0;   // the same geometry for every member
  const FieldSet& nl = B ? tab[mb].fs[FS_NL] : nl0;
  constexpr int TB = 8;
  const long long ncol = 2 * g.sp;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int eq = blockIdx.y;
  if (c >= ncol) return;
  const int np = g.np, Nyp = g.ny;
  const long long pp = ncol;
  const TriRow* Rw = s.tri + eq * np;
  const int ze = (eq == 0) ? 3 : (eq == 1 ? 2 : (eq == 2 ? 0 : 1));
  double* u = (double*)((eq == 0) ? s.cth : (eq == 1 ? s.cu2 : (eq == 2 ? s.cu1 : s.cu3))) + c;
  const double* yv = (const double*)nl.p[ze] + c;
  const int lo = (eq == 0) ? g.jstart_th - 1 : (eq == 1 ? 1 : g.jstart - 1);
  const int hi = (eq == 0) ? g.jend_th + 1 : (eq == 1 ? Nyp + 1 : g.jend + 1);
  double xn = 0.0;
  bool bad = false;
  for (int jt = np - 1; jt >= 0; jt -= TB) {
    double xg[TB];
#pragma unroll
    for (int q = 0; q < TB; ++q) {
      const int j = jt - q;
      xg[q] = (j >= 0) ? yv[(long long)j * pp] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < TB; ++q) {
      const int j = jt - q;
      if (j < 0) break;
      const double ib = Rw[j].ibp;
      const double xv = (j == np - 1) ? xg[q] * ib : xg[q] * ib - Rw[j].u * ib * xn;
      xn = xv;
      bad = bad || !(fabs(xv) <= 1.7976931348623157e308);
      if (j >= lo && j <= hi) u[(long long)j * pp] = xv;
    }
  }
  if (bad) atomicOr(B ? tab[mb].g.flags : g.flags, DB_FLAG_NONFINITE);
}
// ---------------------------------------------------------------------------
// rem_div factors: per (kx, kzp) column, rows 1..Nyp of the Poisson system
// (solver.f90:1326-1333 with apply_BC_rem_div_mpi 2341-2368), forward
// eliminated once: a'_j and 1/b'_j as two planes-by-modes arrays in the
// pfac buffer (the forward sweep reads only a', the backward only 1/b').
__device__ __forceinline__ double* pfac_a(const State& s, const Geom&) { return (double*)s.pfac; }
__device__ __forceinline__ double* pfac_ib(const State& s, const Geom& g) {
  return (double*)s.pfac + (long long)g.np * g.sp;
}
__global__ void k_pfac(Geom g, double2* pfac2) {
  double* pa = (double*)pfac2;
  double* pib = pa + (long long)g.np * g.sp;
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
  pa[(long long)1 * g.sp + (long long)kzp * g.kxs + kx] = 0.0;
  pib[(long long)1 * g.sp + (long long)kzp * g.kxs + kx] = 1.0 / dp;
  for (int j = 2; j <= Nyp; ++j) {
    row(j, l, d, u);
    const double a = -l / bprev;
    const double b = d + a * up;
    pa[(long long)j * g.sp + (long long)kzp * g.kxs + kx] = a;
    pib[(long long)j * g.sp + (long long)kzp * g.kxs + kx] = 1.0 / b;
    bprev = b;
    up = u;
  }
}

// divergence removal + pressure update (solver.f90:1302-1379, 1261-1267).
// The Poisson matrix of a (kx, kzp) column is real, so the real and the
// imaginary part of phi are two independent real systems: one thread per
// column and part (part = threadIdx.x & 1, the pair in adjacent lanes, so a
// warp reads 16 consecutive modes).  Part 0 (phi real) sees the divergence
// -kx Im u1 + Dy Re u2 - kz Im u3 and corrects Im u1, Im u3, Re u2, Re cp;
// part 1 the other halves, so the two threads never touch the same value.
// The rows of both sweeps are handled in batches of RB whose loads are all
// issued first (each thread keeps several rows in flight).  Large planes:
// RB 3 at 72 registers, seven CTAs per SM, so the 131 k threads of a
// 512x512 plane fit one wave (at six, a partial second wave walked every row
// again); small planes, whose threads fit a wave anyway: RB 4 (more rows in
// flight per thread), six CTAs per SM.  B: member-batched (blockIdx.z =
// member).
template <int RB, int LB, bool B = false>
__global__ void __launch_bounds__(128, LB) k_rem_div(const __grid_constant__ State s0, Geom g0, int rk, int update_cp,
                                                      const MemberArgs* __restrict__ tab) {
  const int mb = B ? (int)blockIdx.z : 0;
  const State& s = B ? tab[mb].s : s0;
  const Geom& g = g0;   // the same geometry for every member
  const int t = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  const int kx = t >> 1, part = t & 1;
  if (kx > g.nkx) return;
  const int Nyp = g.ny;
  const long long c0 = (long long)kzp * g.kxs + kx, sp = g.sp;
  const long long q0 = 2 * c0 + part, qs = 2 * sp;   // this part, as doubles
  const double* u1 = reinterpret_cast<const double*>(s.cu1);
  const double* u3 = reinterpret_cast<const double*>(s.cu3);
  double* w1p = reinterpret_cast<double*>(s.cu1);
  double* w3p = reinterpret_cast<double*>(s.cu3);
  double* u2 = reinterpret_cast<double*>(s.cu2);
  double* cpp = reinterpret_cast<double*>(s.cp);
  double* ph = reinterpret_cast<double*>(s.phi_g);
  const double* pfa = pfac_a(s, g);
  const double* pfb = pfac_ib(s, g);
  // d/dx, d/dz of the other part: Re(i k a) = -k Im a, Im(i k a) = k Re a
  const long long qo = 2 * c0 + (part ^ 1);
  const double sgn = part ? 1.0 : -1.0;
  const double kxv = sgn * g.kx[kx], kzv = sgn * g.kz[kzp];
  const bool zero_mode = (kx == 0 && kzp == 0);
  // forward sweep: g_1 = 0 (BC row), g_j = rhs_j + a'_j g_{j-1}; rhs_Nyp = 0
  double gp = 0.0;
  ph[1 * qs + q0] = gp;
  double u2c = u2[2 * qs + q0];
  for (int jb = 2; jb <= Nyp; jb += RB) {
    double pa[RB], u2n[RB], a1[RB], a3[RB];
#pragma unroll
    for (int c = 0; c < RB; ++c) {
      const int j = jb + c;
      const bool in = j <= Nyp, mid = j < Nyp;
      pa[c] = in ? pfa[(long long)j * sp + c0] : 0.0;
      u2n[c] = in ? u2[(long long)(j + 1) * qs + q0] : 0.0;
      a1[c] = mid ? u1[(long long)j * qs + qo] : 0.0;
      a3[c] = mid ? u3[(long long)j * qs + qo] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < RB; ++c) {
      const int j = jb + c;
      if (j > Nyp) break;
      const double rhs = (j < Nyp) ? kxv * a1[c] + (u2n[c] - u2c) / g.dyf[j] + kzv * a3[c] : 0.0;
      gp = rhs + pa[c] * gp;
      ph[(long long)j * qs + q0] = gp;
      u2c = u2n[c];
    }
  }
  // backward sweep with the projection (solver.f90:1361-1376) and cp update:
  // u1 -= i kx phi, u3 -= i kz phi touch the other part of u1, u3 (sign as
  // above with phi in place of a)
  const double itemp4 = 1.0 / s.sc->h_bar[rk];
  double phin = 0.0;
  for (int jt = Nyp; jt >= 1; jt -= RB) {
    double ib[RB], gj[RB], v1[RB], v3[RB], v2[RB], pc[RB];
#pragma unroll
    for (int c = 0; c < RB; ++c) {
      const int j = jt - c;
      const bool in = j >= 1;
      const long long a = (long long)j * qs;
      ib[c] = in ? pfb[(long long)j * sp + c0] : 0.0;
      gj[c] = in ? ph[a + q0] : 0.0;
      v1[c] = in ? u1[a + qo] : 0.0;
      v3[c] = in ? u3[a + qo] : 0.0;
      v2[c] = (in && j + 1 <= Nyp) ? u2[a + qs + q0] : 0.0;
      pc[c] = (in && update_cp && j >= g.jstart && j <= g.jend) ? cpp[a + q0] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < RB; ++c) {
      const int j = jt - c;
      if (j < 1) break;
      double cj;
      if (j == Nyp) cj = 0.0;
      else if (j == 1) cj = zero_mode ? 0.0 : -1.0;
      else cj = 1.0 / (g.dy[j + 1] * g.dyf[j]);
      const double phi = (j == Nyp) ? gj[c] * ib[c] : (gj[c] - cj * phin) * ib[c];
      const long long a = (long long)j * qs;
      w1p[a + qo] = v1[c] + kxv * phi;   // (u1 - i kx phi) in the other part
      w3p[a + qo] = v3[c] + kzv * phi;
      if (j + 1 <= Nyp) u2[a + qs + q0] = v2[c] - (phin - phi) / g.dy[j + 1];   // u2(j+1) -= Dy phi
      if (update_cp && j >= g.jstart && j <= g.jend) cpp[a + q0] = pc[c] + phi * itemp4;
      phin = phi;
    }
  }
}

// ---------------------------------------------------------------------------
// courant: CFL minimum over the physical velocity (flow.f90:781-808)
__device__ __forceinline__ unsigned long long dbits(double v) { return (unsigned long long)__double_as_longlong(v); }

template <typename R>
__global__ void __launch_bounds__(256) k_courant_reduce(const __grid_constant__ State s, Geom g, Phys ph, CflCtl ctl) {
  DevScalars* sc = s.sc;
  const R* U1 = (const R*)s.u1;
  const R* U2 = (const R*)s.u2;
  const R* U3 = (const R*)s.u3;
  if (!ctl.force && !(ctl.variable_dt && (sc->time_step % ctl.update_dt) == 0)) return;
  const long long n = (long long)g.pp;
  const int jlo = ph.front ? g.jstart : 1, jhi = ph.front ? g.jend : g.ny;
  const double f = ph.ro_inv / ph.delta;
  // min over points of CFL dx / |u1 - U| etc. = CFL / max of |u1 - U| / dx
  // etc.: a running maximum per thread, one division per CTA
  const double idx_ = 1.0 / ph.dx, idz_ = 1.0 / ph.dz;
  double amax = 0.0;
  bool bad = false;
  for (int j = jlo + (int)blockIdx.y; j <= jhi; j += gridDim.y) {   // per-row constants once per row
    const double c1 = ph.front ? ph.dthdz * g.gyf[j] / f : 0.0;
    const double c3 = ph.front ? (1.0 / f) * ph.dthdx * (g.gyf[j] - 0.5 * ph.ly) : 0.0;
    const double idy = 1.0 / g.dy[j];
    const R* u1r = U1 + (long long)j * n;
    const R* u2r = U2 + (long long)j * n;
    const R* u3r = U3 + (long long)j * n;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
      const double v1 = (double)u1r[p], v2 = (double)u2r[p], v3 = (double)u3r[p];
      const double a = fmax(fabs(v1 - c1) * idx_, fmax(fabs(v2) * idy, fabs(v3 + c3) * idz_));
      bad = bad || !(a <= 1.7976931348623157e308);   // a non-finite velocity
      amax = fmax(amax, a);
    }
  }
  if (bad) atomicOr(&sc->flags, 1);
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) amax = fmax(amax, red[w]);
    if (amax > 0.0) atomicMin(&sc->dt_min_bits, dbits(ctl.cfl / amax));
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
// the same for every member of a batch (end = 0: begin)
__global__ void k_steps_batch(const MemberArgs* __restrict__ tab, int n, int end) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DevScalars* sc = tab[i].s.sc;
  if (end) sc->time += sc->delta_t;
  else sc->time_step += 1;
}

// max |div| at GYF rows 2..Nyp-1 (the rows rem_div zeroes)
__global__ void k_divergence(const __grid_constant__ State s, Geom g) {
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
__global__ void k_bc_vel_post(const __grid_constant__ State s, Geom g, Phys ph) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzp = blockIdx.y;
  if (kx > g.nkx) return;
  const long long c0 = (long long)kzp * g.kxs + kx;
  GhostCol a, b, c;
  load_col(a, s.cu1 + c0, g.sp, g.ny);
  load_col(b, s.cu2 + c0, g.sp, g.ny);
  load_col(c, s.cu3 + c0, g.sp, g.ny);
  bc_vel_post(a, b, c, g, ph, kx == 0 && kzp == 0, s.sc->time);
  store_ghosts(a, s.cu1 + c0, g.sp, g.ny);
  store_ghosts(b, s.cu2 + c0, g.sp, g.ny);
  store_ghosts(c, s.cu3 + c0, g.sp, g.ny);
}

// ---------------------------------------------------------------------------
// launchers

template <int N, typename R>
static void go_products_t(const Geom& g, const State& s, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  if constexpr (N <= 512) {
    const int zr = prod_zr<N>() < g.nz ? prod_zr<N>() : g.nz;
    constexpr int PROD_SLOTS = prod_slots<R>();
    const size_t smem = (size_t)PROD_SLOTS * 4 * zr * N * sizeof(R) + (size_t)3 * zr * prod_sq<N>() * sizeof(C) +
                        PROD_SLOTS * sizeof(uint64_t);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_products_st<N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nzb = g.nz / zr;
    const int gmax = (g.tune_pgrid > 0 ? g.tune_pgrid : 2) * sm_count();
    // plane ranges: about four items per CTA, at least four planes each
    int nch = (4 * gmax + nzb - 1) / nzb;
    nch = nch < 1 ? 1 : (nch > g.np / 4 ? (g.np / 4 > 0 ? g.np / 4 : 1) : nch);
    const int jlen = (g.np + nch - 1) / nch;
    nch = (g.np + jlen - 1) / jlen;
    const int nitems = nzb * nch;
    const int grid = nitems < gmax ? nitems : gmax;
    k_products_st<N, R><<<grid, 3 * FftShape<N>::T * zr, smem, st>>>(s, g, zr, nzb, jlen, nitems, nullptr);
  } else {
    const size_t smem = (size_t)3 * padded(N) * sizeof(C);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_products<N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_products<N, R><<<dim3(g.nz, g.np, 2), 3 * FftShape<N>::T, smem, st>>>(s, g);
  }
}
template <int N, typename R>
static void go_products_les_t(const Geom& g, const State& s, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int zr = prod_zr<N>() < g.nz ? prod_zr<N>() : g.nz;
  const size_t smem = (size_t)3 * zr * padded(N) * sizeof(C);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_products_les<N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_products_les<N, R><<<dim3(g.nz / zr, g.np, 2), 3 * FftShape<N>::T * zr, smem, st>>>(s, g, zr);
}
template <int N>
static void go_products(const Geom& g, const State& s, cudaStream_t st, bool les) {
  if (les) {
    if (g.prec) go_products_les_t<N, float>(g, s, st); else go_products_les_t<N, double>(g, s, st);
  } else {
    if (g.prec) go_products_t<N, float>(g, s, st); else go_products_t<N, double>(g, s, st);
  }
}
template <int N, typename R>
static void go_zpass_t(const Geom& g, const Phys& ph, const State& s, int rk, const double2* ghost, cudaStream_t st) {
  constexpr int T = FftShape<N>::T;
  constexpr bool EFAST = sizeof(R) == sizeof(double);
  size_t smem = (size_t)KT * (3 * padded(N) + 1) * sizeof(typename CplxOf<R>::type);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_zpass_rhs<N, R, EFAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const dim3 grid = EFAST ? dim3(4, g.kxs / KT, g.np) : dim3(g.kxs / KT, g.np, 4);
  k_zpass_rhs<N, R, EFAST><<<grid, KT * T, smem, st>>>(s, g, ph, rk, ghost);
}
template <int N>
static void go_zpass_split(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st) {
  const FieldSet nl = fset(s.nls[0], s.nls[1], s.nls[2], s.nls[3], s.nls[4], s.nls[5], s.nls[6], s.nls[7]);
  launch_fwd_z(g, fset(s.xh[0], s.xh[2], s.xh[4], s.xh[6], s.xh[1], s.xh[3], s.xh[5], s.xh[7]), nl, 8, st);
  k_rhs_modes<<<dim3(4, (g.nkzp * g.kxs + 255) / 256, g.np), 256, 0, st>>>(s, g, ph, rk, nl);
  launch_inv_z(g, nl, fset(s.xh[0], s.xh[2], s.xh[4], s.xh[6]), 4, st);
}
template <int N>
static void go_zpass(const Geom& g, const Phys& ph, const State& s, int rk, const double2* ghost, cudaStream_t st) {
  // FP32: one fused kernel; FP64: the three stages (the fused FP64 kernel
  // spills at 128 registers), over the spectral scratch db_init allocates
  if (g.prec) go_zpass_t<N, float>(g, ph, s, rk, ghost, st);
  else go_zpass_split<N>(g, ph, s, rk, st);
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

cudaError_t launch_products(const Geom& g, const State& s, cudaStream_t st, bool les) {
  DB_DISPATCH_N2(g.nx, go_products, g, s, st, les);
  return cudaGetLastError();
}
cudaError_t launch_zpass_rhs(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st,
                             const double2* ghost) {
  if (!g.prec && !s.nls[0]) return cudaErrorInvalidValue;
  DB_DISPATCH_N2(g.nz, go_zpass, g, ph, s, rk, ghost, st);
  return cudaGetLastError();
}
// without LES: the nonlinear terms into spectral scratch, then the spectral
// RHS with the CN solves.  FP64 fields: Z(N_e) / Nz into s.crs[e] and
// Z(M_e) / Nz into s.nls[4 + e] (k_fwd_z, 4-column CTAs), combined in
// k_rhs_cn; FP32 fields: NL_e into s.crs[e] (k_fwd_z_nl).
cudaError_t launch_zpass_spec(const Geom& g, const State& s, cudaStream_t st) {
  if (!s.crs[0] || (!g.prec && !s.nls[4])) return cudaErrorInvalidValue;
  if (!g.prec)
    return launch_fwd_z(g, fset(s.xh[0], s.xh[2], s.xh[4], s.xh[6], s.xh[1], s.xh[3], s.xh[5], s.xh[7]),
                        fset(s.crs[0], s.crs[1], s.crs[2], s.crs[3], s.nls[4], s.nls[5], s.nls[6], s.nls[7]), 8, st);
  return launch_fwd_z_nl(g, fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[4], s.xh[5], s.xh[6], s.xh[7]),
                         fset(s.crs[0], s.crs[1], s.crs[2], s.crs[3]), st);
}
cudaError_t launch_rhs_cn(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st) {
  const FieldSet nl = fset(s.crs[0], s.crs[1], s.crs[2], s.crs[3], s.nls[4], s.nls[5], s.nls[6], s.nls[7]);
  if (!g.prec) k_rhs_cn<true><<<(unsigned)((g.sp + 31) / 32), 32, 0, st>>>(s, g, ph, rk, nl, nullptr);
  else k_rhs_cn<false><<<(unsigned)((g.sp + 31) / 32), 32, 0, st>>>(s, g, ph, rk, nl, nullptr);
  k_cn_back<><<<dim3((unsigned)((2 * g.sp + 127) / 128), 4), 128, 0, st>>>(s, g, nl, nullptr);
  return cudaGetLastError();
}
cudaError_t launch_tri_coef(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st) {
  const size_t smem = (size_t)g.np * sizeof(TriRow);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_tri_coef<>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_tri_coef<><<<4, 256, smem, st>>>(g, ph, s.tri, s.sc, rk, nullptr);
  return cudaGetLastError();
}
cudaError_t launch_courant(const Geom& g, const Phys& ph, const State& s, CflCtl ctl, cudaStream_t st) {
  const dim3 grid(16, 74);   // x: within a row, y: rows
  if (g.prec) k_courant_reduce<float><<<grid, 256, 0, st>>>(s, g, ph, ctl);
  else k_courant_reduce<double><<<grid, 256, 0, st>>>(s, g, ph, ctl);
  k_courant_final<<<1, 1, 0, st>>>(s.sc, ph, ctl);
  return cudaGetLastError();
}
cudaError_t launch_courant_final(const Phys& ph, const State& s, CflCtl ctl, cudaStream_t st) {
  k_courant_final<<<1, 1, 0, st>>>(s.sc, ph, ctl);
  return cudaGetLastError();
}
cudaError_t launch_rem_div(const Geom& g, const State& s, int rk, int update_cp, cudaStream_t st) {
  const dim3 grid((2 * (g.nkx + 1) + 127) / 128, g.nkzp);
  if ((long long)grid.x * grid.y > 6LL * sm_count()) k_rem_div<3, 7><<<grid, 128, 0, st>>>(s, g, rk, update_cp, nullptr);
  else k_rem_div<4, 6><<<grid, 128, 0, st>>>(s, g, rk, update_cp, nullptr);
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

// ---------------------------------------------------------------------------
// member-batched substep (ensembles without LES at a fixed dt): the kernels
// of the spectral substep above, each launched once for every member

MemberArgs member_args(const Geom& g, const Phys& ph, const State& s) {
  MemberArgs a{};
  a.s = s;
  a.g = g;
  a.ph = ph;
  a.fs[FS_CU4] = fset(s.cu1, s.cu2, s.cu3, s.cth);
  a.fs[FS_XH4] = fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]);
  a.fs[FS_U4] = fset(s.u1, s.u2, s.u3, s.th);
  a.fs[FS_XH8] = fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[4], s.xh[5], s.xh[6], s.xh[7]);
  a.fs[FS_XH8Z] = fset(s.xh[0], s.xh[2], s.xh[4], s.xh[6], s.xh[1], s.xh[3], s.xh[5], s.xh[7]);
  a.fs[FS_NL] = fset(s.crs[0], s.crs[1], s.crs[2], s.crs[3], s.nls[4], s.nls[5], s.nls[6], s.nls[7]);
  return a;
}

// products: one item (a z block over a plane range) per CTA; the plane
// ranges minimise waves x planes walked per item (each range re-reads its
// two neighbouring planes)
template <int N, typename R>
static cudaError_t go_products_bt(const Geom& g, const Batch& bt, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  if constexpr (N <= 512) {
    const int zr = prod_zr<N>() < g.nz ? prod_zr<N>() : g.nz;
    constexpr int PROD_SLOTS = prod_slots<R>();
    const size_t smem = (size_t)PROD_SLOTS * 4 * zr * N * sizeof(R) + (size_t)3 * zr * prod_sq<N>() * sizeof(C) +
                        PROD_SLOTS * sizeof(uint64_t);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_products_st<N, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nzb = g.nz / zr;
    const long long res = (long long)(PROD_SLOTS == 4 ? 2 : 3) * sm_count();
    int best = 1;
    long long bcost = -1;
    for (int nch = 1; nch <= (g.np / 4 > 1 ? g.np / 4 : 1); ++nch) {
      const int jl = (g.np + nch - 1) / nch, nc = (g.np + jl - 1) / jl;
      const long long items = (long long)bt.n * nzb * nc;
      const long long cost = (items + res - 1) / res * (jl + 2);
      if (bcost < 0 || cost < bcost) { bcost = cost; best = nch; }
    }
    const int jlen = (g.np + best - 1) / best, nitems = nzb * ((g.np + jlen - 1) / jlen);
    k_products_st<N, R, true><<<dim3(nitems, bt.n), 3 * FftShape<N>::T * zr, smem, st>>>(State{}, g, zr, nzb, jlen,
                                                                                        nitems, bt.tab);
    return cudaGetLastError();
  } else {
    return cudaErrorInvalidValue;
  }
}
template <int N>
static cudaError_t go_products_b(const Geom& g, const Batch& bt, cudaStream_t st) {
  return g.prec ? go_products_bt<N, float>(g, bt, st) : go_products_bt<N, double>(g, bt, st);
}

cudaError_t launch_steps_batch(const Batch& b, int end, cudaStream_t st) {
  if (!b.tab || b.n < 1) return cudaErrorInvalidValue;
  k_steps_batch<<<(b.n + 127) / 128, 128, 0, st>>>(b.tab, b.n, end);
  return cudaGetLastError();
}

cudaError_t launch_substep_batch(const Geom& g, const Batch& b, int rk, cudaStream_t st, cudaStream_t st_side,
                                 cudaEvent_t ev_fork, cudaEvent_t ev_join) {
  if (!b.tab || b.n < 1 || b.n > 65535 / MAXF || g.nx > 512) return cudaErrorInvalidValue;
  cudaError_t e;
  Batch bt = b;
  // the implicit systems' rows on the side stream, joined before the solves
  if ((e = cudaEventRecord(ev_fork, st))) return e;
  if ((e = cudaStreamWaitEvent(st_side, ev_fork, 0))) return e;
  const size_t tsm = (size_t)g.np * sizeof(TriRow);
  if (tsm > 48 * 1024) cudaFuncSetAttribute(k_tri_coef<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm);
  k_tri_coef<true><<<dim3(4, bt.n), 256, tsm, st_side>>>(g, Phys{}, nullptr, nullptr, rk, bt.tab);
  if ((e = cudaGetLastError())) return e;
  if ((e = cudaEventRecord(ev_join, st_side))) return e;
  // velocity and buoyancy to physical space, products, z-pass of the products
  bt.nf = 4; bt.fin = FS_CU4; bt.fout = FS_XH4;
  if ((e = launch_inv_z_batch(g, bt, st))) return e;
  bt.fin = FS_XH4; bt.fout = FS_U4;
  if ((e = launch_inv_x_batch(g, bt, st))) return e;
  cudaError_t pe = cudaSuccess;
  switch (g.nx) {
    case 16: pe = go_products_b<16>(g, bt, st); break;
    case 32: pe = go_products_b<32>(g, bt, st); break;
    case 64: pe = go_products_b<64>(g, bt, st); break;
    case 128: pe = go_products_b<128>(g, bt, st); break;
    case 256: pe = go_products_b<256>(g, bt, st); break;
    case 512: pe = go_products_b<512>(g, bt, st); break;
    default: return cudaErrorInvalidValue;
  }
  if (pe) return pe;
  if (g.prec) {
    bt.nf = 4; bt.fin = FS_XH8; bt.fout = FS_NL;
    if ((e = launch_fwd_z_nl_batch(g, bt, st))) return e;
  } else {
    bt.nf = 8; bt.fin = FS_XH8Z; bt.fout = FS_NL;
    if ((e = launch_fwd_z_batch(g, bt, st))) return e;
  }
  // spectral RHS + CN solves, projection
  if ((e = cudaStreamWaitEvent(st, ev_join, 0))) return e;
  const dim3 gr((unsigned)((g.sp + 31) / 32), bt.n);
  if (!g.prec) k_rhs_cn<true, true><<<gr, 32, 0, st>>>(State{}, g, Phys{}, rk, FieldSet{}, bt.tab);
  else k_rhs_cn<false, true><<<gr, 32, 0, st>>>(State{}, g, Phys{}, rk, FieldSet{}, bt.tab);
  k_cn_back<true><<<dim3((unsigned)((2 * g.sp + 127) / 128), 4, bt.n), 128, 0, st>>>(State{}, g, FieldSet{}, bt.tab);
  const dim3 grd((2 * (g.nkx + 1) + 127) / 128, g.nkzp, bt.n);
  if ((long long)grd.x * grd.y * grd.z > 6LL * sm_count())
    k_rem_div<3, 7, true><<<grd, 128, 0, st>>>(State{}, g, rk, 1, bt.tab);
  else
    k_rem_div<4, 6, true><<<grd, 128, 0, st>>>(State{}, g, rk, 1, bt.tab);
  return cudaGetLastError();
}

}  // namespace db
