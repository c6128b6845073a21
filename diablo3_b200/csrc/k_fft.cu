// k_fft.cu -- batched 2-D xz transforms between the physical, x-half (Xh)
// and packed spectral layouts (db_common.cuh).
//
// fft_xz_to_fourier (for/fft.f90:242-307) = k_fwd_x then k_fwd_z;
// fft_xz_to_physical (for/fft.f90:311-374) = k_inv_z then k_inv_x.
// The MPI transpose of the reference (fft.f90:283, 358) disappears: the
// z-pass reads x-half rows of a plane directly, in tiles of KT kx columns.
//
// x-pass: two real rows a, b go through one complex FFT of z = a + i b;
//   A_m = (Z_m + conj Z_{N-m}) / 2,  B_m = -i (Z_m - conj Z_{N-m}) / 2.
// Inverse: Z_m = A_m + i B_m, Z_{N-m} = conj A_m + i conj B_m, with the
// imaginary parts of the DC and Nyquist modes dropped as FFTW's c2r does and
// modes above Nkx zeroed (the 2/3 de-aliasing, fft.f90:259-261, 366-368).
// All transforms keep their data in registers (fft_reg.cuh).
//
// R is the real type of the physical and x-half fields: double, or float on
// the mixed path, where the spectral state stays FP64 and is converted on
// the z-pass load/store.
#include "../../include/diablo_b200.h"
#include "db_kernels.cuh"
#include "fft_reg.cuh"
#include "umma.cuh"

namespace db {

// k_fwd_z, k_inv_z: planes per CTA (each CTA transforms ZPJ planes in turn,
// the next plane's tile prefetched into L2 while this one is transformed:
// FP64 z-pass 1.64 -> 1.43 ms, inverse 0.86 -> 0.79 ms per substep at
// 512x257x512; the mixed path's k_fwd_z_nl measured slower in this form,
// 1.32 -> 1.44 ms, and keeps one plane per CTA)
constexpr int ZPJ = 2;

// a hint that brings the line holding p into L2 (p must be a valid global
// address)
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(p)));
}

// ---------------------------------------------------------------------------
// Each group of T = N/E threads (one warp for N <= 512) transforms one
// sequence; a CTA holds NS = blockDim / T independent sequences.

// physical -> Xh: sequence = rows (2q, 2q+1) of one plane/field
template <int N, typename R>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_fwd_x(const __grid_constant__ FieldSet in, const __grid_constant__ FieldSet out, Geom g) {
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int q2 = blockIdx.x * (blockDim.x / T) + seq;
  const int j = blockIdx.y, f = blockIdx.z;
  C* sq = sm + seq * padded(N);
  Twiddles<N, E, C> tw;
  load_twiddles<N, E>(tw, lane, tw_x<R>(g));
  const R* ra = (const R*)in.p[f] + (long long)j * g.pp + (long long)(2 * q2) * g.nx;
  const R* rb = ra + g.nx;
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = mkc<C>(__ldg(ra + lane + q * T), __ldg(rb + lane + q * T));
  fft_reg<N, -1>(v, lane, true, sq, tw);
  SEQ_SYNC(N);
#pragma unroll
  for (int q = 0; q < E; ++q) sq[pidx(lane + q * T)] = v[q];
  SEQ_SYNC(N);
  C* oa = (C*)out.p[f] + (long long)j * g.hp + (long long)(2 * q2) * g.kxs;
  C* ob = oa + g.kxs;
  const R s = (R)(0.5 / (double)N);
  for (int m = lane; m < g.kxs; m += T) {
    C A = mkc<C>(0, 0), B = A;
    if (m <= g.nkx) {
      const C zm = sq[pidx(m)], zn = cconj(sq[pidx((N - m) & (N - 1))]);
      A = mkc<C>((zm.x + zn.x) * s, (zm.y + zn.y) * s);
      B = mkc<C>((zm.y - zn.y) * s, -(zm.x - zn.x) * s);  // -i (zm - zn) / 2
    }
    oa[m] = A;
    ob[m] = B;
  }
}

// Xh -> physical; fields f with bit f of dmask set are differentiated in x
// (multiplied by i kx before the transform)
template <int N, typename R>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_inv_x(const __grid_constant__ FieldSet in, const __grid_constant__ FieldSet out, Geom g, unsigned dmask) {
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int q2 = blockIdx.x * (blockDim.x / T) + seq;
  const int j = blockIdx.y, f = blockIdx.z;
  C* sq = sm + seq * padded(N);
  Twiddles<N, E, C> tw;
  load_twiddles<N, E>(tw, lane, tw_x<R>(g));
  const C* ia = (const C*)in.p[f] + (long long)j * g.hp + (long long)(2 * q2) * g.kxs;
  const C* ib = ia + g.kxs;
  const bool dx = (dmask >> f) & 1u;
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const int e = lane + q * T;
    C z = mkc<C>(0, 0);
    if (e <= g.nkx) {
      C A = __ldg(ia + e), B = __ldg(ib + e);
      if (dx) { A = cmul_i(A, (R)g.kx[e]); B = cmul_i(B, (R)g.kx[e]); }
      if (e == 0) { A.y = 0; B.y = 0; }
      z = mkc<C>(A.x - B.y, A.y + B.x);            // A + iB
    } else if (e >= N - g.nkx) {
      C A = __ldg(ia + (N - e)), B = __ldg(ib + (N - e));
      if (dx) { A = cmul_i(A, (R)g.kx[N - e]); B = cmul_i(B, (R)g.kx[N - e]); }
      z = mkc<C>(A.x + B.y, B.x - A.y);            // conj A + i conj B
    }
    v[q] = z;
  }
  fft_reg<N, +1>(v, lane, true, sq, tw);
  R* ra = (R*)out.p[f] + (long long)j * g.pp + (long long)(2 * q2) * g.nx;
  R* rb = ra + g.nx;
#pragma unroll
  for (int q = 0; q < E; ++q) {
    ra[lane + q * T] = v[q].x;
    rb[lane + q * T] = v[q].y;
  }
}

// Xh -> packed spectral (FP64), scaled by 1/Nz; sequence = one kx column of a plane.
// accumulate: out = base + transform, base = out itself, or for rows 0, 1,
// Nyp, Nyp+1 the ghost overlay (field f % 4) when one is given
// B: member-batched (blockIdx.z = member * nf + field)
template <int N, typename R, bool ACC, bool B = false>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_fwd_z(const __grid_constant__ FieldSet in0, const __grid_constant__ FieldSet out0, Geom g0, int accumulate,
                                                          const double2* __restrict__ ghost, const __grid_constant__ Batch bt) {
  const int m = B ? (int)blockIdx.z / bt.nf : 0, f = B ? (int)blockIdx.z - m * bt.nf : (int)blockIdx.z;
  const FieldSet& in = B ? bt.tab[m].fs[bt.fin] : in0;
  const FieldSet& out = B ? bt.tab[m].fs[bt.fout] : out0;
  const Geom& g = g0;   // the same geometry for every member
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  // column-fastest mapping: a warp reads ns consecutive kx of 32/ns rows
  // (whole sectors); the sequence's threads are then spread over the CTA
  // and the exchanges use CTA barriers.  A CTA transforms ZPJ planes in
  // turn, the next plane's tile prefetched into L2 while this one is
  // transformed.
  const int ns = blockDim.x / T;
  const int seq = threadIdx.x % ns, lane = threadIdx.x / ns;
  const int kx = blockIdx.x * ns + seq;
  const bool active = kx < g.kxs;
  C* sq = sm + seq * (padded(N) + 1);   // staggered so the ns columns use different banks
  const C* twt = tw_z<R>(g);   // twiddles fetched per pass (fewer live registers)
  const double s = 1.0 / (double)N;
  for (int jj = 0; jj < ZPJ; ++jj) {
    const int j = blockIdx.y * ZPJ + jj;
    if (j >= g.np) break;                 // uniform over the CTA
    if (jj > 0) __syncthreads();          // the exchange buffers are free again
    const C* src = (const C*)in.p[f] + (long long)j * g.hp + kx;
    if (active && jj + 1 < ZPJ && j + 1 < g.np) {
#pragma unroll
      for (int q = 0; q < E; ++q) prefetch_l2(src + g.hp + (long long)(lane + q * T) * g.kxs);
    }
    C v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = active ? __ldg(src + (long long)(lane + q * T) * g.kxs) : mkc<C>(0, 0);
    double2* dst = (double2*)out.p[f] + (long long)j * g.sp + kx;
    // ACC: the FP64 values the transform adds to are loaded before the
    // transform, so their latency hides behind it
    double2 bv[ACC ? E : 1];
    if (ACC) {
      const double2* base = dst;
      if (ghost) {
        const int qg = (j <= 1) ? j : (j >= g.ny ? j - g.ny + 2 : -1);
        if (qg >= 0) base = ghost + (long long)(4 * (f & 3) + qg) * g.sp + kx;
      }
#pragma unroll
      for (int q = 0; q < (ACC ? E : 1); ++q) {
        const int z = lane + q * T;
        const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
        bv[q] = (active && kzp >= 0) ? base[(long long)kzp * g.kxs] : make_double2(0.0, 0.0);
      }
    }
    fft_reg_lazy<N, -1, true>(v, lane, active, sq, twt);
    if (active) {
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const int z = lane + q * T;
        const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
        if (kzp >= 0) {
          double2 w = cscale(to_d2(v[q]), s);
          if (ACC) w = cadd(bv[ACC ? q : 0], w);
          dst[(long long)kzp * g.kxs] = w;
        }
      }
    }
  }
}

// The nonlinear terms of the substep without LES on the mixed path: for
// equation e (blockIdx.z; 0 u1, 1 u3, 2 u2, 3 th) and ns kx columns of
// plane j, NL_e = (Z(N_e) + i kz Z(M_e)) / Nz from the x-half product fields
// in.p[2e] (N_e) and in.p[2e+1] (M_e), FP64 into out.p[e] (packed
// spectral): one output field instead of two.  The first half of the CTA
// transforms M, the second half N (one transform per thread, so neither
// holds two sequences' registers); the M half parks Z(M) in shared memory
// in natural order for the N half.  Planes outside the equation's solved
// range (which the RHS does not read) are skipped.  (For FP64 fields the
// two-field form of k_fwd_z measured faster: its 4-column CTAs read 64-byte
// row segments, where the halves of a 256-thread CTA hold 2 columns.)
template <int N>
constexpr int znl_threads() { return FftShape<N>::T >= 256 ? 2 * FftShape<N>::T : 256; }
// B: member-batched (blockIdx.z = member * 4 + equation)
template <int N, typename R, bool B = false>
__global__ void __launch_bounds__(znl_threads<N>(), FftShape<N>::T >= 256 ? 1 : DB_LB_FFT)
    k_fwd_z_nl(const __grid_constant__ FieldSet in0, const __grid_constant__ FieldSet out0, Geom g0, int ns,
               const __grid_constant__ Batch bt) {
  const int m = B ? (int)blockIdx.z >> 2 : 0, e = B ? (int)blockIdx.z & 3 : (int)blockIdx.z;
  const FieldSet& in = B ? bt.tab[m].fs[bt.fin] : in0;
  const FieldSet& out = B ? bt.tab[m].fs[bt.fout] : out0;
  const Geom& g = g0;   // the same geometry for every member
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int half = threadIdx.x / (ns * T);   // 0: M, 1: N (whole warps)
  const int t = threadIdx.x % (ns * T);
  const int seq = t % ns, lane = t / ns;     // column-fastest, as k_fwd_z
  const int kx = blockIdx.x * ns + seq, j = blockIdx.y;
  const int jlo = (e == 2) ? 2 : (e == 3 ? g.jstart_th : g.jstart);
  const int jhi = (e == 2) ? g.ny : (e == 3 ? g.jend_th : g.jend);
  if (j < jlo || j > jhi) return;   // uniform over the CTA
  const bool active = kx < g.kxs;
  C* sq = sm + (half * ns + seq) * (padded(N) + 1);    // exchange buffer of this sequence
  C* sz = sm + (2 * ns + seq) * (padded(N) + 1);       // Z(M) of column seq
  const C* src = (const C*)in.p[2 * e + 1 - half] + (long long)j * g.hp + kx;
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = active ? __ldg(src + (long long)(lane + q * T) * g.kxs) : mkc<C>(0, 0);
  fft_reg_lazy<N, -1, true>(v, lane, active, sq, tw_z<R>(g));
  if (half == 0) {
#pragma unroll
    for (int q = 0; q < E; ++q) sz[pidx(lane + q * T)] = v[q];
  }
  __syncthreads();
  if (half == 0 || !active) return;
  const double inz = 1.0 / (double)N;
  double2* dst = (double2*)out.p[e] + (long long)j * g.sp + kx;
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const int z = lane + q * T;
    const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
    if (kzp >= 0) {
      const double kzv = g.kz[kzp];
      const double2 zm = to_d2(sz[pidx(z)]), zn = to_d2(v[q]);
      dst[(long long)kzp * g.kxs] = make_double2((zn.x - kzv * zm.y) * inz, (zn.y + kzv * zm.x) * inz);
    }
  }
}

// packed spectral (FP64) -> Xh (zero-filled de-aliased rows, unnormalised);
// fields f with bit f of dmask set are differentiated in z (times i kz).
// mean (optional): the (0,0) mode of fields 0..3, i.e. the plane mean of
// the physical field, goes to mean[f np + j] in FP64 and is left out of the
// transform, so the physical field holds the fluctuation about the mean
// and its FP32 rounding scales with the fluctuation (the consumers add the
// mean back)
// B: member-batched (blockIdx.z = member * nf + field; no dmask, ghost or mean)
template <int N, typename R, bool B = false>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_inv_z(const __grid_constant__ FieldSet in0, const __grid_constant__ FieldSet out0, Geom g0, unsigned dmask,
                                                          const double2* __restrict__ ghost, double* __restrict__ mean,
                                                          const __grid_constant__ Batch bt) {
  const int m = B ? (int)blockIdx.z / bt.nf : 0, f = B ? (int)blockIdx.z - m * bt.nf : (int)blockIdx.z;
  const FieldSet& in = B ? bt.tab[m].fs[bt.fin] : in0;
  const FieldSet& out = B ? bt.tab[m].fs[bt.fout] : out0;
  const Geom& g = g0;   // the same geometry for every member
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int ns = blockDim.x / T;   // column-fastest mapping, as k_fwd_z
  const int seq = threadIdx.x % ns, lane = threadIdx.x / ns;
  const int kx = blockIdx.x * ns + seq;
  const bool active = kx < g.kxs;
  C* sq = sm + seq * (padded(N) + 1);
  const C* twt = tw_z<R>(g);   // twiddles fetched per pass (fewer live registers)
  const bool dz = (dmask >> f) & 1u;
  // ZPJ planes in turn, as k_fwd_z (the next plane's retained rows
  // prefetched into L2)
  for (int jj = 0; jj < ZPJ; ++jj) {
    const int j = blockIdx.y * ZPJ + jj;
    if (j >= g.np) break;                 // uniform over the CTA
    if (jj > 0) __syncthreads();          // the exchange buffers are free again
    const double2* src = (const double2*)in.p[f] + (long long)j * g.sp + kx;
    if (active && jj + 1 < ZPJ && j + 1 < g.np) {
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const int z = lane + q * T;
        const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
        if (kzp >= 0) prefetch_l2(src + g.sp + (long long)kzp * g.kxs);
      }
    }
    if (ghost) {   // rows 0, 1, Nyp, Nyp+1 from the overlay
      const int q = (j <= 1) ? j : (j >= g.ny ? j - g.ny + 2 : -1);
      if (q >= 0) src = ghost + (long long)(4 * (f & 3) + q) * g.sp + kx;
    }
    C v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int z = lane + q * T;
      const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
      double2 a = (active && kzp >= 0) ? __ldg(src + (long long)kzp * g.kxs) : make_double2(0.0, 0.0);
      if (dz && kzp >= 0) a = cmul_i(a, g.kz[kzp]);
      if (mean && f < 4 && kx == 0 && z == 0) {
        mean[(long long)f * g.np + j] = a.x;
        a = make_double2(0.0, 0.0);
      }
      v[q] = from_d2<C>(a);
    }
    fft_reg_lazy<N, +1, true>(v, lane, active, sq, twt);
    if (active) {
      C* dst = (C*)out.p[f] + (long long)j * g.hp + kx;
#pragma unroll
      for (int q = 0; q < E; ++q) dst[(long long)(lane + q * T) * g.kxs] = v[q];
    }
  }
}

// ---------------------------------------------------------------------------
// x-pass kernels with TMA-staged input.  A CTA of NS sequences is persistent
// over items (field, plane, block of NS row pairs); the rows of one item are
// contiguous, so one thread brings the NEXT item's rows into the other half
// of a double buffer with a single cp.async.bulk while the CTA transforms the
// current item from shared memory: the load latency hides behind the FFT.
constexpr uint32_t STAGE_WAIT = 1u << 24;

template <int N, typename R>
__global__ void __launch_bounds__(256, 2) k_fwd_x_st(const __grid_constant__ FieldSet in, const __grid_constant__ FieldSet out, Geom g, int nblk,
                                                     int nitems) {
  using C = typename CplxOf<R>::type;
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int ns = blockDim.x / T;                       // sequences (row pairs) per item
  const uint32_t row_bytes = N * sizeof(R);
  const uint32_t item_bytes = 2u * ns * row_bytes;
  R* stage0 = reinterpret_cast<R*>(sm_raw);
  C* xbuf = reinterpret_cast<C*>(sm_raw + 2 * item_bytes);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm_raw + 2 * item_bytes + (size_t)ns * padded(N) * sizeof(C));
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  C* sq = xbuf + seq * padded(N);
  const C* twt = tw_x<R>(g);   // twiddles fetched per pass (fewer live registers)
  auto src = [&](int it) -> const R* {
    const int f = it / (g.np * nblk), r = it % (g.np * nblk), j = r / nblk, b = r % nblk;
    return (const R*)in.p[f] + (long long)j * g.pp + (long long)(2 * ns * b) * g.nx;
  };
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0 && (int)blockIdx.x < nitems) {
    mbar_expect_tx(&mbar[0], item_bytes);
    bulk_g2s(stage0, src(blockIdx.x), item_bytes, &mbar[0]);
  }
  int k = 0;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x, ++k) {
    const int s = k & 1;
    const int nxt = it + gridDim.x;
    if (threadIdx.x == 0 && nxt < nitems) {   // prefetch the next item into the other buffer
      fence_async_smem();
      mbar_expect_tx(&mbar[s ^ 1], item_bytes);
      bulk_g2s(reinterpret_cast<unsigned char*>(stage0) + (s ^ 1) * item_bytes, src(nxt), item_bytes, &mbar[s ^ 1]);
    }
    const bool got =
        __syncthreads_and(mbar_wait_first(&mbar[s], (uint32_t)((k >> 1) & 1), g.wait_first, STAGE_WAIT) ? 1 : 0) != 0;
    if (!got) {   // record it, let the copies in flight land (bounded), leave
      if (threadIdx.x == 0) {
        atomicOr(g.flags, DB_FLAG_WAIT_TIMEOUT);
        mbar_wait(&mbar[s], (uint32_t)((k >> 1) & 1), STAGE_WAIT);
        if (nxt < nitems) mbar_wait(&mbar[s ^ 1], (uint32_t)(((k + 1) >> 1) & 1), STAGE_WAIT);
      }
      return;
    }
    const R* ra = reinterpret_cast<const R*>(reinterpret_cast<const unsigned char*>(stage0) + s * item_bytes) +
                  (2 * seq) * N;
    const R* rb = ra + N;
    C v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = mkc<C>(ra[lane + q * T], rb[lane + q * T]);
    fft_reg_lazy<N, -1>(v, lane, true, sq, twt);
    SEQ_SYNC(N);
#pragma unroll
    for (int q = 0; q < E; ++q) sq[pidx(lane + q * T)] = v[q];
    SEQ_SYNC(N);
    const int f = it / (g.np * nblk), r = it % (g.np * nblk), j = r / nblk, b = r % nblk;
    C* oa = (C*)out.p[f] + (long long)j * g.hp + (long long)(2 * (ns * b + seq)) * g.kxs;
    C* ob = oa + g.kxs;
    const R sc = (R)(0.5 / (double)N);
    for (int m = lane; m < g.kxs; m += T) {
      C A = mkc<C>(0, 0), B = A;
      if (m <= g.nkx) {
        const C zm = sq[pidx(m)], zn = cconj(sq[pidx((N - m) & (N - 1))]);
        A = mkc<C>((zm.x + zn.x) * sc, (zm.y + zn.y) * sc);
        B = mkc<C>((zm.y - zn.y) * sc, -(zm.x - zn.x) * sc);
      }
      oa[m] = A;
      ob[m] = B;
    }
    __syncthreads();   // stage s and the exchange buffers are free again
  }
}

// CFL: instead of storing u1, u2, u3 (fields 0..2), reduce the courant
// terms of their physical values (k_courant_reduce's per-point maximum is
// the maximum over the three fields' own terms, so each field reduces its
// own): |u1 - U| / dx, |u2| / dy(j), |u3 + W| / dz over the planes the
// reference's courant visits (for/flow.f90:777-806), then CFL / max per CTA
// into the device minimum, as k_courant_reduce does.  Planes outside that
// range are not transformed.
struct CflArgs {
  Phys ph;
  CflCtl ctl;
  DevScalars* sc;
};

// B: member-batched (the persistent CTAs walk the items of every member,
// member = item / nitems; g is member 0's geometry, the same for all; no
// dmask, not with CFL)
template <int N, typename R, bool CFL, bool B = false>
__global__ void __launch_bounds__(256, 2) k_inv_x_st(const __grid_constant__ FieldSet in, const __grid_constant__ FieldSet out, Geom g,
                                                      unsigned dmask, int nblk, int nitems,
                                                      const __grid_constant__ CflArgs cf, const __grid_constant__ Batch bt) {
  static_assert(!(B && CFL), "the CFL x-pass is not batched");
  const int ntot = B ? nitems * bt.n : nitems;
  auto fs_in = [&](int it) -> const FieldSet& { return B ? bt.tab[it / nitems].fs[bt.fin] : in; };
  auto fs_out = [&](int it) -> const FieldSet& { return B ? bt.tab[it / nitems].fs[bt.fout] : out; };
  using C = typename CplxOf<R>::type;
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int ns = blockDim.x / T;
  const uint32_t row_bytes = (uint32_t)g.kxs * sizeof(C);
  const uint32_t item_bytes = 2u * ns * row_bytes;
  C* stage0 = reinterpret_cast<C*>(sm_raw);
  C* xbuf = reinterpret_cast<C*>(sm_raw + 2 * item_bytes);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm_raw + 2 * item_bytes + (size_t)ns * padded(N) * sizeof(C));
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  C* sq = xbuf + seq * padded(N);
  const C* twt = tw_x<R>(g);   // twiddles fetched per pass (fewer live registers)
  auto src = [&](int it) -> const C* {
    const int li = B ? it % nitems : it;
    const int f = li / (g.np * nblk), r = li % (g.np * nblk), j = r / nblk, b = r % nblk;
    return (const C*)fs_in(it).p[f] + (long long)j * g.hp + (long long)(2 * ns * b) * g.kxs;
  };
  // CFL: courant's gate (for/flow.f90:746-750) and plane range
  if (CFL && !cf.ctl.force && !(cf.ctl.variable_dt && (cf.sc->time_step % cf.ctl.update_dt) == 0)) return;
  const int jlo = CFL ? (cf.ph.front ? g.jstart : 1) : 0;
  const int jhi = CFL ? (cf.ph.front ? g.jend : g.ny) : 0;
  double amax = 0.0;
  bool bad = false;
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0 && (int)blockIdx.x < ntot) {
    mbar_expect_tx(&mbar[0], item_bytes);
    bulk_g2s(stage0, src(blockIdx.x), item_bytes, &mbar[0]);
  }
  int k = 0;
  for (int it = blockIdx.x; it < ntot; it += gridDim.x, ++k) {
    const int s = k & 1;
    const int nxt = it + gridDim.x;
    if (threadIdx.x == 0 && nxt < ntot) {
      fence_async_smem();
      mbar_expect_tx(&mbar[s ^ 1], item_bytes);
      bulk_g2s(reinterpret_cast<unsigned char*>(stage0) + (s ^ 1) * item_bytes, src(nxt), item_bytes, &mbar[s ^ 1]);
    }
    const bool got =
        __syncthreads_and(mbar_wait_first(&mbar[s], (uint32_t)((k >> 1) & 1), g.wait_first, STAGE_WAIT) ? 1 : 0) != 0;
    if (!got) {   // record it, let the copies in flight land (bounded), leave
      if (threadIdx.x == 0) {
        atomicOr(B ? bt.tab[it / nitems].g.flags : g.flags, DB_FLAG_WAIT_TIMEOUT);
        mbar_wait(&mbar[s], (uint32_t)((k >> 1) & 1), STAGE_WAIT);
        if (nxt < ntot) mbar_wait(&mbar[s ^ 1], (uint32_t)(((k + 1) >> 1) & 1), STAGE_WAIT);
      }
      return;
    }
    const int li = B ? it % nitems : it;
    const int f = li / (g.np * nblk), r = li % (g.np * nblk), j = r / nblk, b = r % nblk;
    if (CFL && (j < jlo || j > jhi)) {   // uniform over the CTA: not a courant plane
      __syncthreads();
      continue;
    }
    const C* ia = reinterpret_cast<const C*>(reinterpret_cast<const unsigned char*>(stage0) + s * item_bytes) +
                  (2 * seq) * g.kxs;
    const C* ib = ia + g.kxs;
    const bool dx = (dmask >> f) & 1u;
    C v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const int e = lane + q * T;
      C z = mkc<C>(0, 0);
      if (e <= g.nkx) {
        C ra = ia[e], rb = ib[e];   // the two rows' coefficients
        if (dx) { ra = cmul_i(ra, (R)g.kx[e]); rb = cmul_i(rb, (R)g.kx[e]); }
        if (e == 0) { ra.y = 0; rb.y = 0; }
        z = mkc<C>(ra.x - rb.y, ra.y + rb.x);
      } else if (e >= N - g.nkx) {
        C ra = ia[N - e], rb = ib[N - e];
        if (dx) { ra = cmul_i(ra, (R)g.kx[N - e]); rb = cmul_i(rb, (R)g.kx[N - e]); }
        z = mkc<C>(ra.x + rb.y, rb.x - ra.y);
      }
      v[q] = z;
    }
    fft_reg_lazy<N, +1>(v, lane, true, sq, twt);
    if (CFL) {
      // |u1 - c1| / dx, |u2| / dy, |u3 + c3| / dz with k_courant_reduce's operations
      const double fr = cf.ph.ro_inv / cf.ph.delta;
      double c = 0.0, w;
      if (f == 0) {
        c = cf.ph.front ? cf.ph.dthdz * g.gyf[j] / fr : 0.0;   // -c1, subtracted below as v - c1
        w = 1.0 / cf.ph.dx;
      } else if (f == 1) {
        w = 1.0 / g.dy[j];
      } else {
        c = cf.ph.front ? (1.0 / fr) * cf.ph.dthdx * (g.gyf[j] - 0.5 * cf.ph.ly) : 0.0;   // c3
        w = 1.0 / cf.ph.dz;
      }
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const double va = (double)v[q].x, vb = (double)v[q].y;
        const double ta = (f == 0 ? fabs(va - c) : (f == 1 ? fabs(va) : fabs(va + c))) * w;
        const double tb = (f == 0 ? fabs(vb - c) : (f == 1 ? fabs(vb) : fabs(vb + c))) * w;
        bad = bad || !(ta <= 1.7976931348623157e308) || !(tb <= 1.7976931348623157e308);
        amax = fmax(amax, fmax(ta, tb));
      }
    } else {
      R* ra = (R*)fs_out(it).p[f] + (long long)j * g.pp + (long long)(2 * (ns * b + seq)) * g.nx;
      R* rb = ra + g.nx;
#pragma unroll
      for (int q = 0; q < E; ++q) {
        ra[lane + q * T] = v[q].x;
        rb[lane + q * T] = v[q].y;
      }
    }
    __syncthreads();
  }
  if (CFL) {
    if (bad) atomicOr(&cf.sc->flags, DB_FLAG_NONFINITE);
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) amax = fmax(amax, red[w]);
      if (amax > 0.0)
        atomicMin(&cf.sc->dt_min_bits, (unsigned long long)__double_as_longlong(cf.ctl.cfl / amax));
    }
  }
}

// ---------------------------------------------------------------------------
// launchers

// sequences per CTA: 256 threads, or one sequence when it needs more
template <int N>
constexpr int seqs_per_cta() {
  return FftShape<N>::T >= 256 ? 1 : 256 / FftShape<N>::T;
}

#define DB_DISPATCH_N(n, FN, ...)                                   \
  switch (n) {                                                      \
    case 16: FN<16>(__VA_ARGS__); break;                            \
    case 32: FN<32>(__VA_ARGS__); break;                            \
    case 64: FN<64>(__VA_ARGS__); break;                            \
    case 128: FN<128>(__VA_ARGS__); break;                          \
    case 256: FN<256>(__VA_ARGS__); break;                          \
    case 512: FN<512>(__VA_ARGS__); break;                          \
    case 1024: FN<1024>(__VA_ARGS__); break;                        \
    case 2048: FN<2048>(__VA_ARGS__); break;                        \
    default: return cudaErrorInvalidValue;                          \
  }

template <typename K>
static void smem_attr(K kern, size_t smem) {
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// sequences per item of the staged x-pass: cps (<= seqs_per_cta, divides nz/2)
template <int N>
static int xpass_cps(const Geom& g) {
  constexpr int ns = seqs_per_cta<N>();
  int npairs = g.nz / 2;
  int want = (g.tune_xcps > 0 && g.tune_xcps <= ns) ? g.tune_xcps : ns;
  int cps = want < npairs ? want : npairs;
  while (npairs % cps) --cps;
  return cps;
}
static int xpass_ctas_per_sm(const Geom& g) { return g.tune_xgrid > 0 ? g.tune_xgrid : 2; }
template <int N>
static int zpass_ns(const Geom& g) {
  constexpr int ns = seqs_per_cta<N>();
  return (g.tune_zns > 0 && g.tune_zns <= ns) ? g.tune_zns : ns;
}
int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int N, typename R>
static void go_fwd_x_t(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int cps = xpass_cps<N>(g);
  const int nblk = (g.nz / 2) / cps, nitems = nblk * g.np * nf;
  const size_t smem = 2 * (size_t)(2 * cps * N * sizeof(R)) + (size_t)cps * padded(N) * sizeof(C) + 16;
  smem_attr(k_fwd_x_st<N, R>, smem);
  const int gmax = xpass_ctas_per_sm(g) * sm_count();
  const int grid = nitems < gmax ? nitems : gmax;
  k_fwd_x_st<N, R><<<grid, cps * FftShape<N>::T, smem, st>>>(in, out, g, nblk, nitems);
}
template <int N, typename R>
static void go_inv_x_t(const Geom& g, FieldSet in, FieldSet out, int nf, unsigned dmask, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int cps = xpass_cps<N>(g);
  const int nblk = (g.nz / 2) / cps, nitems = nblk * g.np * nf;
  const size_t smem = 2 * (size_t)(2 * cps * g.kxs * sizeof(C)) + (size_t)cps * padded(N) * sizeof(C) + 16;
  smem_attr(k_inv_x_st<N, R, false>, smem);
  const int gmax = xpass_ctas_per_sm(g) * sm_count();
  const int grid = nitems < gmax ? nitems : gmax;
  k_inv_x_st<N, R, false><<<grid, cps * FftShape<N>::T, smem, st>>>(in, out, g, dmask, nblk, nitems, CflArgs{}, Batch{});
}
template <int N, typename R>
static void go_inv_x_cfl_t(const Geom& g, FieldSet in, const CflArgs& cf, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int cps = xpass_cps<N>(g);
  const int nblk = (g.nz / 2) / cps, nitems = nblk * g.np * 3;
  const size_t smem = 2 * (size_t)(2 * cps * g.kxs * sizeof(C)) + (size_t)cps * padded(N) * sizeof(C) + 16;
  smem_attr(k_inv_x_st<N, R, true>, smem);
  const int gmax = xpass_ctas_per_sm(g) * sm_count();
  const int grid = nitems < gmax ? nitems : gmax;
  k_inv_x_st<N, R, true><<<grid, cps * FftShape<N>::T, smem, st>>>(in, FieldSet{}, g, 0u, nblk, nitems, cf, Batch{});
}
template <int N>
static void go_inv_x_cfl(const Geom& g, FieldSet in, const CflArgs& cf, cudaStream_t st) {
  if (g.prec) go_inv_x_cfl_t<N, float>(g, in, cf, st);
  else go_inv_x_cfl_t<N, double>(g, in, cf, st);
}
template <int N, typename R>
static void go_fwd_z_t(const Geom& g, FieldSet in, FieldSet out, int nf, int acc, const double2* ghost,
                       cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int ns = zpass_ns<N>(g);
  size_t smem = (size_t)ns * (padded(N) + 1) * sizeof(C);
  const dim3 grid((g.kxs + ns - 1) / ns, (g.np + ZPJ - 1) / ZPJ, nf);
  if (acc) {
    smem_attr(k_fwd_z<N, R, true>, smem);
    k_fwd_z<N, R, true><<<grid, ns * FftShape<N>::T, smem, st>>>(in, out, g, 1, ghost, Batch{});
  } else {
    smem_attr(k_fwd_z<N, R, false>, smem);
    k_fwd_z<N, R, false><<<grid, ns * FftShape<N>::T, smem, st>>>(in, out, g, 0, ghost, Batch{});
  }
}
template <int N, typename R>
static void go_inv_z_t(const Geom& g, FieldSet in, FieldSet out, int nf, unsigned dmask, const double2* ghost,
                       double* mean, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int ns = zpass_ns<N>(g);
  size_t smem = (size_t)ns * (padded(N) + 1) * sizeof(C);
  smem_attr(k_inv_z<N, R>, smem);
  k_inv_z<N, R><<<dim3((g.kxs + ns - 1) / ns, (g.np + ZPJ - 1) / ZPJ, nf), ns * FftShape<N>::T, smem, st>>>(in, out, g, dmask, ghost,
                                                                                          mean, Batch{});
}
template <int N, typename R>
static void go_fwd_z_nl_t(const Geom& g, FieldSet in, FieldSet out, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  constexpr int T = FftShape<N>::T;
  const int ns = znl_threads<N>() / (2 * T);
  const size_t smem = (size_t)3 * ns * (padded(N) + 1) * sizeof(C);
  smem_attr(k_fwd_z_nl<N, R>, smem);
  k_fwd_z_nl<N, R><<<dim3((g.kxs + ns - 1) / ns, g.np, 4), 2 * ns * T, smem, st>>>(in, out, g, ns, Batch{});
}
template <int N>
static void go_fwd_z_nl(const Geom& g, FieldSet in, FieldSet out, cudaStream_t st) {
  if (g.prec) go_fwd_z_nl_t<N, float>(g, in, out, st);
  else go_fwd_z_nl_t<N, double>(g, in, out, st);
}
template <int N>
static void go_fwd_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  if (g.prec) go_fwd_x_t<N, float>(g, in, out, nf, st);
  else go_fwd_x_t<N, double>(g, in, out, nf, st);
}
template <int N>
static void go_inv_x(const Geom& g, FieldSet in, FieldSet out, int nf, unsigned dmask, cudaStream_t st) {
  if (g.prec) go_inv_x_t<N, float>(g, in, out, nf, dmask, st);
  else go_inv_x_t<N, double>(g, in, out, nf, dmask, st);
}
template <int N>
static void go_fwd_z(const Geom& g, FieldSet in, FieldSet out, int nf, int acc, const double2* ghost,
                     cudaStream_t st) {
  if (g.prec) go_fwd_z_t<N, float>(g, in, out, nf, acc, ghost, st);
  else go_fwd_z_t<N, double>(g, in, out, nf, acc, ghost, st);
}
template <int N>
static void go_inv_z(const Geom& g, FieldSet in, FieldSet out, int nf, unsigned dmask, const double2* ghost,
                     double* mean, cudaStream_t st) {
  if (g.prec) go_inv_z_t<N, float>(g, in, out, nf, dmask, ghost, mean, st);
  else go_inv_z_t<N, double>(g, in, out, nf, dmask, ghost, mean, st);
}

cudaError_t launch_fwd_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  if (nf < 1 || nf > MAXF) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nx, go_fwd_x, g, in, out, nf, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, unsigned dmask) {
  if (nf < 1 || nf > MAXF) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nx, go_inv_x, g, in, out, nf, dmask, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_x_cfl(const Geom& g, const Phys& ph, const State& s, CflCtl ctl, FieldSet in, cudaStream_t st) {
  const CflArgs cf{ph, ctl, s.sc};
  DB_DISPATCH_N(g.nx, go_inv_x_cfl, g, in, cf, st);
  return cudaGetLastError();
}
cudaError_t launch_fwd_z_nl(const Geom& g, FieldSet in, FieldSet out, cudaStream_t st) {
  DB_DISPATCH_N(g.nz, go_fwd_z_nl, g, in, out, st);
  return cudaGetLastError();
}
cudaError_t launch_fwd_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, int accumulate,
                         const double2* ghost) {
  if (nf < 1 || nf > MAXF) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_fwd_z, g, in, out, nf, accumulate, ghost, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, unsigned dmask,
                         const double2* ghost, double* mean) {
  if (nf < 1 || nf > MAXF) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_inv_z, g, in, out, nf, dmask, ghost, mean, st);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// member-batched transforms: the shapes of the single-context launchers with
// the member folded into blockIdx.z (z-passes) or blockIdx.y (x-pass, each
// member's items over its own share of the persistent CTAs)

template <int N, typename R>
static void go_inv_x_bt(const Geom& g, const Batch& bt, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int cps = xpass_cps<N>(g);
  const int nblk = (g.nz / 2) / cps, nitems = nblk * g.np * bt.nf;
  const size_t smem = 2 * (size_t)(2 * cps * g.kxs * sizeof(C)) + (size_t)cps * padded(N) * sizeof(C) + 16;
  smem_attr(k_inv_x_st<N, R, false, true>, smem);
  const int gmax = xpass_ctas_per_sm(g) * sm_count();
  const long long ntot = (long long)nitems * bt.n;
  const int grid = ntot < gmax ? (int)ntot : gmax;
  k_inv_x_st<N, R, false, true><<<grid, cps * FftShape<N>::T, smem, st>>>(FieldSet{}, FieldSet{}, g, 0u, nblk,
                                                                           nitems, CflArgs{}, bt);
}
template <int N, typename R>
static void go_inv_z_bt(const Geom& g, const Batch& bt, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int ns = zpass_ns<N>(g);
  const size_t smem = (size_t)ns * (padded(N) + 1) * sizeof(C);
  smem_attr(k_inv_z<N, R, true>, smem);
  k_inv_z<N, R, true><<<dim3((g.kxs + ns - 1) / ns, (g.np + ZPJ - 1) / ZPJ, bt.n * bt.nf), ns * FftShape<N>::T, smem,
                        st>>>(
      FieldSet{}, FieldSet{}, g, 0u, nullptr, nullptr, bt);
}
template <int N, typename R>
static void go_fwd_z_bt(const Geom& g, const Batch& bt, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  const int ns = zpass_ns<N>(g);
  const size_t smem = (size_t)ns * (padded(N) + 1) * sizeof(C);
  smem_attr(k_fwd_z<N, R, false, true>, smem);
  k_fwd_z<N, R, false, true><<<dim3((g.kxs + ns - 1) / ns, (g.np + ZPJ - 1) / ZPJ, bt.n * bt.nf), ns * FftShape<N>::T,
                               smem, st>>>(
      FieldSet{}, FieldSet{}, g, 0, nullptr, bt);
}
template <int N, typename R>
static void go_fwd_z_nl_bt(const Geom& g, const Batch& bt, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  constexpr int T = FftShape<N>::T;
  const int ns = znl_threads<N>() / (2 * T);
  const size_t smem = (size_t)3 * ns * (padded(N) + 1) * sizeof(C);
  smem_attr(k_fwd_z_nl<N, R, true>, smem);
  k_fwd_z_nl<N, R, true><<<dim3((g.kxs + ns - 1) / ns, g.np, 4 * bt.n), 2 * ns * T, smem, st>>>(
      FieldSet{}, FieldSet{}, g, ns, bt);
}
template <int N>
static void go_inv_x_b(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (g.prec) go_inv_x_bt<N, float>(g, bt, st); else go_inv_x_bt<N, double>(g, bt, st);
}
template <int N>
static void go_inv_z_b(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (g.prec) go_inv_z_bt<N, float>(g, bt, st); else go_inv_z_bt<N, double>(g, bt, st);
}
template <int N>
static void go_fwd_z_b(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (g.prec) go_fwd_z_bt<N, float>(g, bt, st); else go_fwd_z_bt<N, double>(g, bt, st);
}
template <int N>
static void go_fwd_z_nl_b(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (g.prec) go_fwd_z_nl_bt<N, float>(g, bt, st); else go_fwd_z_nl_bt<N, double>(g, bt, st);
}

static bool batch_ok(const Batch& bt) { return bt.tab && bt.n >= 1 && bt.n <= 65535 / MAXF && bt.nf >= 1 && bt.nf <= MAXF; }

cudaError_t launch_inv_x_batch(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (!batch_ok(bt)) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nx, go_inv_x_b, g, bt, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_z_batch(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (!batch_ok(bt)) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_inv_z_b, g, bt, st);
  return cudaGetLastError();
}
cudaError_t launch_fwd_z_batch(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (!batch_ok(bt)) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_fwd_z_b, g, bt, st);
  return cudaGetLastError();
}
cudaError_t launch_fwd_z_nl_batch(const Geom& g, const Batch& bt, cudaStream_t st) {
  if (!batch_ok(bt)) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_fwd_z_nl_b, g, bt, st);
  return cudaGetLastError();
}

}  // namespace db
