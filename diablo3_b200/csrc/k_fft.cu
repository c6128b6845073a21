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
#include "db_kernels.cuh"
#include "fft_reg.cuh"

namespace db {

// ---------------------------------------------------------------------------
// Each group of T = N/E threads (one warp for N <= 512) transforms one
// sequence; a CTA holds NS = blockDim / T independent sequences.

// physical -> Xh: sequence = rows (2q, 2q+1) of one plane/field
template <int N, typename R>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_fwd_x(FieldSet in, FieldSet out, Geom g) {
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
__global__ void __launch_bounds__(256, DB_LB_FFT) k_inv_x(FieldSet in, FieldSet out, Geom g, unsigned dmask) {
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
template <int N, typename R>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_fwd_z(FieldSet in, FieldSet out, Geom g, int accumulate,
                                                          const double2* __restrict__ ghost) {
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int kx = blockIdx.x * (blockDim.x / T) + seq, j = blockIdx.y, f = blockIdx.z;
  const bool active = kx < g.kxs;
  C* sq = sm + seq * padded(N);
  Twiddles<N, E, C> tw;
  load_twiddles<N, E>(tw, lane, tw_z<R>(g));
  const C* src = (const C*)in.p[f] + (long long)j * g.hp + kx;
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = active ? __ldg(src + (long long)(lane + q * T) * g.kxs) : mkc<C>(0, 0);
  fft_reg<N, -1>(v, lane, active, sq, tw);
  if (!active) return;
  double2* dst = (double2*)out.p[f] + (long long)j * g.sp + kx;
  const double2* base = dst;
  if (accumulate && ghost) {
    const int qg = (j <= 1) ? j : (j >= g.ny ? j - g.ny + 2 : -1);
    if (qg >= 0) base = ghost + (long long)(4 * (f & 3) + qg) * g.sp + kx;
  }
  const double s = 1.0 / (double)N;
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const int z = lane + q * T;
    const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
    if (kzp >= 0) {
      double2 w = cscale(to_d2(v[q]), s);
      if (accumulate) w = cadd(base[(long long)kzp * g.kxs], w);
      dst[(long long)kzp * g.kxs] = w;
    }
  }
}

// packed spectral (FP64) -> Xh (zero-filled de-aliased rows, unnormalised);
// fields f with bit f of dmask set are differentiated in z (times i kz)
template <int N, typename R>
__global__ void __launch_bounds__(256, DB_LB_FFT) k_inv_z(FieldSet in, FieldSet out, Geom g, unsigned dmask,
                                                          const double2* __restrict__ ghost) {
  using C = typename CplxOf<R>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  using S = FftShape<N>;
  constexpr int E = S::E, T = S::T;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int kx = blockIdx.x * (blockDim.x / T) + seq, j = blockIdx.y, f = blockIdx.z;
  const bool active = kx < g.kxs;
  C* sq = sm + seq * padded(N);
  Twiddles<N, E, C> tw;
  load_twiddles<N, E>(tw, lane, tw_z<R>(g));
  const double2* src = (const double2*)in.p[f] + (long long)j * g.sp + kx;
  if (ghost) {   // rows 0, 1, Nyp, Nyp+1 from the overlay
    const int q = (j <= 1) ? j : (j >= g.ny ? j - g.ny + 2 : -1);
    if (q >= 0) src = ghost + (long long)(4 * (f & 3) + q) * g.sp + kx;
  }
  const bool dz = (dmask >> f) & 1u;
  C v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const int z = lane + q * T;
    const int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
    double2 a = (active && kzp >= 0) ? __ldg(src + (long long)kzp * g.kxs) : make_double2(0.0, 0.0);
    if (dz && kzp >= 0) a = cmul_i(a, g.kz[kzp]);
    v[q] = from_d2<C>(a);
  }
  fft_reg<N, +1>(v, lane, active, sq, tw);
  if (!active) return;
  C* dst = (C*)out.p[f] + (long long)j * g.hp + kx;
#pragma unroll
  for (int q = 0; q < E; ++q) dst[(long long)(lane + q * T) * g.kxs] = v[q];
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

template <int N, typename R>
static void go_fwd_x_t(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  constexpr int ns = seqs_per_cta<N>();
  int npairs = g.nz / 2;
  int cps = ns < npairs ? ns : npairs;
  while (npairs % cps) --cps;
  size_t smem = (size_t)cps * padded(N) * sizeof(C);
  smem_attr(k_fwd_x<N, R>, smem);
  k_fwd_x<N, R><<<dim3(npairs / cps, g.np, nf), cps * FftShape<N>::T, smem, st>>>(in, out, g);
}
template <int N, typename R>
static void go_inv_x_t(const Geom& g, FieldSet in, FieldSet out, int nf, unsigned dmask, cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  constexpr int ns = seqs_per_cta<N>();
  int npairs = g.nz / 2;
  int cps = ns < npairs ? ns : npairs;
  while (npairs % cps) --cps;
  size_t smem = (size_t)cps * padded(N) * sizeof(C);
  smem_attr(k_inv_x<N, R>, smem);
  k_inv_x<N, R><<<dim3(npairs / cps, g.np, nf), cps * FftShape<N>::T, smem, st>>>(in, out, g, dmask);
}
template <int N, typename R>
static void go_fwd_z_t(const Geom& g, FieldSet in, FieldSet out, int nf, int acc, const double2* ghost,
                       cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  constexpr int ns = seqs_per_cta<N>();
  size_t smem = (size_t)ns * padded(N) * sizeof(C);
  smem_attr(k_fwd_z<N, R>, smem);
  k_fwd_z<N, R><<<dim3((g.kxs + ns - 1) / ns, g.np, nf), ns * FftShape<N>::T, smem, st>>>(in, out, g, acc, ghost);
}
template <int N, typename R>
static void go_inv_z_t(const Geom& g, FieldSet in, FieldSet out, int nf, unsigned dmask, const double2* ghost,
                       cudaStream_t st) {
  using C = typename CplxOf<R>::type;
  constexpr int ns = seqs_per_cta<N>();
  size_t smem = (size_t)ns * padded(N) * sizeof(C);
  smem_attr(k_inv_z<N, R>, smem);
  k_inv_z<N, R><<<dim3((g.kxs + ns - 1) / ns, g.np, nf), ns * FftShape<N>::T, smem, st>>>(in, out, g, dmask, ghost);
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
                     cudaStream_t st) {
  if (g.prec) go_inv_z_t<N, float>(g, in, out, nf, dmask, ghost, st);
  else go_inv_z_t<N, double>(g, in, out, nf, dmask, ghost, st);
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
cudaError_t launch_fwd_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, int accumulate,
                         const double2* ghost) {
  if (nf < 1 || nf > MAXF) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_fwd_z, g, in, out, nf, accumulate, ghost, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, unsigned dmask,
                         const double2* ghost) {
  if (nf < 1 || nf > MAXF) return cudaErrorInvalidValue;
  DB_DISPATCH_N(g.nz, go_inv_z, g, in, out, nf, dmask, ghost, st);
  return cudaGetLastError();
}

}  // namespace db
