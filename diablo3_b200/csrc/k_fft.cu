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
#include "db_kernels.cuh"
#include "fft_smem.cuh"

namespace db {

constexpr int ZPAD = 1;  // double2 padding per shared-memory sequence

// ---------------------------------------------------------------------------
// physical -> Xh, one CTA = ZP pairs of z-rows (2q, 2q+1) of one plane/field
template <int N>
__global__ void __launch_bounds__(512) k_fwd_x(FieldSet in, FieldSet out, Geom g, int zp) {
  extern __shared__ double2 sm[];
  constexpr int T = N / 8;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int q = blockIdx.x * zp + seq;
  const int j = blockIdx.y, f = blockIdx.z;
  const bool active = (seq < zp) && (2 * q + 1 < g.nz);
  double2* buf = sm + seq * (N + ZPAD);
  const double* src = (const double*)in.p[f];
  if (active) {
    const double* ra = src + (long long)j * g.pp + (long long)(2 * q) * g.nx;
    const double* rb = ra + g.nx;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      int e = lane + m * T;
      buf[e] = make_double2(ra[e], rb[e]);
    }
  }
  __syncthreads();
  fft_inplace<N, -1>(buf, lane, active, g.twx);
  if (active) {
    double2* oa = (double2*)out.p[f] + (long long)j * g.hp + (long long)(2 * q) * g.kxs;
    double2* ob = oa + g.kxs;
    const double s = 0.5 / (double)N;
    for (int m = lane; m < g.kxs; m += T) {
      double2 A = make_double2(0.0, 0.0), B = A;
      if (m <= g.nkx) {
        double2 zm = buf[m], zn = cconj(buf[(N - m) & (N - 1)]);
        double2 sp = cadd(zm, zn), dm = csub(zm, zn);
        A = cscale(sp, s);
        B = make_double2(dm.y * s, -dm.x * s);  // -i (zm - zn) / 2
      }
      oa[m] = A;
      ob[m] = B;
    }
  }
}

// Xh -> physical
template <int N>
__global__ void __launch_bounds__(512) k_inv_x(FieldSet in, FieldSet out, Geom g, int zp) {
  extern __shared__ double2 sm[];
  constexpr int T = N / 8;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int q = blockIdx.x * zp + seq;
  const int j = blockIdx.y, f = blockIdx.z;
  const bool active = (seq < zp) && (2 * q + 1 < g.nz);
  double2* buf = sm + seq * (N + ZPAD);
  if (active) {
    const double2* ia = (const double2*)in.p[f] + (long long)j * g.hp + (long long)(2 * q) * g.kxs;
    const double2* ib = ia + g.kxs;
    for (int m = lane; m <= N / 2; m += T) {
      double2 A = make_double2(0.0, 0.0), B = A;
      if (m <= g.nkx) {
        A = ia[m];
        B = ib[m];
      }
      if (m == 0 || m == N / 2) {
        A.y = 0.0;
        B.y = 0.0;
      }
      buf[m] = make_double2(A.x - B.y, A.y + B.x);                        // A + iB
      if (m > 0 && m < N / 2) buf[N - m] = make_double2(A.x + B.y, B.x - A.y);  // conj A + i conj B
    }
  }
  __syncthreads();
  fft_inplace<N, +1>(buf, lane, active, g.twx);
  if (active) {
    double* ra = (double*)out.p[f] + (long long)j * g.pp + (long long)(2 * q) * g.nx;
    double* rb = ra + g.nx;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      int e = lane + m * T;
      double2 v = buf[e];
      ra[e] = v.x;
      rb[e] = v.y;
    }
  }
}

// Xh -> packed spectral, scaled by 1/Nz; one CTA = KT kx columns of a plane
template <int N>
__global__ void __launch_bounds__(512) k_fwd_z(FieldSet in, FieldSet out, Geom g) {
  extern __shared__ double2 sm[];
  constexpr int T = N / 8;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int kx0 = blockIdx.x * KT, j = blockIdx.y, f = blockIdx.z;
  const double2* src = (const double2*)in.p[f] + (long long)j * g.hp + kx0;
  for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x) {
    int z = idx / KT, kl = idx % KT;
    sm[kl * (N + ZPAD) + z] = src[(long long)z * g.kxs + kl];
  }
  __syncthreads();
  fft_inplace<N, -1>(sm + seq * (N + ZPAD), lane, seq < KT, g.twz);
  double2* dst = (double2*)out.p[f] + (long long)j * g.sp + kx0;
  const double s = 1.0 / (double)N;
  for (int idx = threadIdx.x; idx < KT * g.nkzp; idx += blockDim.x) {
    int kzp = idx / KT, kl = idx % KT;
    int z = (kzp <= g.nkz) ? kzp : kzp + N - g.nkzp;
    dst[(long long)kzp * g.kxs + kl] = cscale(sm[kl * (N + ZPAD) + z], s);
  }
}

// packed spectral -> Xh (zero-filled de-aliased rows, unnormalised)
template <int N>
__global__ void __launch_bounds__(512) k_inv_z(FieldSet in, FieldSet out, Geom g) {
  extern __shared__ double2 sm[];
  constexpr int T = N / 8;
  const int seq = threadIdx.x / T, lane = threadIdx.x % T;
  const int kx0 = blockIdx.x * KT, j = blockIdx.y, f = blockIdx.z;
  const double2* src = (const double2*)in.p[f] + (long long)j * g.sp + kx0;
  for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x) {
    int z = idx / KT, kl = idx % KT;
    int kzp = (z <= g.nkz) ? z : (z >= N - g.nkz ? z - N + g.nkzp : -1);
    sm[kl * (N + ZPAD) + z] = (kzp >= 0) ? src[(long long)kzp * g.kxs + kl] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  fft_inplace<N, +1>(sm + seq * (N + ZPAD), lane, seq < KT, g.twz);
  double2* dst = (double2*)out.p[f] + (long long)j * g.hp + kx0;
  for (int idx = threadIdx.x; idx < KT * N; idx += blockDim.x) {
    int z = idx / KT, kl = idx % KT;
    dst[(long long)z * g.kxs + kl] = sm[kl * (N + ZPAD) + z];
  }
}

// ---------------------------------------------------------------------------
// launchers

int x_rows_per_cta(int n, int nz) {
  int zp = 256 / (n / 8);
  if (zp < 1) zp = 1;
  while (zp > 1 && ((nz / 2) % zp) != 0) --zp;
  return zp;
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
    case 4096: FN<4096>(__VA_ARGS__); break;                        \
    default: return cudaErrorInvalidValue;                          \
  }

template <int N>
static void go_fwd_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  int zp = x_rows_per_cta(N, g.nz);
  dim3 grid(g.nz / 2 / zp, g.np, nf);
  size_t smem = (size_t)zp * (N + ZPAD) * sizeof(double2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_fwd_x<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fwd_x<N><<<grid, zp * (N / 8), smem, st>>>(in, out, g, zp);
}
template <int N>
static void go_inv_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  int zp = x_rows_per_cta(N, g.nz);
  dim3 grid(g.nz / 2 / zp, g.np, nf);
  size_t smem = (size_t)zp * (N + ZPAD) * sizeof(double2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_inv_x<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_inv_x<N><<<grid, zp * (N / 8), smem, st>>>(in, out, g, zp);
}
template <int N>
static void go_fwd_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  dim3 grid(g.kxs / KT, g.np, nf);
  size_t smem = (size_t)KT * (N + ZPAD) * sizeof(double2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_fwd_z<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fwd_z<N><<<grid, KT * (N / 8), smem, st>>>(in, out, g);
}
template <int N>
static void go_inv_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  dim3 grid(g.kxs / KT, g.np, nf);
  size_t smem = (size_t)KT * (N + ZPAD) * sizeof(double2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_inv_z<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_inv_z<N><<<grid, KT * (N / 8), smem, st>>>(in, out, g);
}

cudaError_t launch_fwd_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  DB_DISPATCH_N(g.nx, go_fwd_x, g, in, out, nf, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  DB_DISPATCH_N(g.nx, go_inv_x, g, in, out, nf, st);
  return cudaGetLastError();
}
cudaError_t launch_fwd_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  DB_DISPATCH_N(g.nz, go_fwd_z, g, in, out, nf, st);
  return cudaGetLastError();
}
cudaError_t launch_inv_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st) {
  DB_DISPATCH_N(g.nz, go_inv_z, g, in, out, nf, st);
  return cudaGetLastError();
}

}  // namespace db
