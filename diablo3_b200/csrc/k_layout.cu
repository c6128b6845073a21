// k_layout.cu -- spectral fields between the device's compact layout
// [j][kzp][kx] (kx < kxs, kzp < 2 Nkz + 1) and the reference layout of the
// host arrays, complex (0:Nx/2, 0:Nz+1, 0:Nyp+1) (for/fft.f90:71-124), on
// the device: a host transfer is then one DMA of the caller's array.
#include "db_kernels.cuh"

namespace db {

__global__ void k_spec_to_ref(Geom g, int nxp1, int nz2, const double2* __restrict__ src, double2* __restrict__ ref) {
  const long long n = (long long)g.np * nz2 * nxp1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % nxp1);
    const long long r = e / nxp1;
    const int k = (int)(r % nz2), j = (int)(r / nz2);
    ref[e] = (k < g.nkzp && i <= g.nkx) ? src[(long long)j * g.sp + (long long)k * g.kxs + i]
                                        : make_double2(0.0, 0.0);
  }
}

__global__ void k_ref_to_spec(Geom g, int nxp1, int nz2, const double2* __restrict__ ref, double2* __restrict__ dst) {
  const long long n = (long long)g.np * g.sp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % g.kxs);
    const long long r = e / g.kxs;
    const int k = (int)(r % g.nkzp), j = (int)(r / g.nkzp);
    dst[e] = (i <= g.nkx) ? ref[((long long)j * nz2 + k) * nxp1 + i] : make_double2(0.0, 0.0);
  }
}

// physical field: reference layout (0:Nx+1, 0:Nz+1, 0:Nyp+1) doubles, x
// fastest <-> compact [j][z][x] at the context's precision; the padding
// (x >= Nx, z >= Nz) is neither read nor written
template <typename R>
__global__ void k_phys_from_ref(Geom g, int nx2, int nz2, const double* __restrict__ ref, R* __restrict__ dst) {
  const long long n = (long long)g.np * g.pp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % g.nx);
    const long long r = e / g.nx;
    const int z = (int)(r % g.nz), j = (int)(r / g.nz);
    dst[e] = (R)ref[((long long)j * nz2 + z) * nx2 + x];
  }
}

template <typename R>
__global__ void k_phys_to_ref(Geom g, int nx2, int nz2, const R* __restrict__ src, double* __restrict__ ref) {
  const long long n = (long long)g.np * g.pp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % g.nx);
    const long long r = e / g.nx;
    const int z = (int)(r % g.nz), j = (int)(r / g.nz);
    ref[((long long)j * nz2 + z) * nx2 + x] = (double)src[e];
  }
}

static int grid_for(long long n) {
  const long long b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? b : 148 * 16);
}

cudaError_t launch_spec_to_ref(const Geom& g, int nx, int nz, const double2* src, double2* ref, cudaStream_t st) {
  const int nxp1 = nx / 2 + 1, nz2 = nz + 2;
  k_spec_to_ref<<<grid_for((long long)g.np * nz2 * nxp1), 256, 0, st>>>(g, nxp1, nz2, src, ref);
  return cudaGetLastError();
}

cudaError_t launch_ref_to_spec(const Geom& g, int nx, int nz, const double2* ref, double2* dst, cudaStream_t st) {
  const int nxp1 = nx / 2 + 1, nz2 = nz + 2;
  k_ref_to_spec<<<grid_for((long long)g.np * g.sp), 256, 0, st>>>(g, nxp1, nz2, ref, dst);
  return cudaGetLastError();
}

cudaError_t launch_phys_from_ref(const Geom& g, int nx, int nz, const double* ref, void* dst, cudaStream_t st) {
  const long long n = (long long)g.np * g.pp;
  if (g.prec) k_phys_from_ref<float><<<grid_for(n), 256, 0, st>>>(g, nx + 2, nz + 2, ref, (float*)dst);
  else k_phys_from_ref<double><<<grid_for(n), 256, 0, st>>>(g, nx + 2, nz + 2, ref, (double*)dst);
  return cudaGetLastError();
}

cudaError_t launch_phys_to_ref(const Geom& g, int nx, int nz, const void* src, double* ref, cudaStream_t st) {
  const long long n = (long long)g.np * g.pp;
  if (g.prec) k_phys_to_ref<float><<<grid_for(n), 256, 0, st>>>(g, nx + 2, nz + 2, (const float*)src, ref);
  else k_phys_to_ref<double><<<grid_for(n), 256, 0, st>>>(g, nx + 2, nz + 2, (const double*)src, ref);
  return cudaGetLastError();
}

}  // namespace db
