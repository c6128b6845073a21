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

}  // namespace db
