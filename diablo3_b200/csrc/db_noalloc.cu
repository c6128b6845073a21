// db_noalloc.cu -- divergence removal that allocates nothing.
//
// Some callers cannot call cudaMalloc: a Fortran host whose device arrays
// are owned by another memory manager (CUDA Fortran / OpenACC pools), a code
// that must not allocate once its time loop runs (allocation can stall or
// fail under memory pressure), or a plugin inside a framework that forbids
// allocating behind its allocator.  db_rem_div_static serves them: it works
// directly on the caller's device arrays in the reference spectral layout
// and keeps its working memory in a file-scope device array whose size is
// fixed when the library is loaded (every GPU that loads the library holds
// those 8 MiB until the process exits).
//
// The scratch array is a device symbol: host code must not pass its name to
// a kernel (on the host the name is only a stand-in).  Its device address is
// fetched once per device with cudaGetSymbolAddress, on the first call made
// while that device is current; that first call should therefore come
// before any stream capture.  The grid GY is kept in the array too: a call
// copies the caller's (host, pageable) gy to the device only when its
// values or ny differ from the ones the previous call on that device left
// there.  Every call shares the array, so calls that overlap on the GPU
// (two streams, two threads) race; serialise them.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/diablo_b200.h"

namespace {

// 8 MiB: grid GY values + per chunk of columns the forward-sweep values g_j
// (complex) and 1/b'_j (real) of the Poisson Thomas solve.
constexpr long long kScratchBytes = 8ll << 20;
constexpr long long kScratchElems = kScratchBytes / 16;   // double2 entries
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_rd_scratch[kScratchElems];

std::mutex g_mu;
double2* g_scratch_ptr[kMaxDevices] = {};
// the GY values the scratch of each device holds (host copy; empty = none)
std::vector<double> g_gy_held[kMaxDevices];


struct RefGeomLite {
  int nyp, nkx, nkzp, nkz, nxp1, nz2;
  double two_pi_lx, two_pi_lz;   // 2 pi_ref / Lx, 2 pi_ref / Lz
  int chunk;                     // columns per launch
};

// GY(j) for j = 1..Nyp+1 is stored in scratch[0 .. Nyp] (.x); metrics as
// create_grid_chan builds them (for/domain.f90:276-300, 538-565).
__device__ __forceinline__ double gyv(const double2* s, int j) { return s[j - 1].x; }
__device__ __forceinline__ double gyf_in(const double2* s, int j) { return 0.5 * (gyv(s, j) + gyv(s, j + 1)); }
__device__ __forceinline__ double gyfv(const double2* s, int j, int nyp) {
  if (j == 0) return 2.0 * gyf_in(s, 1) - gyf_in(s, 2);
  if (j == nyp + 1) return 2.0 * gyf_in(s, nyp) - gyf_in(s, nyp - 1);
  return gyf_in(s, j);
}
__device__ __forceinline__ double dyv(const double2* s, int j, int nyp) {
  return gyfv(s, j, nyp) - gyfv(s, j - 1, nyp);
}
__device__ __forceinline__ double dyfv(const double2* s, int j, int nyp) {
  if (j == 0) j = 1;
  if (j == nyp + 1) j = nyp;
  return gyv(s, j + 1) - gyv(s, j);
}

// rem_div_chan (for/solver.f90:1302-1379) for one chunk of (kx, kz) columns,
// arrays in the reference layout cu(0:Nxp, 0:Nz+1, 0:Nyp+1).  The scratch
// of the chunk's columns is interleaved by column (row j of column t at
// j * chunk + t), so the loads and stores of a warp are contiguous.
__global__ void k_rem_div_static(double2* cu1, double2* cu2, double2* cu3, double2* scratch,
                                 RefGeomLite G, int col0) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = col0 + t;
  const int ncols = (G.nkx + 1) * G.nkzp;
  if (t >= G.chunk || col >= ncols) return;
  const int kx = col % (G.nkx + 1), kzp = col / (G.nkx + 1);
  const int nyp = G.nyp, np = nyp + 2;
  const long long cs = G.chunk;
  const double2* gys = scratch;                                   // GY values
  double2* gbuf = scratch + np + t;                               // g_j at gbuf[j cs]
  double* ibuf = (double*)(scratch + np + cs * np) + t;           // 1/b'_j at ibuf[j cs]
  const double kxv = kx * G.two_pi_lx;
  const double kzv = (kzp <= G.nkz ? kzp : kzp - G.nkzp) * G.two_pi_lz;
  const double kx2 = kxv * kxv, kz2 = kzv * kzv;
  const bool zero_mode = (kx == 0 && kzp == 0);
  const long long plane = (long long)G.nz2 * G.nxp1;
  const long long c0 = (long long)kzp * G.nxp1 + kx;
  // forward elimination: row 1 and row Nyp are the BC rows (solver.f90:2341-2368)
  double bprev = 1.0;                    // b'_1 = 1
  double uprev = zero_mode ? 0.0 : -1.0; // u_1
  double2 gp = make_double2(0.0, 0.0);
  gbuf[cs] = gp;
  ibuf[cs] = 1.0;
  for (int j = 2; j <= nyp; ++j) {
    double l, d, u;
    double2 rhs = make_double2(0.0, 0.0);
    if (j == nyp) {
      l = 1.0; d = -1.0; u = 0.0;
    } else {
      const double dyj = dyv(gys, j, nyp), dyj1 = dyv(gys, j + 1, nyp), dyfj = dyfv(gys, j, nyp);
      l = 1. / (dyj * dyfj);
      d = -kx2 - kz2 - 1. / (dyj1 * dyfj) - 1. / (dyj * dyfj);
      u = 1. / (dyj1 * dyfj);
      const double2 a1 = cu1[j * plane + c0], a3 = cu3[j * plane + c0];
      const double2 b0 = cu2[j * plane + c0], b1 = cu2[(j + 1) * plane + c0];
      rhs = make_double2(-kxv * a1.y + (b1.x - b0.x) / dyfj - kzv * a3.y,
                         kxv * a1.x + (b1.y - b0.y) / dyfj + kzv * a3.x);
    }
    const double a = -l / bprev;
    const double b = d + a * uprev;
    gp = make_double2(rhs.x + a * gp.x, rhs.y + a * gp.y);
    gbuf[j * cs] = gp;
    ibuf[j * cs] = 1.0 / b;
    bprev = b;
    uprev = u;
  }
  // back substitution with the projection (solver.f90:1347-1376)
  double2 phin = make_double2(0.0, 0.0);
  for (int j = nyp; j >= 1; --j) {
    double cj;
    if (j == nyp) cj = 0.0;
    else if (j == 1) cj = zero_mode ? 0.0 : -1.0;
    else cj = 1.0 / (dyv(gys, j + 1, nyp) * dyfv(gys, j, nyp));
    const double2 gj = gbuf[j * cs];
    const double ib = ibuf[j * cs];
    const double2 phi = make_double2((gj.x - cj * phin.x) * ib, (gj.y - cj * phin.y) * ib);
    const long long a = j * plane + c0;
    double2 v1 = cu1[a], v3 = cu3[a];
    v1.x += kxv * phi.y; v1.y -= kxv * phi.x;
    v3.x += kzv * phi.y; v3.y -= kzv * phi.x;
    cu1[a] = v1;
    cu3[a] = v3;
    if (j + 1 <= nyp) {
      const long long b = (j + 1) * plane + c0;
      const double w = 1.0 / dyv(gys, j + 1, nyp);
      double2 v2 = cu2[b];
      v2.x -= (phin.x - phi.x) * w;
      v2.y -= (phin.y - phi.y) * w;
      cu2[b] = v2;
    }
    phin = phi;
  }
}

}  // namespace

extern "C" int db_rem_div_static(const db_params* p, const double* gy, double* cu1, double* cu2,
                                 double* cu3, void* stream) {
  if (!p || !gy || !cu1 || !cu2 || !cu3) {
    return DB_ERR_ARG;
  }
  if (p->nx < 8 || p->nz < 8 || p->ny < 4 || p->lx <= 0 || p->lz <= 0) {
    return DB_ERR_ARG;
  }
  const int np = p->ny + 2;
  // scratch: np entries of GY, then chunk * np complex g plus chunk * np real 1/b'
  const long long per_col = (long long)np + ((long long)np + 1) / 2;
  const long long chunk_ll = (kScratchElems - np) / per_col;
  if (chunk_ll < 32) return DB_ERR_SIZE;  // ny > 10697 does not fit the static scratch
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    return DB_ERR_CUDA;
  }
  double2* scratch = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_rd_scratch);
      if (e != cudaSuccess) {
        return DB_ERR_CUDA;
      }
      g_scratch_ptr[dev] = (double2*)ptr;
    }
    scratch = g_scratch_ptr[dev];
    // GY(1:Nyp+1) into the first entries (.x), unless the previous call on
    // this device left the same values there; nothing else must start at
    // zero: every scratch entry a launch reads is written earlier in it
    std::vector<double>& held = g_gy_held[dev];
    const size_t ngy = (size_t)p->ny + 1;
    if (held.size() != ngy || !std::equal(held.begin(), held.end(), gy)) {
      e = cudaMemcpy2DAsync(scratch, sizeof(double2), gy, sizeof(double), sizeof(double), ngy,
                            cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) {
        held.clear();
        return DB_ERR_CUDA;
      }
      try {
        held.assign(gy, gy + ngy);
      } catch (...) {
        held.clear();   // copy again next time
      }
    }
  }
  RefGeomLite G;
  G.nyp = p->ny;
  G.nkx = p->nx / 3;
  G.nkz = p->nz / 3;
  G.nkzp = 2 * G.nkz + 1;
  G.nxp1 = p->nx / 2 + 1;
  G.nz2 = p->nz + 2;
  const double pi_ref = (double)(4.0f * atanf(1.0f));  // for/fft.f90:147
  G.two_pi_lx = (2. * pi_ref) / p->lx;
  G.two_pi_lz = (2. * pi_ref) / p->lz;
  const int ncols = (G.nkx + 1) * G.nkzp;
  G.chunk = (int)(chunk_ll < ncols ? chunk_ll : ncols);
  for (int c0 = 0; c0 < ncols; c0 += G.chunk) {
    k_rem_div_static<<<(G.chunk + 127) / 128, 128, 0, st>>>((double2*)cu1, (double2*)cu2, (double2*)cu3,
                                                           scratch, G, c0);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      return DB_ERR_CUDA;
    }
  }
  return DB_OK;
}
