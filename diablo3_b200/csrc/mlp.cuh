// mlp.cuh -- interface of the learned-closure kernels (k_mlp.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace db {

struct LesRow;

// closure features computed from the physical fields of an LES substep
// (les_feat.cuh) instead of read from a feature array
struct LesFeatSrc {
  const void* f[12];      // u1 u2 u3 th, their d/dx, their d/dz: physical [j][z][x], FP32 or FP64
  const LesRow* lrow;     // per-row metrics
  long long pp;           // points per plane (Nx Nz)
  int ny;                 // Nyp
  double dxs, dzs;        // x, z filter widths
  const double* mean;     // plane means of u1 u2 u3 th ([f][Nyp+2]) when f[0..3] hold fluctuations, else null
};

struct MlpArgs {
  const float* feat;      // [n][16] raw features
  const float* target;    // [n][2] (training)
  float* out;             // [n][2] (inference)
  const float* params;    // DB_SGS_NPARAMS FP32
  const float* norm;      // mean[16], 1/std[16], out_scale[2]
  float* grads;           // DB_SGS_NPARAMS (training, accumulated)
  float* loss;            // sum of squared errors (training, accumulated)
  int n;                  // points (any count; the last tile is padded)
  int* err;               // set when a tensor-core wait gave up
  LesFeatSrc les;         // feature source of launch_mlp_les
};

cudaError_t launch_mlp(const MlpArgs& a, bool train, int max_ctas, cudaStream_t st);
// inference on the features of a.les (fields FP32 when fp32, else FP64);
// a.feat unused, a.n = planes x points per plane (row 0 gets zero features)
cudaError_t launch_mlp_les(const MlpArgs& a, bool fp32, cudaStream_t st);
cudaError_t launch_adam(float* params, float* grads, float* m1, float* m2, int n, float lr, int step,
                        cudaStream_t st);
cudaError_t launch_umma_gemm(const uint16_t* A, const uint16_t* B, float* D, int K, int N, int* err,
                             cudaStream_t st);

}  // namespace db

struct db_sgs_net;
// closure inference on a stream (no synchronisation), and the device
// training-range bounds lo[16], hi[16] of a network
int sgs_forward_async(db_sgs_net* n, const float* d_feat, float* d_out, long long npts, cudaStream_t st);
int sgs_forward_les_async(db_sgs_net* n, const db::LesFeatSrc& src, bool fp32, float* d_out, long long npts,
                          cudaStream_t st);
const float* sgs_range_dev(const db_sgs_net* n);
