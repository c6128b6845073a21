// db_sgs.cu -- C-ABI of the learned SGS closure (include/diablo_b200.h):
// device buffers of one network and the calls into k_mlp.cu.
#include <cuda_runtime.h>

#include <new>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/diablo_b200.h"

#include "mlp.cuh"

struct db_sgs_net {
  cudaStream_t st = nullptr;
  float* params = nullptr;   // FP32 master weights
  float* grads = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* norm = nullptr;     // mean[16], 1/std[16], out_scale[2]
  float* loss = nullptr;
  float* range = nullptr;    // lo[16], hi[16] of the training features
  int* err = nullptr;
  int step = 0;
  int sms = 148;
};

static int sgs_fail(cudaError_t e) { return e == cudaSuccess ? DB_OK : DB_ERR_CUDA; }
#define SCK(x)                                \
  do {                                        \
    cudaError_t e_ = (x);                     \
    if (e_ != cudaSuccess) return DB_ERR_CUDA; \
  } while (0)

extern "C" int db_sgs_create(void* stream, db_sgs_net** out) {
  if (!out) return DB_ERR_ARG;
  *out = nullptr;
  db_sgs_net* n = new (std::nothrow) db_sgs_net();
  if (!n) return DB_ERR_CUDA;   // host allocation failed (nothing may throw past the C-ABI)
  n->st = (cudaStream_t)stream;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t P = DB_SGS_NPARAMS * sizeof(float);
  if (cudaMalloc(&n->params, P) != cudaSuccess || cudaMalloc(&n->grads, P) != cudaSuccess ||
      cudaMalloc(&n->m1, P) != cudaSuccess || cudaMalloc(&n->m2, P) != cudaSuccess ||
      cudaMalloc(&n->norm, 64 * sizeof(float)) != cudaSuccess || cudaMalloc(&n->loss, sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->err, sizeof(int)) != cudaSuccess || cudaMalloc(&n->range, 32 * sizeof(float)) != cudaSuccess) {
    db_sgs_destroy(n);
    return DB_ERR_CUDA;
  }
  cudaMemset(n->params, 0, P);
  cudaMemset(n->grads, 0, P);
  cudaMemset(n->m1, 0, P);
  cudaMemset(n->m2, 0, P);
  cudaMemset(n->norm, 0, 64 * sizeof(float));
  cudaMemset(n->err, 0, sizeof(int));
  {
    float r[32];
    for (int f = 0; f < 16; ++f) { r[f] = -3.0e38f; r[16 + f] = 3.0e38f; }   // no fallback until set
    cudaMemcpy(n->range, r, sizeof(r), cudaMemcpyHostToDevice);
  }
  *out = n;
  return DB_OK;
}

extern "C" int db_sgs_destroy(db_sgs_net* n) {
  if (!n) return DB_ERR_ARG;
  if (n->st) cudaStreamSynchronize(n->st);
  cudaFree(n->params);
  cudaFree(n->grads);
  cudaFree(n->m1);
  cudaFree(n->m2);
  cudaFree(n->norm);
  cudaFree(n->loss);
  cudaFree(n->err);
  cudaFree(n->range);
  delete n;
  return DB_OK;
}

extern "C" int db_sgs_set(db_sgs_net* n, const float* params, const float* mean, const float* std_,
                          const float* out_scale) {
  if (!n || !params || !mean || !std_ || !out_scale) return DB_ERR_ARG;
  float norm[2 * DB_SGS_NFEAT + 2];
  for (int f = 0; f < DB_SGS_NFEAT; ++f) {
    if (!(std_[f] > 0.0f)) return DB_ERR_ARG;
    norm[f] = mean[f];
    norm[DB_SGS_NFEAT + f] = 1.0f / std_[f];
  }
  norm[2 * DB_SGS_NFEAT] = out_scale[0];
  norm[2 * DB_SGS_NFEAT + 1] = out_scale[1];
  const size_t P = DB_SGS_NPARAMS * sizeof(float);
  SCK(cudaMemcpyAsync(n->params, params, P, cudaMemcpyHostToDevice, n->st));
  SCK(cudaMemcpyAsync(n->norm, norm, sizeof(norm), cudaMemcpyHostToDevice, n->st));
  SCK(cudaMemsetAsync(n->grads, 0, P, n->st));
  SCK(cudaMemsetAsync(n->m1, 0, P, n->st));
  SCK(cudaMemsetAsync(n->m2, 0, P, n->st));
  SCK(cudaStreamSynchronize(n->st));
  n->step = 0;
  return DB_OK;
}

extern "C" int db_sgs_set_range(db_sgs_net* n, const float* lo, const float* hi) {
  if (!n || !lo || !hi) return DB_ERR_ARG;
  float r[32];
  for (int f = 0; f < 16; ++f) {
    if (!(lo[f] <= hi[f])) return DB_ERR_ARG;
    r[f] = lo[f];
    r[16 + f] = hi[f];
  }
  SCK(cudaMemcpyAsync(n->range, r, sizeof(r), cudaMemcpyHostToDevice, n->st));
  SCK(cudaStreamSynchronize(n->st));
  return DB_OK;
}

const float* sgs_range_dev(const db_sgs_net* n) { return n->range; }

extern "C" int db_sgs_get(db_sgs_net* n, float* params) {
  if (!n || !params) return DB_ERR_ARG;
  SCK(cudaMemcpyAsync(params, n->params, DB_SGS_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost, n->st));
  SCK(cudaStreamSynchronize(n->st));
  return DB_OK;
}

static int check_err(db_sgs_net* n) {
  int e = 0;
  SCK(cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->st));
  SCK(cudaStreamSynchronize(n->st));
  return e ? DB_ERR_TIMEOUT : DB_OK;
}

// issue the forward pass on the net's stream (no synchronisation)
int sgs_forward_async(db_sgs_net* n, const float* d_feat, float* d_out, long long npts, cudaStream_t st) {
  if (npts > 0x7fffffffLL) return DB_ERR_SIZE;
  db::MlpArgs a{d_feat, nullptr, d_out, n->params, n->norm, nullptr, nullptr, (int)npts, n->err};
  return sgs_fail(db::launch_mlp(a, false, 4 * n->sms, st));
}

int sgs_forward_les_async(db_sgs_net* n, const db::LesFeatSrc& src, bool fp32, float* d_out, long long npts,
                          cudaStream_t st) {
  if (npts > 0x7fffffffLL) return DB_ERR_SIZE;
  db::MlpArgs a{nullptr, nullptr, d_out, n->params, n->norm, nullptr, nullptr, (int)npts, n->err, src};
  return sgs_fail(db::launch_mlp_les(a, fp32, st));
}

extern "C" int db_sgs_forward(db_sgs_net* n, const float* d_feat, float* d_out, long long npts) {
  if (!n || !d_feat || !d_out || npts < 0) return DB_ERR_ARG;
  int rc = sgs_forward_async(n, d_feat, d_out, npts, n->st);
  if (rc) return rc;
  return check_err(n);
}

static int grad_pass(db_sgs_net* n, const float* d_feat, const float* d_target, long long npts, double* loss) {
  if (npts > 0x7fffffffLL) return DB_ERR_SIZE;
  SCK(cudaMemsetAsync(n->loss, 0, sizeof(float), n->st));
  db::MlpArgs a{d_feat, d_target, nullptr, n->params, n->norm, n->grads, n->loss, (int)npts, n->err};
  SCK(db::launch_mlp(a, true, n->sms, n->st));
  if (loss) {
    float l = 0.0f;
    SCK(cudaMemcpyAsync(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->st));
    SCK(cudaStreamSynchronize(n->st));
    *loss = (double)l / (double)npts;
  }
  return check_err(n);
}

extern "C" int db_sgs_gradient(db_sgs_net* n, const float* d_feat, const float* d_target, long long npts,
                               float* grads, double* loss) {
  if (!n || !d_feat || !d_target || !grads || npts <= 0) return DB_ERR_ARG;
  const size_t P = DB_SGS_NPARAMS * sizeof(float);
  SCK(cudaMemsetAsync(n->grads, 0, P, n->st));
  int rc = grad_pass(n, d_feat, d_target, npts, loss);
  if (rc) return rc;
  SCK(cudaMemcpyAsync(grads, n->grads, P, cudaMemcpyDeviceToHost, n->st));
  SCK(cudaMemsetAsync(n->grads, 0, P, n->st));
  SCK(cudaStreamSynchronize(n->st));
  return DB_OK;
}

extern "C" int db_sgs_train_step(db_sgs_net* n, const float* d_feat, const float* d_target, long long npts,
                                 float lr, double* loss) {
  if (!n || !d_feat || !d_target || npts <= 0 || !(lr > 0.0f)) return DB_ERR_ARG;
  int rc = grad_pass(n, d_feat, d_target, npts, loss);
  if (rc) return rc;
  n->step += 1;
  SCK(db::launch_adam(n->params, n->grads, n->m1, n->m2, DB_SGS_NPARAMS, lr, n->step, n->st));
  SCK(cudaStreamSynchronize(n->st));
  return DB_OK;
}

extern "C" int db_sgs_gemm_check(const uint16_t* A, const uint16_t* B, float* D, int K, int N) {
  if (!A || !B || !D || K < 16 || K > 256 || (K % 16) || N < 16 || N > 256 || (N % 16)) return DB_ERR_ARG;
  uint16_t *dA = nullptr, *dB = nullptr;
  float* dD = nullptr;
  int* derr = nullptr;
  int rc = DB_OK;
  if (cudaMalloc(&dA, 128 * K * 2) != cudaSuccess || cudaMalloc(&dB, N * K * 2) != cudaSuccess ||
      cudaMalloc(&dD, 128 * N * 4) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
    rc = DB_ERR_CUDA;
  } else {
    cudaMemset(derr, 0, sizeof(int));
    cudaMemcpy(dA, A, 128 * K * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, N * K * 2, cudaMemcpyHostToDevice);
    if (db::launch_umma_gemm(dA, dB, dD, K, N, derr, 0) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
      rc = DB_ERR_CUDA;
    } else {
      int e = 0;
      cudaMemcpy(&e, derr, sizeof(int), cudaMemcpyDeviceToHost);
      cudaMemcpy(D, dD, 128 * N * 4, cudaMemcpyDeviceToHost);
      if (e) rc = DB_ERR_TIMEOUT;
    }
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(derr);
  return rc;
}

