// k_mlp.cu -- learned SGS closure: a 16 -> 64 -> 64 -> 64 -> 2 MLP (GELU
// hidden layers, softplus outputs nu_t, kappa_t >= 0) on the 5th-generation
// tensor cores.  BF16 weights and activations, FP32 accumulation in tensor
// memory (umma.cuh), FP32 master weights and Adam.
//
// One CTA of 128 threads works on tiles of 128 points; thread t owns point
// (row) t of the tile and reads row t of every accumulator from tensor
// memory.  k_mlp_train runs the forward and backward passes; k_mlp_infer the
// forward pass only, its features read from an array or formed from the LES
// substep's physical fields.
//   forward   X W1^T -> z1 -> h1 = gelu(z1) (tanh form) -> h1 W2^T -> z2 -> ... -> h3,
//             y = W4 h3 + b4 on CUDA cores (N = 2), out = softplus(y) * scale
//   backward  (training) dy = dL/dy; dh3 = dy W4, dz3 = dh3 gelu'(z3);
//             [dW3 | db3] += dz3^T [h2 | 1]   (tensor core, M padded to 128)
//             dh2 = dz3 W3                     (tensor core)
//             z2 is recomputed by the tensor core instead of being stored;
//             likewise down to [dW1 | db1] += dz1^T [x | 1].
//             dW4, db4 by warp reductions.  The loss is the mean square error
//             of the scaled outputs against the targets.
// Gradients are summed over the CTA's tiles in tensor memory and added to a
// global FP32 buffer once per CTA.
#include <cuda_bf16.h>
#include <math.h>

#include <type_traits>

#include "../../include/diablo_b200.h"
#include "les_feat.cuh"
#include "mlp.cuh"
#include "umma.cuh"

namespace db {

constexpr int NF = 16, NH = 64, NO = 2, TILE = 128;
// parameter packing (FP32): W1[64][16] b1 W2[64][64] b2 W3[64][64] b3 W4[2][64] b4
constexpr int P_W1 = 0, P_B1 = 1024, P_W2 = 1088, P_B2 = 5184, P_W3 = 5248, P_B3 = 9344, P_W4 = 9408,
              P_B4 = 9536, P_TOTAL = 9538;
static_assert(P_TOTAL == DB_SGS_NPARAMS, "parameter count");



// GELU in its tanh form (Hendrycks & Gimpel 2016),
//   gelu(x) = x/2 (1 + tanh(u)),  u = sqrt(2/pi) (x + 0.044715 x^3),
// with the hardware tanh approximation (relative error ~5e-4, below the
// BF16 rounding of the activations); the hidden-layer epilogues are the
// closure's CUDA-core bottleneck, so the activation must be cheap.
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float GELU_K = 0.7978845608028654f;   // sqrt(2 / pi)
constexpr float GELU_C = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
  const float t = tanh_hw(GELU_K * x * (1.0f + GELU_C * x * x));
  return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_d(float x) {
  const float x2 = x * x;
  const float t = tanh_hw(GELU_K * x * (1.0f + GELU_C * x2));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * GELU_K * (1.0f + 3.0f * GELU_C * x2);
}
__device__ __forceinline__ float softplus(float y) { return y > 20.0f ? y : log1pf(expf(y)); }
__device__ __forceinline__ float sigm(float y) { return 1.0f / (1.0f + expf(-y)); }

// a in the low half, b in the high half, each rounded to nearest; the
// paired conversion is one instruction for the two values
__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// 8 consecutive K values of one row into a K-major tile (one 16-byte store)
__device__ __forceinline__ void put8(unsigned char* tile, int row, int k0, int K, const float* v) {
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + kmajor_offset(row, k0, K)) = q;
}
__device__ __forceinline__ void put1(unsigned char* tile, int row, int k, int K, float v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + kmajor_offset(row, k, K)) = __float2bfloat16_rn(v);
}

// shared-memory plan of the training kernel (bytes): the forward tiles, the
// transposed tiles and the gradient operands
struct PlanTrain {
  static constexpr uint32_t X = 0;                                     // [128][16]
  static constexpr uint32_t H1 = X + TILE * NF * 2;                    // [128][64]
  static constexpr uint32_t H2 = H1 + TILE * NH * 2;                   // [128][64]
  static constexpr uint32_t W1 = H2 + TILE * NH * 2;                   // [64][16]
  static constexpr uint32_t W2 = W1 + NH * NF * 2;                     // [64][64]
  static constexpr uint32_t W3 = W2 + NH * NH * 2;                     // [64][64]
  static constexpr uint32_t XT = W3 + NH * NH * 2;                     // [32][128]: x^T, ones row, zeros
  static constexpr uint32_t H1T = XT + 32 * TILE * 2;                  // [80][128]: h1^T, ones, zeros
  static constexpr uint32_t H2T = H1T + 80 * TILE * 2;                 // [80][128]
  static constexpr uint32_t DZ = H2T + 80 * TILE * 2;                 // [128][64] dz
  static constexpr uint32_t DZT = DZ + TILE * NH * 2;                  // [128][128] dz^T (rows >= 64 zero)
  static constexpr uint32_t W2T = DZT + TILE * TILE * 2; // [64][64] W2^T
  static constexpr uint32_t W3T = W2T + NH * NH * 2;                   // [64][64] W3^T
  static constexpr uint32_t RED = W3T + NH * NH * 2;                   // dW4, db4 partial sums (floats)
  static constexpr uint32_t MBAR = RED + 136 * 4;
  static constexpr uint32_t SLOT = MBAR + 8;
  static constexpr uint32_t BYTES = SLOT + 8;
  static constexpr uint32_t TMEM_COLS = 512;
  // tensor-memory columns: z accumulator, dh accumulator, [dW3|db3], [dW2|db2], [dW1|db1]
  static constexpr uint32_t C_Z = 0, C_H = 64, C_G3 = 128, C_G2 = 256, C_G1 = 384;
};

constexpr uint32_t WAIT_ITERS = 1u << 22;   // bounded mbarrier waits

__global__ void __launch_bounds__(TILE, 1) k_mlp_train(MlpArgs a) {
  using PL = PlanTrain;
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + PL::MBAR);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + PL::SLOT);
  const float* P = a.params;

  // ---- weights to shared memory (BF16, K-major), once per CTA
  for (int r = t; r < NH; r += TILE) {
    float v[8];
    for (int k0 = 0; k0 < NF; k0 += 8) {
      for (int i = 0; i < 8; ++i) v[i] = P[P_W1 + r * NF + k0 + i];
      put8(sm + PL::W1, r, k0, NF, v);
    }
    for (int k0 = 0; k0 < NH; k0 += 8) {
      for (int i = 0; i < 8; ++i) v[i] = P[P_W2 + r * NH + k0 + i];
      put8(sm + PL::W2, r, k0, NH, v);
      for (int i = 0; i < 8; ++i) v[i] = P[P_W3 + r * NH + k0 + i];
      put8(sm + PL::W3, r, k0, NH, v);
      // transposes: row r = input index, K = output index
      for (int i = 0; i < 8; ++i) v[i] = P[P_W2 + (k0 + i) * NH + r];
      put8(sm + PL::W2T, r, k0, NH, v);
      for (int i = 0; i < 8; ++i) v[i] = P[P_W3 + (k0 + i) * NH + r];
      put8(sm + PL::W3T, r, k0, NH, v);
    }
  }
  // constant rows of the transposed operands: ones row (bias gradients),
  // zero padding, and the zero upper half of dz^T
  for (int m = t; m < TILE; m += TILE) {
    put1(sm + PL::XT, NF, m, TILE, 1.0f);
    for (int r = NF + 1; r < 32; ++r) put1(sm + PL::XT, r, m, TILE, 0.0f);
    put1(sm + PL::H1T, NH, m, TILE, 1.0f);
    put1(sm + PL::H2T, NH, m, TILE, 1.0f);
    for (int r = NH + 1; r < 80; ++r) {
      put1(sm + PL::H1T, r, m, TILE, 0.0f);
      put1(sm + PL::H2T, r, m, TILE, 0.0f);
    }
    for (int r = NH; r < TILE; ++r) put1(sm + PL::DZT, r, m, TILE, 0.0f);
  }
  float* red = reinterpret_cast<float*>(sm + PL::RED);
  for (int i = t; i < 136; i += TILE) red[i] = 0.0f;
  if (t == 0) mbar_init(mbar, 1);
  if (warp == 0) {
    tmem_alloc(slot, PL::TMEM_COLS);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *slot;
  const uint32_t trow = tbase + ((uint32_t)(warp * 32) << 16);   // this warp's lanes
  uint32_t phase = 0;
  bool ok = true;

  const float* mu = a.norm;
  const float* isd = a.norm + NF;
  const float osc0 = a.norm[2 * NF], osc1 = a.norm[2 * NF + 1];
  const uint32_t id64 = umma_idesc_bf16(128, NH), id80 = umma_idesc_bf16(128, 80), id32 = umma_idesc_bf16(128, 32);
  const uint32_t aX = smem_u32(sm + PL::X), aH1 = smem_u32(sm + PL::H1), aH2 = smem_u32(sm + PL::H2);
  const uint32_t aW1 = smem_u32(sm + PL::W1), aW2 = smem_u32(sm + PL::W2), aW3 = smem_u32(sm + PL::W3);

  // issue a GEMM D (+)= A B^T over K (steps of 16) by thread 0
  auto gemm = [&](uint32_t dcol, uint32_t a_addr, uint32_t a_sbo, uint32_t b_addr, uint32_t b_sbo, int K,
                  uint32_t idesc, bool acc) {
    for (int s = 0; s < K / 16; ++s)
      umma_bf16(tbase + dcol, umma_desc(a_addr + 256 * s, 128, a_sbo), umma_desc(b_addr + 256 * s, 128, b_sbo),
                idesc, acc || s > 0);
  };
  // commit, wait, and agree on the outcome (a wait that gave up leaves the
  // layer pending for the drain at the end)
  bool pend = false;
  auto sync_mma = [&]() -> bool {
    if (t == 0) umma_commit(mbar);
    const bool w = mbar_wait(mbar, phase, WAIT_ITERS);
    if (w) phase ^= 1u;
    else pend = true;
    tc_fence_after();
    return __syncthreads_and(w ? 1 : 0) != 0;
  };
  // epilogue of a hidden layer: row of z from tensor memory -> h = gelu(z)
  // into the next A tile (and its transpose when training)
  auto hidden_out = [&](const float* bias, unsigned char* tileA, unsigned char* tileT) {
    for (int c = 0; c < NH; c += 16) {
      float z[16];
      tmem_ld16(trow + PL::C_Z + c, z);
      tmem_wait_ld();
      float h[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) h[i] = gelu(z[i] + bias[c + i]);
      put8(tileA, t, c, NH, h);
      put8(tileA, t, c + 8, NH, h + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) put1(tileT, c + i, t, TILE, h[i]);
    }
  };

  __shared__ float sb[3 * NH + NO + NO * NH];   // b1 b2 b3 b4 W4 (FP32)
  for (int i = t; i < NH; i += TILE) {
    sb[i] = P[P_B1 + i];
    sb[NH + i] = P[P_B2 + i];
    sb[2 * NH + i] = P[P_B3 + i];
  }
  for (int i = t; i < NO * NH; i += TILE) sb[3 * NH + NO + i] = P[P_W4 + i];
  if (t < NO) sb[3 * NH + t] = P[P_B4 + t];
  __syncthreads();
  const float* b1 = sb;
  const float* b2 = sb + NH;
  const float* b3 = sb + 2 * NH;
  const float* b4 = sb + 3 * NH;
  const float* W4 = sb + 3 * NH + NO;

  float lsum = 0.0f;
  bool first = true;
  const int ntiles = (a.n + TILE - 1) / TILE;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int p = tile * TILE + t;
    const bool live = p < a.n;
    // ---- features, normalised, to BF16
    float x[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) x[f] = live ? (a.feat[(long long)p * NF + f] - mu[f]) * isd[f] : 0.0f;
    put8(sm + PL::X, t, 0, NF, x);
    put8(sm + PL::X, t, 8, NF, x + 8);
#pragma unroll
    for (int f = 0; f < NF; ++f) put1(sm + PL::XT, f, t, TILE, x[f]);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- layer 1..3
    if (t == 0) gemm(PL::C_Z, aX, NF * 16, aW1, NF * 16, NF, id64, false);
    if (!(ok = sync_mma())) break;
    hidden_out(b1, sm + PL::H1, sm + PL::H1T);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t == 0) gemm(PL::C_Z, aH1, NH * 16, aW2, NH * 16, NH, id64, false);
    if (!(ok = sync_mma())) break;
    hidden_out(b2, sm + PL::H2, sm + PL::H2T);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t == 0) gemm(PL::C_Z, aH2, NH * 16, aW3, NH * 16, NH, id64, false);
    if (!(ok = sync_mma())) break;
    // ---- output layer on CUDA cores (z3 stays in tensor memory)
    float y0 = b4[0], y1 = b4[1];
    for (int c = 0; c < NH; c += 16) {
      float z[16];
      tmem_ld16(trow + PL::C_Z + c, z);
      tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float h = gelu(z[i] + b3[c + i]);
        y0 += W4[c + i] * h;
        y1 += W4[NH + c + i] * h;
      }
    }
    const float s0 = softplus(y0) * osc0, s1 = softplus(y1) * osc1;
    // ---- loss and dL/dy (mean over the batch of the squared error)
    float dy0 = 0.0f, dy1 = 0.0f;
    if (live) {
      const float e0 = s0 - a.target[(long long)p * 2], e1 = s1 - a.target[(long long)p * 2 + 1];
      lsum += e0 * e0 + e1 * e1;
      const float g = 2.0f / (float)a.n;
      dy0 = g * e0 * osc0 * sigm(y0);
      dy1 = g * e1 * osc1 * sigm(y1);
    }
    float* red = reinterpret_cast<float*>(sm + PL::RED);
    {   // db4
      float r0 = dy0, r1 = dy1;
      for (int o = 16; o > 0; o >>= 1) {
        r0 += __shfl_xor_sync(0xffffffffu, r0, o);
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
      }
      if (lane == 0) {
        atomicAdd(&red[128], r0);
        atomicAdd(&red[129], r1);
      }
    }
    // dh3 = dy W4, dz3 = dh3 gelu'(z3); dW4 += dy h3 (warp sums)
    for (int c = 0; c < NH; c += 16) {
      float z[16];
      tmem_ld16(trow + PL::C_Z + c, z);
      tmem_wait_ld();
      float dz[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float zz = z[i] + b3[c + i];
        const float h = gelu(zz);
        float g0 = dy0 * h, g1 = dy1 * h;
        for (int o = 16; o > 0; o >>= 1) {
          g0 += __shfl_xor_sync(0xffffffffu, g0, o);
          g1 += __shfl_xor_sync(0xffffffffu, g1, o);
        }
        if (lane == 0) {
          atomicAdd(&red[c + i], g0);
          atomicAdd(&red[NH + c + i], g1);
        }
        dz[i] = (dy0 * W4[c + i] + dy1 * W4[NH + c + i]) * gelu_d(zz);
      }
      put8(sm + PL::DZ, t, c, NH, dz);
      put8(sm + PL::DZ, t, c + 8, NH, dz + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) put1(sm + PL::DZT, c + i, t, TILE, dz[i]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t aDZ = smem_u32(sm + PL::DZ), aDZT = smem_u32(sm + PL::DZT);
    if (t == 0) {
      gemm(PL::C_G3, aDZT, TILE * 16, smem_u32(sm + PL::H2T), TILE * 16, TILE, id80, !first);   // [dW3|db3]
      gemm(PL::C_H, aDZ, NH * 16, smem_u32(sm + PL::W3T), NH * 16, NH, id64, false);           // dh2
      gemm(PL::C_Z, aH1, NH * 16, aW2, NH * 16, NH, id64, false);                               // z2 again
    }
    if (!(ok = sync_mma())) break;
    // dz2 = dh2 gelu'(z2)
    for (int c = 0; c < NH; c += 16) {
      float z[16], dh[16];
      tmem_ld16(trow + PL::C_Z + c, z);
      tmem_ld16(trow + PL::C_H + c, dh);
      tmem_wait_ld();
      float dz[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) dz[i] = dh[i] * gelu_d(z[i] + b2[c + i]);
      put8(sm + PL::DZ, t, c, NH, dz);
      put8(sm + PL::DZ, t, c + 8, NH, dz + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) put1(sm + PL::DZT, c + i, t, TILE, dz[i]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t == 0) {
      gemm(PL::C_G2, aDZT, TILE * 16, smem_u32(sm + PL::H1T), TILE * 16, TILE, id80, !first);   // [dW2|db2]
      gemm(PL::C_H, aDZ, NH * 16, smem_u32(sm + PL::W2T), NH * 16, NH, id64, false);           // dh1
      gemm(PL::C_Z, aX, NF * 16, aW1, NF * 16, NF, id64, false);                                // z1 again
    }
    if (!(ok = sync_mma())) break;
    // dz1 = dh1 gelu'(z1) -> dz1^T only
    for (int c = 0; c < NH; c += 16) {
      float z[16], dh[16];
      tmem_ld16(trow + PL::C_Z + c, z);
      tmem_ld16(trow + PL::C_H + c, dh);
      tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) put1(sm + PL::DZT, c + i, t, TILE, dh[i] * gelu_d(z[i] + b1[c + i]));
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t == 0) gemm(PL::C_G1, aDZT, TILE * 16, smem_u32(sm + PL::XT), TILE * 16, TILE, id32, !first);  // [dW1|db1]
    if (!(ok = sync_mma())) break;
    first = false;
  }

  if (ok && !first) {
    // gradients of this CTA: rows 0..63 of the accumulators are lanes 0..63
    if (warp < 2) {
      const int o = t;   // output unit
      float v[16];
      for (int c = 0; c < 80; c += 16) {
        tmem_ld16(trow + PL::C_G3 + c, v);
        tmem_wait_ld();
        for (int i = 0; i < 16; ++i) {
          const int col = c + i;
          if (col < NH) atomicAdd(&a.grads[P_W3 + o * NH + col], v[i]);
          else if (col == NH) atomicAdd(&a.grads[P_B3 + o], v[i]);
        }
        tmem_ld16(trow + PL::C_G2 + c, v);
        tmem_wait_ld();
        for (int i = 0; i < 16; ++i) {
          const int col = c + i;
          if (col < NH) atomicAdd(&a.grads[P_W2 + o * NH + col], v[i]);
          else if (col == NH) atomicAdd(&a.grads[P_B2 + o], v[i]);
        }
      }
      for (int c = 0; c < 32; c += 16) {
        tmem_ld16(trow + PL::C_G1 + c, v);
        tmem_wait_ld();
        for (int i = 0; i < 16; ++i) {
          const int col = c + i;
          if (col < NF) atomicAdd(&a.grads[P_W1 + o * NF + col], v[i]);
          else if (col == NF) atomicAdd(&a.grads[P_B1 + o], v[i]);
        }
      }
    }
    __syncthreads();
    const float* red = reinterpret_cast<const float*>(sm + PL::RED);
    for (int i = t; i < NO * NH; i += TILE) atomicAdd(&a.grads[P_W4 + i], red[i]);
    if (t < NO) atomicAdd(&a.grads[P_B4 + t], red[128 + t]);
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0 && lsum != 0.0f) atomicAdd(a.loss, lsum);
  if (!ok && t == 0) {
    atomicExch(a.err, 1);
    // the layer still in flight (bounded) before freeing; should this wait
    // give up too, the tensor memory is freed all the same: a CTA that kept
    // it would leave later CTAs on its SM waiting in tcgen05.alloc, and the
    // flag already marks this launch's outputs invalid
    if (pend) mbar_wait(mbar, phase, WAIT_ITERS);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tbase, PL::TMEM_COLS);
}

// Adam (bias-corrected) on the FP32 master weights; grads are consumed and zeroed
// ---------------------------------------------------------------------------
// Inference.  Same arithmetic as the forward half of k_mlp (BF16 operands,
// FP32 accumulation, the same rounding points), laid out for throughput:
// the X tile aliases the start of the H tile (layer 1 has finished reading X
// when its epilogue writes H, and layers 2 and 3 have finished reading H
// when the next epilogue or the next tile writes it), so a CTA needs 35 KB of
// shared memory and six CTAs share an SM, whose tiles overlap one another's
// tensor-core waits.  SRC 0 reads features from a.feat; SRC 1 / 2 form them
// from the LES substep's FP32 / FP64 physical fields (les_feat.cuh), point
// p = j * pp + col of GY row j, row 0 getting zero features.
struct PlanInf {
  static constexpr uint32_t H = 0;                       // [128][64]; X [128][16] at its start
  static constexpr uint32_t W1 = H + TILE * NH * 2;      // [64][16]
  static constexpr uint32_t W2 = W1 + NH * NF * 2;       // [64][64]
  static constexpr uint32_t W3 = W2 + NH * NH * 2;       // [64][64]
  static constexpr uint32_t MBAR = W3 + NH * NH * 2;
  static constexpr uint32_t SLOT = MBAR + 8;
  static constexpr uint32_t BYTES = SLOT + 8;
  static constexpr uint32_t TMEM_COLS = 64;
};
constexpr int INF_CTAS_PER_SM = 6;

// biases, output weights interleaved per hidden unit, feature normalisation
struct __align__(16) InfConst {
  float b[3][NH];
  float2 w4[NH];   // (W4[0][i], W4[1][i])
  float b4[4];     // b4[0..1], padding
  float mu[NF], isd[NF];
};

// packed FP32 pair arithmetic (the f32x2 instructions of sm_100): one
// instruction rounds each lane exactly like its scalar form
__device__ __forceinline__ uint64_t f2(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2split(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
// gelu of two pre-activations z + c (the tanh form of gelu(), two lanes at
// a time: x = z + c, u = K x (1 + C x^2), h = x/2 + x/2 tanh(u))
__device__ __forceinline__ void gelu_pair(float z0, float z1, float c0, float c1, float& h0, float& h1) {
  const uint64_t x = add2(f2(z0, z1), f2(c0, c1));
  const uint64_t w = fma2(mul2(x, x), f2(GELU_C, GELU_C), f2(1.0f, 1.0f));
  const uint64_t u = mul2(mul2(x, f2(GELU_K, GELU_K)), w);
  float u0, u1;
  f2split(u, u0, u1);
  const uint64_t hx = mul2(x, f2(0.5f, 0.5f));
  const uint64_t hh = fma2(hx, f2(tanh_hw(u0), tanh_hw(u1)), hx);
  f2split(hh, h0, h1);
}
static_assert(INF_CTAS_PER_SM * PlanInf::TMEM_COLS <= 512, "tensor memory of the resident CTAs");

template <int SRC>
__global__ void __launch_bounds__(TILE, INF_CTAS_PER_SM) k_mlp_infer(MlpArgs a) {
  using PL = PlanInf;
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, warp = t >> 5;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + PL::MBAR);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + PL::SLOT);
  const float* P = a.params;
  for (int r = t; r < NH; r += TILE) {
    float v[8];
    for (int k0 = 0; k0 < NF; k0 += 8) {
      for (int i = 0; i < 8; ++i) v[i] = P[P_W1 + r * NF + k0 + i];
      put8(sm + PL::W1, r, k0, NF, v);
    }
    for (int k0 = 0; k0 < NH; k0 += 8) {
      for (int i = 0; i < 8; ++i) v[i] = P[P_W2 + r * NH + k0 + i];
      put8(sm + PL::W2, r, k0, NH, v);
      for (int i = 0; i < 8; ++i) v[i] = P[P_W3 + r * NH + k0 + i];
      put8(sm + PL::W3, r, k0, NH, v);
    }
  }
  __shared__ InfConst cs;
  for (int i = t; i < NH; i += TILE) {
    cs.b[0][i] = P[P_B1 + i];
    cs.b[1][i] = P[P_B2 + i];
    cs.b[2][i] = P[P_B3 + i];
    cs.w4[i] = make_float2(P[P_W4 + i], P[P_W4 + NH + i]);
  }
  if (t < NO) cs.b4[t] = P[P_B4 + t];
  if (t < NF) {
    cs.mu[t] = a.norm[t];
    cs.isd[t] = a.norm[NF + t];
  }
  if (t == 0) mbar_init(mbar, 1);
  if (warp == 0) {
    tmem_alloc(slot, PL::TMEM_COLS);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *slot;
  const uint32_t trow = tbase + ((uint32_t)(warp * 32) << 16);
  const float osc0 = a.norm[2 * NF], osc1 = a.norm[2 * NF + 1];
  const uint32_t id64 = umma_idesc_bf16(128, NH);
  const uint32_t aH = smem_u32(sm + PL::H);
  const uint32_t aW1 = smem_u32(sm + PL::W1), aW2 = smem_u32(sm + PL::W2), aW3 = smem_u32(sm + PL::W3);
  uint32_t phase = 0;
  bool ok = true;
  auto gemm = [&](uint32_t a_addr, uint32_t a_sbo, uint32_t b_addr, uint32_t b_sbo, int K) {
    for (int s = 0; s < K / 16; ++s)
      umma_bf16(tbase, umma_desc(a_addr + 256 * s, 128, a_sbo), umma_desc(b_addr + 256 * s, 128, b_sbo), id64,
                s > 0);
  };
  // operands written by this CTA's threads are visible to the tensor core,
  // and every thread's earlier tensor-memory reads are done, before t0 issues
  auto to_tc = [&]() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  };
  bool pend = false;   // a layer whose wait gave up (thread 0's view)
  auto sync_mma = [&]() -> bool {
    if (t == 0) umma_commit(mbar);
    const bool w = mbar_wait(mbar, phase, WAIT_ITERS);
    if (w) phase ^= 1u;
    else pend = true;
    tc_fence_after();
    return __syncthreads_and(w ? 1 : 0) != 0;
  };
  // gelu(z + bias) of 16 columns from c, bias read four at a time
  auto gelu16 = [&](const float (&z)[16], const float* bias, float (&h)[16]) {
#pragma unroll
    for (int i = 0; i < 16; i += 4) {
      const float4 b = *reinterpret_cast<const float4*>(bias + i);
      gelu_pair(z[i], z[i + 1], b.x, b.y, h[i], h[i + 1]);
      gelu_pair(z[i + 2], z[i + 3], b.z, b.w, h[i + 2], h[i + 3]);
    }
  };
  auto hidden_out = [&](const float* bias) {
#pragma unroll
    for (int c = 0; c < NH; c += 32) {
      float z0[16], z1[16];
      tmem_ld16(trow + c, z0);
      tmem_ld16(trow + c + 16, z1);
      tmem_wait_ld();
      float h[16];
      gelu16(z0, bias + c, h);
      put8(sm + PL::H, t, c, NH, h);
      put8(sm + PL::H, t, c + 8, NH, h + 8);
      gelu16(z1, bias + c + 16, h);
      put8(sm + PL::H, t, c + 16, NH, h);
      put8(sm + PL::H, t, c + 24, NH, h + 8);
    }
  };

  const int ntiles = (a.n + TILE - 1) / TILE;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int p = tile * TILE + t;
    const bool live = p < a.n;
    float fv[NF];
    if constexpr (SRC == 0) {
#pragma unroll
      for (int f = 0; f < NF; ++f) fv[f] = live ? a.feat[(long long)p * NF + f] : 0.0f;
    } else {
      const int j = live ? (int)(p / a.les.pp) : 0;
#pragma unroll
      for (int f = 0; f < NF; ++f) fv[f] = 0.0f;
      if (j >= 1) les_features_at<typename std::conditional<SRC == 1, float, double>::type>(
                      a.les, j, p - (long long)j * a.les.pp, fv);
    }
    float x[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) x[f] = live ? (fv[f] - cs.mu[f]) * cs.isd[f] : 0.0f;
    put8(sm + PL::H, t, 0, NF, x);       // X tile (K = 16) at the start of H
    put8(sm + PL::H, t, 8, NF, x + 8);
    to_tc();
    if (t == 0) gemm(aH, NF * 16, aW1, NF * 16, NF);
    if (!(ok = sync_mma())) break;
    hidden_out(cs.b[0]);
    to_tc();
    if (t == 0) gemm(aH, NH * 16, aW2, NH * 16, NH);
    if (!(ok = sync_mma())) break;
    hidden_out(cs.b[1]);
    to_tc();
    if (t == 0) gemm(aH, NH * 16, aW3, NH * 16, NH);
    if (!(ok = sync_mma())) break;
    // output layer: (y0, y1) += (W4[0][i], W4[1][i]) h_i in order of i
    uint64_t y = f2(cs.b4[0], cs.b4[1]);
#pragma unroll
    for (int c = 0; c < NH; c += 32) {
      float z0[16], z1[16];
      tmem_ld16(trow + c, z0);
      tmem_ld16(trow + c + 16, z1);
      tmem_wait_ld();
      float h[16];
      gelu16(z0, cs.b[2] + c, h);
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const float4 w = *reinterpret_cast<const float4*>(&cs.w4[c + i]);
        y = fma2(f2(w.x, w.y), f2(h[i], h[i]), y);
        y = fma2(f2(w.z, w.w), f2(h[i + 1], h[i + 1]), y);
      }
      gelu16(z1, cs.b[2] + c + 16, h);
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const float4 w = *reinterpret_cast<const float4*>(&cs.w4[c + 16 + i]);
        y = fma2(f2(w.x, w.y), f2(h[i], h[i]), y);
        y = fma2(f2(w.z, w.w), f2(h[i + 1], h[i + 1]), y);
      }
    }
    float y0, y1;
    f2split(y, y0, y1);
    if (live) {
      a.out[(long long)p * 2] = softplus(y0) * osc0;
      a.out[(long long)p * 2 + 1] = softplus(y1) * osc1;
    }
  }
  if (!ok && t == 0) {
    atomicExch(a.err, 1);
    // the layer still in flight (bounded) before freeing; should this wait
    // give up too, the tensor memory is freed all the same: a CTA that kept
    // it would leave later CTAs on its SM waiting in tcgen05.alloc, and the
    // flag already marks this launch's outputs invalid
    if (pend) mbar_wait(mbar, phase, WAIT_ITERS);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tbase, PL::TMEM_COLS);
}

// INF_CTAS_PER_SM resident CTAs per SM: shared memory (the static
// parameter block, InfConst, padded to the dynamic block's 1 KB alignment, the dynamic
// block, and the 1 KB the SM reserves per CTA) within the SM's 228 KB;
// registers by the launch bounds
static_assert(sizeof(InfConst) <= 2048, "parameter block");
static_assert(INF_CTAS_PER_SM * (2048 + PlanInf::BYTES + 1024) <= 228 * 1024, "inference CTAs per SM");

// one wave of resident CTAs, each looping over the tiles
template <int SRC>
static cudaError_t go_infer(const MlpArgs& a, cudaStream_t st) {
  const int ntiles = (a.n + TILE - 1) / TILE;
  if (ntiles == 0) return cudaSuccess;
  cudaFuncSetAttribute(k_mlp_infer<SRC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PlanInf::BYTES);
  const int cap = INF_CTAS_PER_SM * sm_count();
  k_mlp_infer<SRC><<<ntiles < cap ? ntiles : cap, TILE, PlanInf::BYTES, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_les(const MlpArgs& a, bool fp32, cudaStream_t st) {
  return fp32 ? go_infer<1>(a, st) : go_infer<2>(a, st);
}

__global__ void k_adam(float* params, float* grads, float* m1, float* m2, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = grads[i];
  const float m = b1 * m1[i] + (1.0f - b1) * g;
  const float v = b2 * m2[i] + (1.0f - b2) * g * g;
  m1[i] = m;
  m2[i] = v;
  params[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  grads[i] = 0.0f;
}

// single-tile BF16 GEMM D[128][N] = A[128][K] B[N][K]^T through the same
// tensor-core path (a check of the operand layouts and descriptors)
__global__ void __launch_bounds__(128, 1) k_umma_gemm(const uint16_t* A, const uint16_t* B, float* D, int K, int N,
                                                      int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, warp = t >> 5;
  unsigned char* sA = sm;
  unsigned char* sB = sm + 128 * K * 2;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + N * K * 2);
  uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
  for (int i = t; i < 128 * K; i += 128) {
    const int r = i / K, k = i % K;
    *reinterpret_cast<uint16_t*>(sA + kmajor_offset(r, k, K)) = A[i];
  }
  for (int i = t; i < N * K; i += 128) {
    const int r = i / K, k = i % K;
    *reinterpret_cast<uint16_t*>(sB + kmajor_offset(r, k, K)) = B[i];
  }
  if (t == 0) mbar_init(mbar, 1);
  if (warp == 0) {
    tmem_alloc(slot, 256);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *slot;
  if (t == 0) {
    const uint32_t idesc = umma_idesc_bf16(128, N);
    for (int s = 0; s < K / 16; ++s)
      umma_bf16(tbase, umma_desc(smem_u32(sA) + 256 * s, 128, K * 16), umma_desc(smem_u32(sB) + 256 * s, 128, K * 16),
                idesc, s > 0);
    umma_commit(mbar);
  }
  const bool w = mbar_wait(mbar, 0, WAIT_ITERS);
  tc_fence_after();
  const bool ok = __syncthreads_and(w ? 1 : 0) != 0;
  if (ok) {
    for (int c = 0; c < N; c += 16) {
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + c, v);
      tmem_wait_ld();
      for (int i = 0; i < 16; ++i) D[(long long)t * N + c + i] = v[i];
    }
  } else if (t == 0) {
    atomicExch(err, 1);
    // the MMA still in flight (bounded) before freeing; freed even if this
    // wait gives up too (see k_mlp_train)
    if (!w) mbar_wait(mbar, 0, WAIT_ITERS);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tbase, 256);
}

// ---------------------------------------------------------------------------
// launchers
cudaError_t launch_mlp(const MlpArgs& a, bool train, int max_ctas, cudaStream_t st) {
  const int ntiles = (a.n + TILE - 1) / TILE;
  if (ntiles == 0) return cudaSuccess;
  int ctas = ntiles < max_ctas ? ntiles : max_ctas;
  if (train) {
    const size_t smem = PlanTrain::BYTES;
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_mlp_train<<<ctas, TILE, smem, st>>>(a);
    return cudaGetLastError();
  }
  return go_infer<0>(a, st);
}

cudaError_t launch_adam(float* params, float* grads, float* m1, float* m2, int n, float lr, int step,
                        cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<(n + 255) / 256, 256, 0, st>>>(params, grads, m1, m2, n, lr, b1, b2, 1e-8f, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_umma_gemm(const uint16_t* A, const uint16_t* B, float* D, int K, int N, int* err,
                             cudaStream_t st) {
  const size_t smem = (size_t)(128 + N) * K * 2 + 16;
  cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_umma_gemm<<<1, 128, smem, st>>>(A, B, D, K, N, err);
  return cudaGetLastError();
}

size_t mlp_smem_bytes(bool train) { return train ? PlanTrain::BYTES : PlanInf::BYTES; }

}  // namespace db
