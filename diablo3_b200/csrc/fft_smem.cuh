// fft_smem.cuh -- batched FP64 Stockham FFTs in shared memory (sm_100a).
//
// A CTA transforms S sequences of length N (power of two, 16..4096) held in
// shared memory; sequence s, element e sits at buf[s * sstride + e].  The
// work is split as N/8 threads per sequence; every pass each thread holds 8
// complex values in registers (one radix-8, two radix-4 or four radix-2
// butterflies), so the whole CTA reads, syncs, computes and writes back in
// place.  Stockham autosort: the result comes out in natural order.
//
// Pass with radix R after Ns = product of the previous radices, butterfly
// b in [0, N/R):  x_r = in[b + r N/R] * w^(r (b mod Ns) N/(Ns R)),
// X = DFT_R(x),  out[(b / Ns) Ns R + (b mod Ns) + r Ns] = X_r,
// with w = exp(sign 2 pi i / N).  Twiddles come from a table of
// exp(-2 pi i k / N), k < N, built on the host in long double.
#pragma once

#include <cuda_runtime.h>

namespace db {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by i*s (s = +-1)
__device__ __forceinline__ double2 cmul_i(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// In-register DFTs, X_k = sum_n x_n exp(SIGN 2 pi i n k / R).
template <int SIGN>
__device__ __forceinline__ void dft2(double2& a, double2& b) {
  double2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int SIGN>
__device__ __forceinline__ void dft4(double2& x0, double2& x1, double2& x2, double2& x3) {
  double2 a = cadd(x0, x2), b = csub(x0, x2);
  double2 c = cadd(x1, x3), d = cmul_i(csub(x1, x3), (double)SIGN);
  x0 = cadd(a, c);
  x2 = csub(a, c);
  x1 = cadd(b, d);
  x3 = csub(b, d);
}

template <int SIGN>
__device__ __forceinline__ void dft8(double2* x) {
  constexpr double R2 = 0.70710678118654752440084436210484904;  // 1/sqrt(2)
  double2 e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
  double2 o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
  dft4<SIGN>(e0, e1, e2, e3);
  dft4<SIGN>(o0, o1, o2, o3);
  // W8^k o_k, W8 = exp(SIGN 2 pi i / 8) = (1 + SIGN i)/sqrt2
  double2 t1 = make_double2(R2 * (o1.x - SIGN * o1.y), R2 * (o1.y + SIGN * o1.x));
  double2 t2 = cmul_i(o2, (double)SIGN);
  double2 t3 = make_double2(R2 * (-o3.x - SIGN * o3.y), R2 * (-o3.y + SIGN * o3.x));
  x[0] = cadd(e0, o0);
  x[4] = csub(e0, o0);
  x[1] = cadd(e1, t1);
  x[5] = csub(e1, t1);
  x[2] = cadd(e2, t2);
  x[6] = csub(e2, t2);
  x[3] = cadd(e3, t3);
  x[7] = csub(e3, t3);
}

// radix list for each N: first passes radix 8, last pass takes the remainder
template <int N>
struct FftPlan {
  static constexpr int log2n = (N <= 1) ? 0 : 1 + FftPlan<N / 2>::log2n;
  static constexpr int n8 = log2n / 3;                    // radix-8 passes
  static constexpr int rem = log2n - 3 * n8;              // 0, 1 or 2 bits left
  static constexpr int npass = n8 + (rem ? 1 : 0);
};
template <>
struct FftPlan<1> {
  static constexpr int log2n = 0;
};

// One Stockham pass of radix R for sequence base pointer buf (stride 1),
// thread lane in [0, N/8).
template <int N, int R, int SIGN>
__device__ __forceinline__ void stockham_pass_load(const double2* buf, int lane, int Ns,
                                                   const double2* __restrict__ tw, double2* v) {
  constexpr int B = N / R;           // butterflies per sequence
  constexpr int PER = 8 / R;         // butterflies per thread
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    int b = lane + m * (N / 8);
    int kk = b % Ns;
    int tstep = N / (Ns * R);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double2 x = buf[b + r * B];
      if (r > 0 && kk > 0) {
        double2 w = __ldg(&tw[(r * kk * tstep) & (N - 1)]);
        if (SIGN > 0) w.y = -w.y;
        x = cmul(x, w);
      }
      v[m * R + r] = x;
    }
  }
}

template <int N, int R, int SIGN>
__device__ __forceinline__ void stockham_pass_store(double2* buf, int lane, int Ns, double2* v) {
  constexpr int PER = 8 / R;
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    double2* x = v + m * R;
    if (R == 8) dft8<SIGN>(x);
    if (R == 4) dft4<SIGN>(x[0], x[1], x[2], x[3]);
    if (R == 2) dft2<SIGN>(x[0], x[1]);
    int b = lane + m * (N / 8);
    int base = (b / Ns) * Ns * R + (b % Ns);
#pragma unroll
    for (int r = 0; r < R; ++r) buf[base + r * Ns] = x[r];
  }
}

// Full in-place transform of one sequence per thread group; all threads of
// the CTA must call it (it contains __syncthreads).  active = false lets
// surplus threads take part in the barriers only.
template <int N, int SIGN>
__device__ __forceinline__ void fft_inplace(double2* buf, int lane, bool active,
                                            const double2* __restrict__ tw) {
  using P = FftPlan<N>;
  double2 v[8];
  int Ns = 1;
#pragma unroll
  for (int pass = 0; pass < P::npass; ++pass) {
    const bool last_small = (pass == P::npass - 1) && (P::rem != 0);
    if (!last_small) {
      if (active) stockham_pass_load<N, 8, SIGN>(buf, lane, Ns, tw, v);
      __syncthreads();
      if (active) stockham_pass_store<N, 8, SIGN>(buf, lane, Ns, v);
      __syncthreads();
      Ns *= 8;
    } else if (P::rem == 2) {
      if (active) stockham_pass_load<N, 4, SIGN>(buf, lane, Ns, tw, v);
      __syncthreads();
      if (active) stockham_pass_store<N, 4, SIGN>(buf, lane, Ns, v);
      __syncthreads();
      Ns *= 4;
    } else {
      if (active) stockham_pass_load<N, 2, SIGN>(buf, lane, Ns, tw, v);
      __syncthreads();
      if (active) stockham_pass_store<N, 2, SIGN>(buf, lane, Ns, v);
      __syncthreads();
      Ns *= 2;
    }
  }
}

}  // namespace db
