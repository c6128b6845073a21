// cplx_dft.cuh -- complex helpers (FP64 and FP32), the in-register DFTs of
// radix 2, 4 and 8, and the radix plan of a length-N transform (sm_100a).
// The transforms themselves are in fft_reg.cuh: register-resident Stockham
// passes with shared-memory exchanges between them.
//
// Pass with radix R after Ns = product of the previous radices, butterfly
// b in [0, N/R):  x_r = in[b + r N/R] * w^(r (b mod Ns) N/(Ns R)),
// X = DFT_R(x),  out[(b / Ns) Ns R + (b mod Ns) + r Ns] = X_r,
// with w = exp(sign 2 pi i / N).  Twiddles come from a table of
// exp(-2 pi i k / N), k < N, built on the host in long double.
#pragma once

#include <cuda_runtime.h>

namespace db {

// complex type of a real type and back
template <typename R> struct CplxOf;
template <> struct CplxOf<double> { using type = double2; };
template <> struct CplxOf<float> { using type = float2; };
template <typename C> struct RealOf;
template <> struct RealOf<double2> { using type = double; };
template <> struct RealOf<float2> { using type = float; };

template <typename C>
__device__ __forceinline__ C mkc(typename RealOf<C>::type x, typename RealOf<C>::type y) {
  C c;
  c.x = x;
  c.y = y;
  return c;
}
// complex conversions between the FP64 state and an FP32 work type
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2((double)a.x, (double)a.y); }
template <typename C> __device__ __forceinline__ C from_d2(double2 a);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by i*s (s = +-1)
__device__ __forceinline__ double2 cmul_i(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cmul_i(float2 a, float s) { return make_float2(-s * a.y, s * a.x); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// In-register DFTs, X_k = sum_n x_n exp(SIGN 2 pi i n k / R).
template <int SIGN, typename C>
__device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3) {
  using R = typename RealOf<C>::type;
  C a = cadd(x0, x2), b = csub(x0, x2);
  C c = cadd(x1, x3), d = cmul_i(csub(x1, x3), (R)SIGN);
  x0 = cadd(a, c);
  x2 = csub(a, c);
  x1 = cadd(b, d);
  x3 = csub(b, d);
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft8(C* x) {
  using R = typename RealOf<C>::type;
  constexpr R R2 = (R)0.70710678118654752440084436210484904L;  // 1/sqrt(2)
  constexpr R SG = (R)SIGN;
  C e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
  C o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
  dft4<SIGN>(e0, e1, e2, e3);
  dft4<SIGN>(o0, o1, o2, o3);
  // W8^k o_k, W8 = exp(SIGN 2 pi i / 8) = (1 + SIGN i)/sqrt2
  C t1 = mkc<C>(R2 * (o1.x - SG * o1.y), R2 * (o1.y + SG * o1.x));
  C t2 = cmul_i(o2, SG);
  C t3 = mkc<C>(R2 * (-o3.x - SG * o3.y), R2 * (-o3.y + SG * o3.x));
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

}  // namespace db
