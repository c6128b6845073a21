// fft_reg.cuh -- register-resident Stockham FFT (FP64 double2 or FP32 float2
// complex type C), E elements per thread,
// T = N/E threads per sequence (sm_100a).
//
// Thread `lane` of a group holds v[q] = x[lane + q T], q = 0..E-1.  That set
// is the input of every Stockham pass (a radix-R butterfly b reads
// x[b + r N/R]; the thread owns butterflies b = lane + m T, m < E/R, whose
// inputs are v[m + r E/R]) and, after the last pass, the set of
// natural-order outputs the same thread produces.  Global memory is read
// straight into registers and written straight out of them; only the
// npass - 1 exchanges between passes go through shared memory.
//
// Pass with radix R after Ns = product of earlier radices:
//   x_r = in[b + r N/R] * w^(r (b mod Ns) N/(Ns R)),  X = DFT_R(x),
//   out[(b / Ns) Ns R + (b mod Ns) + r Ns] = X_r,     w = exp(SIGN 2 pi i / N).
// The twiddle base w^((b mod Ns) N/(Ns R)) of each butterfly and pass comes
// from a long-double table (fetched once before the first pass by fft_reg,
// or at the start of each pass by fft_reg_lazy); its powers r = 2..R-1 are
// formed by complex multiplication.  The threads of one sequence
// synchronise among themselves only (__syncwarp, or a named barrier when a
// sequence spans several warps).  Shared memory: one padded buffer per
// sequence (one pad slot every 8 elements keeps the radix-8 scatter free of
// bank conflicts), optionally a second one to alternate exchanges.
#pragma once

#include "cplx_dft.cuh"

// barrier over the threads of the calling sequence (see fft_sync_t)
#define SEQ_SYNC(N) ::db::fft_sync_t<::db::FftShape<N>::warp>(::db::FftShape<N>::T)

namespace db {

__host__ __device__ constexpr int padded(int n) { return n + (n >> 3); }
__device__ __forceinline__ int pidx(int i) { return i + (i >> 3); }

// radix of pass p for length N: radix-8 passes, then one pass of 4 or 2
template <int N>
struct RPlan {
  static constexpr int log2n = FftPlan<N>::log2n;
  static constexpr int n8 = log2n / 3;
  static constexpr int rem = log2n - 3 * n8;
  static constexpr int npass = n8 + (rem ? 1 : 0);
  static constexpr int radix(int p) { return (p < n8) ? 8 : (rem == 2 ? 4 : 2); }
  static constexpr int ns(int p) { return p == 0 ? 1 : ns(p - 1) * radix(p - 1); }
};

// 8 elements per thread (FP64 complex: more spills registers)
template <int N>
struct FftShape {
  static constexpr int E = 8;
  static constexpr int T = N / E;
  static constexpr bool warp = (T <= 32);
};

// Synchronise the T threads of one sequence: __syncwarp when they share a
// warp, else named barrier 1 + (sequence index in the CTA) over T threads,
// so the sequences of a CTA never wait for each other.
template <bool WARP>
__device__ __forceinline__ void fft_sync_t(int T) {
  if (WARP) {
    __syncwarp();
  } else {
    const int id = 1 + (int)(threadIdx.x / T);
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(T) : "memory");
  }
}

// twiddle bases of one thread for every pass p >= 1 and butterfly m
template <int N, int E, typename C = double2>
struct Twiddles {
  static constexpr int MAXB = 8;  // E / R <= 8
  C w[RPlan<N>::npass > 1 ? RPlan<N>::npass - 1 : 1][MAXB];
};

template <int N, int E, typename C>
__device__ __forceinline__ void load_twiddles(Twiddles<N, E, C>& tw, int lane, const C* __restrict__ tab) {
  using P = RPlan<N>;
  constexpr int T = N / E;
#pragma unroll
  for (int p = 1; p < P::npass; ++p) {
    constexpr int dummy = 0;
    (void)dummy;
    const int R = P::radix(p), Ns = P::ns(p);
    const int PER = E / R;
#pragma unroll
    for (int m = 0; m < Twiddles<N, E>::MAXB; ++m)
      if (m < PER) tw.w[p - 1][m] = __ldg(&tab[((lane + m * T) % Ns) * (N / (Ns * R))]);
  }
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void twiddle_apply(C* x, C w) {
  if (SIGN > 0) w.y = -w.y;
  if (R == 8) {   // the powers as a depth-3 tree instead of a chain of 6
    const C w2 = cmul(w, w);
    const C w3 = cmul(w2, w), w4 = cmul(w2, w2);
    const C w5 = cmul(w4, w), w6 = cmul(w3, w3), w7 = cmul(w4, w3);
    x[1] = cmul(x[1], w); x[2] = cmul(x[2], w2); x[3] = cmul(x[3], w3); x[4] = cmul(x[4], w4);
    x[5] = cmul(x[5], w5); x[6] = cmul(x[6], w6); x[7] = cmul(x[7], w7);
    return;
  }
  C wr = w;
#pragma unroll
  for (int r = 1; r < R; ++r) {
    x[r] = cmul(x[r], wr);
    if (r + 1 < R) wr = cmul(wr, w);
  }
}

template <int N, int E, int R, int SIGN, typename C>
__device__ __forceinline__ void reg_pass(C (&v)[E], const C* wb) {
  constexpr int PER = E / R;
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = v[m + r * PER];
    if (wb) twiddle_apply<R, SIGN>(x, wb[m]);
    if (R == 8) dft8<SIGN>(x);
    if (R == 4) dft4<SIGN>(x[0], x[1], x[2], x[3]);
    if (R == 2) dft2<SIGN>(x[0], x[1]);
#pragma unroll
    for (int r = 0; r < R; ++r) v[m + r * PER] = x[r];
  }
}

template <int N, int E, int R, typename C>
__device__ __forceinline__ void reg_scatter(const C (&v)[E], int lane, int Ns, C* s) {
  constexpr int T = N / E;
  constexpr int PER = E / R;
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int b = lane + m * T;
    const int base = (b / Ns) * Ns * R + (b % Ns);
#pragma unroll
    for (int r = 0; r < R; ++r) s[pidx(base + r * Ns)] = v[m + r * PER];
  }
}

template <int N, int E, typename C>
__device__ __forceinline__ void reg_gather(C (&v)[E], int lane, const C* s) {
  constexpr int T = N / E;
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = s[pidx(lane + q * T)];
}

// In-register transform of the E values of this thread (single shared
// buffer s of padded(N) double2 per sequence).  Only the T threads of the
// sequence synchronise (active = false joins the barriers only; at most 15
// sequences per CTA).  On return the exchange buffer may still be read by
// other threads of the sequence: SEQ_SYNC before reusing it.
// CTA = true: the sequence's threads are spread over the CTA (strided lane
// mapping) and every exchange uses __syncthreads.
// s1 (optional): a second buffer; exchanges then alternate between s and s1
// and skip the barrier that protects a single buffer from the next scatter.
template <int N, int SIGN, bool CTA = false, typename C>
__device__ __forceinline__ void fft_reg(C (&v)[FftShape<N>::E], int lane, bool active, C* s,
                                        const Twiddles<N, FftShape<N>::E, C>& tw, C* s1 = nullptr) {
  using P = RPlan<N>;
  constexpr int E = FftShape<N>::E;
  constexpr bool W = FftShape<N>::warp;
#pragma unroll
  for (int p = 0; p < P::npass; ++p) {
    constexpr int dummy = 0;
    (void)dummy;
    const int R = P::radix(p), Ns = P::ns(p);
    const C* wb = (p == 0) ? nullptr : tw.w[p > 0 ? p - 1 : 0];
    if (R == 8) {
      if (active) reg_pass<N, E, 8, SIGN>(v, wb);
      if (p + 1 < P::npass) {
        C* sb = (s1 != nullptr && (p & 1)) ? s1 : s;
        if (p > 0 && s1 == nullptr) {
          if (CTA) __syncthreads(); else fft_sync_t<W>(N / E);
        }
        if (active) reg_scatter<N, E, 8>(v, lane, Ns, sb);
        if (CTA) __syncthreads(); else fft_sync_t<W>(N / E);
        if (active) reg_gather<N, E>(v, lane, sb);
      }
    } else if (R == 4) {
      if (active) reg_pass<N, E, 4, SIGN>(v, wb);
    } else {
      if (active) reg_pass<N, E, 2, SIGN>(v, wb);
    }
  }
}

// Same transform with the twiddle base of each pass fetched inside the pass
// (no twiddle registers held across passes; for register-heavy callers).
template <int N, int SIGN, bool CTA = false, typename C>
__device__ __forceinline__ void fft_reg_lazy(C (&v)[FftShape<N>::E], int lane, bool active, C* s,
                                             const C* __restrict__ tab, C* s1 = nullptr) {
  using P = RPlan<N>;
  constexpr int E = FftShape<N>::E;
  constexpr int T = N / E;
  constexpr bool W = FftShape<N>::warp;
#pragma unroll
  for (int p = 0; p < P::npass; ++p) {
    constexpr int dummy = 0;
    (void)dummy;
    const int R = P::radix(p), Ns = P::ns(p);
    C wb[8];
    if (p > 0) {
      const int PER = E / R;
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < PER) wb[m] = __ldg(&tab[((lane + m * T) % Ns) * (N / (Ns * R))]);
    }
    const C* wbp = (p == 0) ? nullptr : wb;
    if (R == 8) {
      if (active) reg_pass<N, E, 8, SIGN>(v, wbp);
      if (p + 1 < P::npass) {
        C* sb = (s1 != nullptr && (p & 1)) ? s1 : s;
        if (p > 0 && s1 == nullptr) {
          if (CTA) __syncthreads(); else fft_sync_t<W>(T);
        }
        if (active) reg_scatter<N, E, 8>(v, lane, Ns, sb);
        if (CTA) __syncthreads(); else fft_sync_t<W>(T);
        if (active) reg_gather<N, E>(v, lane, sb);
      }
    } else if (R == 4) {
      if (active) reg_pass<N, E, 4, SIGN>(v, wbp);
    } else {
      if (active) reg_pass<N, E, 2, SIGN>(v, wbp);
    }
  }
}

}  // namespace db
