// db_common.cuh -- device-side layout, geometry and run scalars.
//
// HBM layout (FP64; with prec = 1 the physical and x-half fields are FP32):
//   spectral field  double2 s[j][kzp][kx]   j in [0, Nyp+2), kzp in [0, 2Nkz],
//                   kx in [0, kxs) with only kx <= Nkx significant (the rest 0).
//                   kzp uses the reference's packing: 0..Nkz, then -Nkz..-1
//                   (for/fft.f90:299-304).
//   x-half field    double2 h[j][z][kx]    z in [0, Nz): x-transformed, not yet
//                   z-transformed ("Xh").
//   physical field  double  u[j][z][x]     x fastest, no padding.
// j runs over all Nyp+2 planes including both ghost planes, as in the
// reference arrays (0:Nyp+1).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace db {

struct Geom {
  int nx, ny, nz;          // Nx, Nyp, Nz
  int np;                  // Nyp + 2 planes
  int nkx, nkz, nkzp;      // Nkx, Nkz, 2 Nkz + 1
  int kxs;                 // kx stride of spectral / Xh rows
  long long sp;            // spectral plane (double2)  = nkzp * kxs
  long long hp;            // Xh plane (double2)        = nz * kxs
  long long pp;            // physical plane (double)   = nz * nx
  int jstart, jend, jstart_th, jend_th;
  // device tables (length np unless noted)
  const double* gy;
  const double* gyf;
  const double* dy;
  const double* dyf;
  const double* kx;        // kxs entries (0 beyond Nkx)
  const double* kz;        // nkzp entries, packed order
  const double2* twx;      // FFT twiddles, Nx entries
  const double2* twz;      // Nz entries
  const float2* twxf;      // the same rounded to FP32 (mixed path)
  const float2* twzf;
  int prec;                // 0: FP64 throughout; 1: mixed (FP32 physical / x-half)
  int* flags;              // DevScalars::flags, for bounded waits that gave up
  // launch shapes picked by db_autotune (0 = built-in default)
  int tune_xcps;           // x-pass: sequences (row pairs) per staged item
  int tune_xgrid;          // x-pass: persistent CTAs per SM
  int tune_zns;            // z-pass: sequences (kx columns) per CTA
  int tune_les_tb;         // LES Thomas: threads per CTA
  int tune_pgrid;          // products: persistent CTAs per SM
  int tune_amd_ch;         // LES closure walk: wall-normal chunks
  // non-blocking checks the first wait on a TMA copy in the products and
  // x-pass kernels makes before it gives up (0 = the built-in bound of
  // blocking polls); draining a copy still in flight before a CTA leaves
  // always uses the built-in bound
  unsigned wait_first;
};

// Physics constants of the substep (host-computed once at init).
struct Phys {
  double nu, beta, nu_v_scale, pr;
  double ro_inv, delta, grav_x, grav_y, grav_z;
  double dthdx, dthdz, ly, lx;
  int front;               // FLAVOUR == 'Front' (for/flow.f90:781)
  int front_tw;            // flavor 'Front' and Ro_inv != 0 (for/solver.f90:48)
  int f_type;
  double px0, omega0, amp_omega0, force_start;
  int ic_type;
  // boundary types / values in the order u_min, v_min, w_min, th_min,
  // u_max, v_max, w_max, th_max; w values carry input_chan's thermal-wind
  // compensation (for/parameters.f90:257-276)
  int bc_type[8];
  double bc_c1[8];
  double dx, dz;           // Lx/Nx, Lz/Nz
  double pi_ref;           // (double)(float)pi, for/fft.f90:147
};

enum { BC_U_MIN = 0, BC_V_MIN, BC_W_MIN, BC_TH_MIN, BC_U_MAX, BC_V_MAX, BC_W_MAX, BC_TH_MAX };

// Run scalars that live in device memory so a captured CUDA graph can replay
// whole steps: courant updates dt and h_bar on the device.
struct DevScalars {
  double delta_t;
  double h_bar[3];
  double time;
  double save_stats_time, save_flow_time;
  double w_bc_ymax_c1_transient;
  unsigned long long dt_min_bits;   // courant reduction (bit pattern of a >= 0 double)
  int time_step;
  int flags;                        // DB_FLAG_* bits
  double max_div;
  double dt_next;                   // courant's new dt, applied after the substep
  int dt_pending;
  int pad_i;
  double pad[2];
};

// RKW3 constants, for/parameters.f90:179-184
__device__ __forceinline__ double beta_bar(int rk) { return rk == 0 ? 1.0 : (rk == 1 ? 25.0 / 8.0 : 9.0 / 4.0); }
__device__ __forceinline__ double zeta_bar(int rk) { return rk == 0 ? 0.0 : (rk == 1 ? -17.0 / 8.0 : -5.0 / 4.0); }

__host__ __device__ __forceinline__ int round_up(int a, int b) { return (a + b - 1) / b * b; }

}  // namespace db
