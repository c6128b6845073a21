/*
 * oracle.h -- TEST INFRASTRUCTURE, not product code.
 *
 * CPU restatement (C, FP64) of the reference's channel substep, used only as
 * the checker by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg.  Arrays use the reference's own aliased layout: real view
 * (0:Nx+1, 0:Nz+1, 0:Nyp+1), complex view (0:Nxp, 0:Nz+1, 0:Nyp+1), one
 * rank (NprocY = NprocZ = 1), N_th = 1.
 *
 * Parity status: UNPINNED against the reference binary.  The reference has
 * no tests or golden vectors and cannot be built here (no Fortran compiler,
 * MPI, FFTW or HDF5).  Its FFT arithmetic lives in FFTW3 (version unpinned,
 * "FFTW v3.3+", README.md:19), restated here from FFTW's published
 * definitions (forward sign -1, unnormalised; r2c keeps modes 0..N/2; c2r
 * assumes Hermitian input and ignores Im of the DC and Nyquist modes).  The
 * transforms are pinned against an O(N^2) long-double DFT and numpy.fft;
 * the solver against analytic known answers (tests/test_oracle.py).
 */
#ifndef DIABLO_ORACLE_H
#define DIABLO_ORACLE_H

#include "../include/diablo_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* Create/destroy.  gy = GY(1:Nyp+1) (ny+1 values). NULL on error. */
orc_ctx* orc_create(const db_params* p, const double* gy);
void orc_destroy(orc_ctx* c);
const char* orc_error(void);

/* Number of doubles in one reference-layout 3-D array. */
long orc_array_len(const orc_ctx* c);

/* Pointers to the reference-layout state arrays (aliased real/complex).
 * id: DB_CU1..DB_CFTH, DB_NU_T, DB_KAPPA_T, or 100+n for the work arrays
 * r1,r2,r3,rth,s1 (100..104). */
double* orc_array(orc_ctx* c, int id);

/* Grid metrics (0:Nyp+1) and wavenumbers. which: 0 gy,1 gyf,2 dy,3 dyf,
 * 4 kx(0:Nxp-1), 5 kz(0:2Nkz). */
const double* orc_metric(const orc_ctx* c, int which);

/* In-place transforms of a reference-layout buffer (for/fft.f90:242-374). */
void orc_fft_xz_to_fourier(orc_ctx* c, double* buf);
void orc_fft_xz_to_physical(orc_ctx* c, double* buf);

/* rk_chan_1 (for/solver.f90:366-1273) for rk_step in {1,2,3}. */
int orc_rk_chan_1(orc_ctx* c, int rk_step);
/* Full time step: time_step += 1, 3 substeps, time += delta_t. */
int orc_step(orc_ctx* c);
/* rem_div_chan (for/solver.f90:1302-1379). */
void orc_rem_div_chan(orc_ctx* c);
/* poisson_p_chan (for/solver.f90:1382-1590): cp from u and th. */
void orc_poisson_p_chan(orc_ctx* c);
/* apply_BC_vel_mpi_post (for/flow.f90:1161-1360). */
void orc_apply_bc_vel_post(orc_ctx* c);
/* courant (for/flow.f90:746-857) on the physical velocity currently held
 * in u1..u3 (caller transforms); returns the new delta_t. */
double orc_courant_physical(orc_ctx* c);

/* Clock access. */
void orc_set_clock(orc_ctx* c, double time, int time_step,
                   double save_stats_time, double save_flow_time);
void orc_get_clock(const orc_ctx* c, double* time, int* time_step,
                   double* delta_t);

/* Complex FFT helpers for pinning: radix-2 FFT used by the oracle and an
 * O(N^2) long-double DFT.  data: n complex (interleaved); sign -1 forward. */
int orc_fft_c2c(double* data, int n, int sign);
void orc_dft_c2c_ld(double* data, int n, int sign);

/* Batched real Thomas exactly as thomas_forward/backward_real_mpi with
 * NprocY = 1 (for/solver.f90:1691-1761, 1816-1852): a,b,c,g are
 * (0:inx-1, 0:ny+1) column-major; solution returned in g. */
void orc_thomas_real(double* a, double* b, double* c, double* g, int ny, int inx);

#ifdef __cplusplus
}
#endif
#endif
