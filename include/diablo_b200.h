/*
 * diablo_b200.h -- C-ABI of the B200 (sm_100a) channel time step.
 *
 * This is the drop-in boundary for DIABLO 3.0's channel solver
 * (wienkers/diablo3, Fortran 90).  Each entry point replaces one Fortran
 * subroutine; the reference interface it stands in for is cited beside it.
 * A Fortran caller binds these through an ISO_C_BINDING interface block
 * (one bind(C) function per entry, arguments by value or as arrays);
 * Python binds them through ctypes (diablo3_b200/lib.py).
 *
 * Conventions
 *  - Coordinates follow the Fortran code: x streamwise (periodic), y
 *    wall-normal (finite differences on a stretched grid), z spanwise
 *    (periodic).  nx, ny, nz are the code's Nx, NY (= Nyp on one rank), Nz.
 *  - "Reference spectral layout" is the Fortran array
 *    complex(8) cu(0:Nxp, 0:Nz+1, 0:Nyp+1), Nxp = Nx/2, column-major, passed
 *    as double* of 2*(Nxp+1)*(Nz+2)*(Nyp+2) values (re, im interleaved).
 *    "Reference physical layout" is real(8) u(0:Nx+1, 0:Nz+1, 0:Nyp+1);
 *    both views alias the same number of doubles (for/fft.f90:71-96).
 *  - Every entry point returns int: 0 on success, a DB_ERR_* code otherwise.
 *    Nothing aborts the process; db_last_error() gives the message.
 *  - A context is not thread-safe: one host thread per context.  All work
 *    is issued on the stream given to db_init (NULL = a stream the context
 *    creates).  Host buffers stay owned by the caller.
 */
#ifndef DIABLO_B200_H
#define DIABLO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DB_ABI_VERSION 1

enum db_error {
  DB_OK = 0,
  DB_ERR_ARG = 1,          /* bad argument (NULL pointer, bad field id) */
  DB_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  DB_ERR_SIZE = 3,         /* grid size not supported */
  DB_ERR_UNSUPPORTED = 4,  /* option the reference supports but not built */
  DB_ERR_STATE = 5,        /* call out of order (e.g. before db_init) */
  DB_ERR_NUMERIC = 6,      /* NaN/Inf or dt <= 0 detected on the device */
  DB_ERR_TIMEOUT = 7       /* a bounded device wait gave up */
};

/* Status flags reported by db_get_status (bit mask). */
enum db_flag {
  DB_FLAG_NONFINITE = 1,   /* NaN/Inf found in the velocity or buoyancy */
  DB_FLAG_DT_NONPOS = 2,   /* courant found dt <= 0 (reference flow.f90:812) */
  DB_FLAG_DT_CAPPED = 4,   /* courant capped dt at 1000 (flow.f90:817) */
  DB_FLAG_DT_TINY = 8,     /* next dt < 1e-10 (flow.f90:848) */
  DB_FLAG_WAIT_TIMEOUT = 16 /* a bounded device wait gave up (data of that step invalid) */
};

/* Field ids for db_upload_field / db_download_field. */
enum db_field {
  DB_CU1 = 0, DB_CU2 = 1, DB_CU3 = 2, DB_CP = 3, DB_CTH = 4,
  DB_CF1 = 5, DB_CF2 = 6, DB_CF3 = 7, DB_CFTH = 8,
  DB_NU_T = 9, DB_KAPPA_T = 10,   /* physical layout, GY points */
  DB_NFIELDS = 11
};

/*
 * Run parameters: the contents of input.dat / input_chan.dat version 3.4
 * (for/parameters.f90:84-121, 202-250) plus grid_def, as the Fortran reads
 * them (before input_chan's thermal-wind compensation, which db_init applies
 * exactly as for/parameters.f90:255-279 does).
 */
typedef struct db_params {
  /* grid_def: code sizes (for/domain.f90:20-24) */
  int32_t nx, ny, nz, n_th;
  /* input.dat */
  double re, beta, lx, ly, lz, nu_v_scale;
  double delta_t, cfl;
  int32_t variable_dt, update_dt;
  double ri, pr;
  int32_t use_les, create_new_flow;
  /* input_chan.dat */
  int32_t time_ad_meth, les_model_type, ic_type, physical_noise;
  double kick, ro, delta, grav_x, grav_y, grav_z;
  int32_t f_type, flavor_front;   /* flavor_front: 1 when FLAVOUR == 'Front' */
  double ubulk0, px0, omega0, amp_omega0, force_start;
  int32_t u_bc_ymin, v_bc_ymin, w_bc_ymin, th_bc_ymin;
  int32_t u_bc_ymax, v_bc_ymax, w_bc_ymax, th_bc_ymax;
  double u_bc_ymin_c1, v_bc_ymin_c1, w_bc_ymin_c1, th_bc_ymin_c1;
  double u_bc_ymax_c1, v_bc_ymax_c1, w_bc_ymax_c1, th_bc_ymax_c1;
  /* Extension (not in the reference): background buoyancy gradient M^2.
   * NaN keeps the reference tie dTHdX = Ro_inv/delta (infinite front) or
   * 2/Lx*Ro_inv (finite front), for/parameters.f90:264,274. */
  double dthdx_override;
  /* run control used by courant's next-event scheduling (flow.f90:825) */
  double time_limit, save_stats_dt, save_flow_dt;
  /* 0 = FP64 throughout (plain path); 1 = mixed: transforms, nonlinear
   * products and the SGS model in FP32 (physical and x-half fields stored
   * FP32), the spectral state, the CN tridiagonal solves, the Poisson solve /
   * divergence removal and diagnostics in FP64 */
  int32_t precision;
  int32_t reserved_i[7];
} db_params;

typedef struct db_status {
  int32_t flags;          /* DB_FLAG_* bits accumulated since last clear */
  int32_t time_step;      /* driver counter (for/diablo.f90:59) */
  double time;            /* simulation time */
  double delta_t;         /* current dt (updated by courant) */
  double max_div;         /* max |div u| over modes, from db_divergence */
} db_status;

typedef struct db_ctx db_ctx;

/* ABI version of the loaded library (DB_ABI_VERSION). */
int db_abi_version(void);

/* Message for the last error on this context (or the last db_init error when
 * ctx is NULL).  Never NULL. */
const char* db_last_error(const db_ctx* ctx);

/*
 * Create a context: allocates the whole state on the current CUDA device,
 * builds grid metrics and wavenumbers.  gy holds the ny+1 values of
 * grid.h5:/grids/y, i.e. GY(1:Nyp+1).
 * Replaces init_parameters' grid/coefficient part + init_fft + allocate_all
 * (for/parameters.f90:75-188, for/domain.f90:246-374, for/fft.f90:128-236,
 * for/flow.f90:176-196).
 */
int db_init(const db_params* p, const double* gy, void* cuda_stream, db_ctx** out);

/* Release all device memory of the context. */
int db_finalize(db_ctx* ctx);

/* Copy spectral state from / to host arrays in the reference spectral layout.
 * Any pointer may be NULL (upload: field set to zero; download: skipped).
 * Replaces the module-global state of for/flow.f90:12-18. */
int db_upload_state(db_ctx* ctx, const double* cu1, const double* cu2,
                    const double* cu3, const double* cp, const double* cth,
                    const double* cf1, const double* cf2, const double* cf3,
                    const double* cfth);
int db_download_state(db_ctx* ctx, double* cu1, double* cu2, double* cu3,
                      double* cp, double* cth, double* cf1, double* cf2,
                      double* cf3, double* cfth);

/* One field (enum db_field): spectral fields in the reference spectral
 * layout, DB_NU_T / DB_KAPPA_T in the reference physical layout. */
int db_upload_field(db_ctx* ctx, int field, const double* host);
int db_download_field(db_ctx* ctx, int field, double* host);

/* Driver clock: time, time_step and the next output times used by courant
 * (for/diablo.f90:59-68, for/flow.f90:825-828). */
int db_set_clock(db_ctx* ctx, double time, int32_t time_step,
                 double save_stats_time, double save_flow_time);
int db_get_status(db_ctx* ctx, db_status* out);
int db_clear_status(db_ctx* ctx);

/* In-place 2-D transforms of one host array in the reference layout.
 * fft_xz_to_fourier: physical -> packed, dealiased spectral, forward scaled
 * by 1/(Nx Nz).  fft_xz_to_physical: inverse, unnormalised.
 * Replace for/fft.f90:242-307 and 311-374. */
int db_fft_xz_to_fourier(db_ctx* ctx, double* inout);
int db_fft_xz_to_physical(db_ctx* ctx, double* inout);

/* The same two transforms on a DEVICE array in the reference layout (for
 * callers whose fields already live in device memory), in place, with every
 * layout change on the device.  Stream-ordered on the context's stream: the
 * call returns once the work is enqueued.  The physical layout's padding
 * (x >= Nx, z >= Nz) is neither read nor written, as in the host forms. */
int db_fft_xz_to_fourier_dev(db_ctx* ctx, double* d_inout);
int db_fft_xz_to_physical_dev(db_ctx* ctx, double* d_inout);

/* RKW3 + Crank-Nicolson substep rk_step in {1,2,3} on the device state.
 * Replaces rk_chan_1 (for/solver.f90:366-1273). */
int db_rk_substep(db_ctx* ctx, int rk_step);

/* nsteps full time steps (3 substeps each, then time += delta_t), replayed
 * from a CUDA graph captured on first use.  Replaces the loop body of
 * for/diablo.f90:58-69 (without I/O). */
int db_rk_steps(db_ctx* ctx, int nsteps);

/* Divergence removal on the spectral velocity (projection, phi kept in the
 * context).  Replaces rem_div_chan (for/solver.f90:1302-1379). */
int db_rem_div(db_ctx* ctx);

/* Ghost/boundary rows of the spectral velocity after an initial condition.
 * Replaces apply_BC_vel_mpi_post (for/flow.f90:1161-1360, 1698-1713). */
int db_apply_bc_vel_post(db_ctx* ctx);

/* CFL time step from the current state (velocity transformed internally),
 * with courant's limits and next-event scheduling; sets delta_t and the RK
 * coefficients.  Replaces courant (for/flow.f90:746-857). */
int db_courant(db_ctx* ctx, double* delta_t_out);

/* Pressure cp from the velocity and the buoyancy (planes 1..Nyp), for a
 * restart whose file holds no pressure.  Replaces poisson_p_chan
 * (for/solver.f90:1382-1590).  FP64 on both precision paths; the first call
 * allocates the diagnostics scratch (see db_budget). */
int db_poisson_p(db_ctx* ctx);

/* max over (kx,kz,j) of |ikx u1 + d(u2)/dy + ikz u3| in spectral space at
 * GYF points j = 2..Nyp-1, the quantity rem_div_chan drives to zero. */
int db_divergence(db_ctx* ctx, double* max_div_out);

/* Mean and energy-budget profiles of save_stats_chan (for/diagnostics.f90:
 * 3-480; compute_TKE 1270-1330, compute_TKE_diss 804-1020, production
 * terms 1385-1425) from the current state, in FP64 on both precision
 * paths (from the FP64 spectral state by Parseval).  out[DB_NSTAT][Nyp+2],
 * row r, plane j; rows that do not exist at a plane (GY rows j < 2) are 0.
 * Averages are over x and z, or over z only for the fronts (IC_Type 5..8),
 * as the reference's homogeneousX.  Rows:
 *   ume, vme, wme, thme   horizontal means (vme at GY points)
 *   urms, vrms, wrms, thrms   rms of the fluctuations (vrms at GY)
 *   uv, wv                <u1'u2'>, <u3'u2'> at GY (u interpolated)
 *   uw                    <u1'u3'>
 *   thv                   <th' (u2'(j) + u2'(j+1))/2>, buoyancy flux
 *   epsilon               nu x the 9 squared fluctuation gradients at GY
 *   chi                   |grad th|^2 with the background gradient */
enum {
  DB_ST_UME, DB_ST_VME, DB_ST_WME, DB_ST_THME, DB_ST_URMS, DB_ST_VRMS, DB_ST_WRMS, DB_ST_THRMS,
  DB_ST_UV, DB_ST_WV, DB_ST_UW, DB_ST_THV, DB_ST_EPSILON, DB_ST_CHI, DB_NSTAT
};
int db_stats(db_ctx* ctx, double* out);

/* The energy-budget terms that need the mean flow as a function of x
 * (for/diagnostics.f90: compute_TKE 1254-1360, compute_TKE_Production
 * 1366-1520, compute_MKE_diss 1097-1250, compute_Vorticity 1525-1730), in
 * FP64 on both precision paths.  The means are those of compute_averages
 * (676-800): x-z means with homogeneousX, z-means per x for the fronts
 * (IC_Type 5..8).  out[DB_NBUD][Nyp+2], row r, plane j; zero where a row
 * does not exist.  Rows:
 *   tke                  0.5 (u'u' + v'v' + w'w') about the means (GYF rows, v at GY)
 *   uu_dudx, wu_dwdx     <u'u'>_z dU/dx, <u'w'>_z dW/dx, x-averaged (GYF)
 *   vu_dvdx, vv_dvdy, uv_dudy, wv_dwdy   the GY-row production terms, with
 *                        the thermal-wind shear in dW/dy
 *   epsilon_m            nu <|grad U_mean|^2> (0 with homogeneousX, where
 *                        the reference skips compute_MKE_diss)
 *   omega_x, omega_y, omega_z   rms vorticity (omega_x about minus the
 *                        thermal-wind shear)
 * The first call allocates FP64 scratch: four physical fields and one
 * x-half field. */
enum {
  DB_BU_TKE, DB_BU_UU_DUDX, DB_BU_WU_DWDX, DB_BU_VU_DVDX, DB_BU_VV_DVDY, DB_BU_UV_DUDY, DB_BU_WV_DWDY,
  DB_BU_EPSILON_M, DB_BU_OMEGA_X, DB_BU_OMEGA_Y, DB_BU_OMEGA_Z, DB_NBUD
};
int db_budget(db_ctx* ctx, double* out);

/* Background potential energy (compute_BPE, for/diagnostics.f90:1733-1856,
 * after Tseng & Ferziger 2001) from the FP64 buoyancy plus its background
 * gradient dTHdX (x - Lx/2): the dyf-weighted PDF over nbin bins (the
 * reference uses nbin = Nx; constant bins over +-1.1 dTHdX Lx/2 with
 * homogeneousX, cos-spaced over +-Ro_inv for the fronts), normalised to sum
 * 1, the bin edges th_bin[nbin + 1] and the BPE.  Any output may be NULL. */
int db_bpe(db_ctx* ctx, int nbin, double* pdf, double* th_bin, double* bpe);

/* A physical field binned into z* coordinates (Bin_Ystar_and_Write,
 * for/diagnostics.f90:1859-1950, Winters et al. 1996): the points of planes
 * jstart_th..jend_th go to the buoyancy bins of db_bpe (the buoyancy plus
 * its background gradient), binned[b] = sum(field dyf) / sum(dyf) over bin
 * b (0/0 for an empty bin, as the reference divides), weight[b] (may be
 * NULL) = sum(dyf).  kind DB_ZS_FIELD: field is a host array in the
 * reference physical layout real(0:Nx+1, 0:Nz+1, 0:Nyp+1) (e.g. the
 * reference's shear2, thw, chi, epsilon or TKE integrands); DB_ZS_KE: the
 * kinetic energy 0.5 (u1^2 + u2^2 + u3^2) of the current state (KE_zstar),
 * field unused.  nbin <= 8192 (the reference uses Nx).  FP64 on both
 * precision paths. */
enum { DB_ZS_FIELD = 0, DB_ZS_KE = 1 };
int db_bin_ystar(db_ctx* ctx, int kind, const double* field, int nbin, double* binned, double* weight);

/* The LES statistics of an LES context, FP64, out[DB_NLES][Nyp+2] (row r,
 * plane j): DB_LS_NU and DB_LS_KAPPA the plane means of the stored nu_t and
 * kappa_t (nu_sgs, kappa_sgs: les_chan for/les.f90:909-935, les_chan_th
 * :1404-1430), DB_LS_EPS2 compute_TKE_diss_les's eps_sgs2
 * (for/diagnostics.f90:2057-2118) at GY rows 2..Nyp from the current state
 * and the stored nu_t (zero on the other planes).  nu_t and kappa_t are
 * those of the closure's last evaluation (the last LES substep, or
 * db_les_eval on the current state, as save_stats_LES_OOL runs les_chan
 * before writing).  DB_ERR_ARG without use_les. */
enum { DB_LS_NU = 0, DB_LS_KAPPA, DB_LS_EPS2, DB_NLES };
int db_les_stats(db_ctx* ctx, double* out);

/*
 * Divergence removal that allocates nothing.  No counterpart in the
 * reference (it follows rem_div_chan's arithmetic, for/solver.f90:1302-1379,
 * but needs no context).  For callers that cannot allocate device memory:
 * their device arrays belong to another memory manager (CUDA Fortran or
 * OpenACC pools), or they must not allocate once their time loop runs.
 * cu1, cu2, cu3 are DEVICE arrays in the reference spectral layout
 * (0:Nxp, 0:Nz+1, 0:Nyp+1) complex(8), projected in place; gy is the HOST
 * grid GY(1:Nyp+1).  Only p->nx, ny, nz, lx, lz are read.  Work is queued on
 * `stream` and is complete when the stream is.  Working memory is an 8 MiB
 * static device array held by every GPU that loads the library; it limits
 * ny to 10697 (DB_ERR_SIZE above that).  The first call on each device looks
 * up that array's address and should come before any stream capture.  The
 * grid is kept in the array: a call copies gy to the device (a host-to-device
 * copy from the caller's array, queued on `stream`) only when ny or the
 * values differ from those of the previous call on that device.  All calls
 * share the array: calls overlapping on the GPU race, so serialise them.
 * Returns DB_ERR_ARG / DB_ERR_SIZE / DB_ERR_CUDA on failure.
 */
int db_rem_div_static(const db_params* p, const double* gy, double* cu1,
                      double* cu2, double* cu3, void* cuda_stream);

/* ---- learned SGS closure (no counterpart in the reference, whose les.f90
 * offers Smagorinsky, dynamic and AMD closures).  A 16 -> 64 -> 64 -> 64 -> 2
 * MLP (GELU in its tanh form, softplus outputs) maps point features to nu_t and kappa_t; its
 * hidden layers run on the tensor cores in BF16 with FP32 accumulation,
 * forward and backward.  Features of a point, in this order: the nine
 * velocity gradients du_i/dx_j (i-major: du1/dx, du1/dy, du1/dz, du2/dx,
 * ...), dth/dx, dth/dy, dth/dz, the filter widths 3 dx, 2 dy(j), 3 dz, and
 * the local N^2 = dth/dy (for/les.f90:1213-1222, 1661-1746). ---- */
#define DB_SGS_NFEAT 16
#define DB_SGS_NPARAMS 9538   /* W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[2][64] b4[2] */

typedef struct db_sgs_net db_sgs_net;

/* Create / destroy a network (device parameters, Adam moments, gradient
 * buffer) on the current device; work goes to cuda_stream (NULL: default). */
int db_sgs_create(void* cuda_stream, db_sgs_net** out);
int db_sgs_destroy(db_sgs_net* net);

/* Parameters (FP32, DB_SGS_NPARAMS in the order above), the input
 * normalisation (feature f enters as (x_f - mean_f) / std_f) and the output
 * units (nu_t = out_scale[0] softplus(y0), kappa_t = out_scale[1]
 * softplus(y1)).  Setting resets the Adam state. */
int db_sgs_set(db_sgs_net* net, const float* params, const float* feat_mean, const float* feat_std,
               const float* out_scale);
int db_sgs_get(db_sgs_net* net, float* params);

/* Training range of the features (raw units): inside a channel step, a GY
 * point whose features leave [lo, hi] keeps the AMD eddy viscosity and
 * diffusivity (model 5) instead of the network's.  Default: no bounds. */
int db_sgs_set_range(db_sgs_net* net, const float* lo, const float* hi);

/* Inference on device arrays: feat[n][16] -> out[n][2] = (nu_t, kappa_t). */
int db_sgs_forward(db_sgs_net* net, const float* d_feat, float* d_out, long long n);

/* Mean squared error of out against d_target[n][2] and its gradient with
 * respect to the parameters (copied to grads, DB_SGS_NPARAMS floats). */
int db_sgs_gradient(db_sgs_net* net, const float* d_feat, const float* d_target, long long n,
                    float* grads, double* loss);

/* One Adam step (beta 0.9 / 0.999, eps 1e-8) of learning rate lr on the
 * batch; loss is the batch's mean squared error before the step. */
int db_sgs_train_step(db_sgs_net* net, const float* d_feat, const float* d_target, long long n, float lr,
                      double* loss);

/* Check of the tensor-core path: D[128][N] = A[128][K] B[N][K]^T with A, B
 * given as BF16 bit patterns (host arrays), K a multiple of 16 up to 256,
 * N a multiple of 16 up to 256. */
int db_sgs_gemm_check(const uint16_t* A, const uint16_t* B, float* D, int K, int N);

/* Use net for les_model_type 6 on this context (the net must outlive it).
 * With use_les and les_model_type 6 the substep evaluates the network at
 * every GY point in place of AMD's coefficients (AMD where the features
 * leave the training range); stepping without a net is DB_ERR_STATE. */
int db_set_sgs_net(db_ctx* ctx, db_sgs_net* net);

/* The SGS model on the current state without stepping: les_chan's ghost
 * rows, gradients and eddy coefficients (for/les.f90:551-795, 1201-1358)
 * for model 5 (AMD) or 6 (the attached network, AMD outside its range).
 * nu_t, kappa_t (reference physical layout, GY points) and feat (FP32
 * [Nyp+2][Nz][Nx][16], the closure's features at GY rows) may be NULL.  The
 * context's nu_t / kappa_t are overwritten, as a substep with LES would. */
int db_les_eval(db_ctx* ctx, int model, double* nu_t, double* kappa_t, float* feat);

/* Training data of the closure from the context's (resolved) state: a box
 * filter of fx x fy x fz fine cells around every GY point of the coarse
 * grid gy_coarse (its GY(1:NYc+1), NYc = (ny - 1) / fy + 1, the same
 * stretching), the exact subgrid stress and buoyancy flux of that filter,
 * and nu_t, kappa_t fitted to them by least squares
 * (nu_t = max(0, -tau^d:S / 2 S:S), kappa_t = max(0, -q.grad th / |grad th|^2)).
 * Writes DEVICE arrays d_feat[n][16] (closure features of the filtered
 * field) and d_target[n][2] for the n = nx/fx * nz/fz * (NYc - 3) points of
 * coarse rows 3..NYc-1; with d_feat or d_target NULL only n is returned.
 * A context without use_les allocates its 8 gradient fields on first use. */
int db_sgs_targets(db_ctx* ctx, int fx, int fy, int fz, const double* gy_coarse, float* d_feat,
                   float* d_target, long long* npts);

/* ---- ensembles (no counterpart in the reference, which runs one channel
 * per MPI job): independent channels advanced together.  Each member is a
 * context of its own (own stream, own parameters: seeds, Ri, ...); one CUDA
 * graph per time step forks into every member's stream, runs that member's
 * step (time_step += 1, three substeps, time += dt) and joins back, so one
 * graph launch advances the whole ensemble and the members' kernels run
 * concurrently.  Members must share use_les, les_model_type,
 * create_new_flow, precision and time_step; they stay usable on their own
 * (db_download_state etc.) between ensemble steps. ---- */
typedef struct db_ensemble db_ensemble;
int db_ensemble_create(db_ctx** members, int n, void* cuda_stream, db_ensemble** out);
int db_ensemble_steps(db_ensemble* ens, int nsteps);
int db_ensemble_destroy(db_ensemble* ens);
const char* db_ensemble_error(const db_ensemble* ens);
/* Batched form: members of the same grid size, solved planes and
 * precision, without LES and at a fixed dt (variable_dt 0), are advanced by
 * batched kernels: each kernel of the step is launched once for a group of
 * consecutive members (the member index is a grid dimension; each member's
 * pointers and parameters come from a device table), each group a chain
 * of such launches on its own branch of the step's graph; results are
 * bit-identical to stepping each member alone.  It is used whenever the
 * members qualify, in one group.  db_ensemble_set_batched(ens,
 * groups): 0 selects the per-member graph branches, groups >= 1 the batched
 * form in that many groups (at most 8 and n; DB_ERR_ARG if the members do
 * not qualify).  db_ensemble_info: *groups 0 for the per-member branches,
 * else the batched form's group count; *kernels_per_step the kernels one
 * ensemble step launches for all members (0 before the first step).  In
 * the batched form the members' own kernel counters do not grow. */
int db_ensemble_set_batched(db_ensemble* ens, int groups);
int db_ensemble_info(const db_ensemble* ens, int* groups, long long* kernels_per_step);

/* ---- measurement hooks (no counterpart in the reference, which only
 * prints wall seconds per iteration, for/diablo.f90:101-107) ---- */

/* Stages of one substep, in launch order. */
enum db_stage {
  DB_ST_INV_Z = 0,     /* cu -> x-half, 4 fields      (fft.f90:322-337)   */
  DB_ST_INV_X = 1,     /* x-half -> u, 4 fields       (fft.f90:364-372)   */
  DB_ST_PRODUCTS = 2,  /* 11 products + x-FFT         (solver.f90:655-964) */
  DB_ST_ZPASS_RHS = 3, /* z-FFT + spectral RHS + inverse z of cr; without
                          LES the z-FFT of the products only             */
  DB_ST_INV_X_R = 4,   /* cr x-half -> r, 4 fields (with LES)             */
  DB_ST_THOMAS = 5,    /* CN explicit + Thomas, 4 eqs (solver.f90:1012-1233);
                          without LES with the spectral RHS, per mode     */
  DB_ST_COURANT = 6,   /* CFL reduction (rk_step 3)   (flow.f90:746-857)  */
  DB_ST_FWD_X = 7,     /* u -> x-half, 4 fields                           */
  DB_ST_FWD_Z = 8,     /* x-half -> cu, 4 fields                          */
  DB_ST_REM_DIV = 9,   /* projection + cp update      (solver.f90:1257-1267) */
  DB_NSTAGES = 10
};

/* Autotuner (no counterpart in the reference): times candidate launch shapes
 * of the x-pass (row pairs per TMA-staged item, persistent CTAs per SM), the
 * z-pass (kx columns per CTA), the products (CTAs per SM) and, with LES,
 * the per-column Thomas (threads per CTA) and the closure walk (wall-normal
 * chunks) on this context's scratch buffers, keeps the fastest, and writes
 * the timings and choices as text into report (may be NULL).  Call between
 * steps; it overwrites only scratch fields (the next substep recomputes
 * them). */
int db_autotune(db_ctx* ctx, char* report, int report_len);

/* The launch shapes in use, or set ones found earlier (0 = built-in
 * default), as DB_NTUNE ints in this order: x-pass row pairs per TMA item,
 * x-pass CTAs per SM, z-pass kx columns per CTA, products CTAs per SM, LES
 * Thomas threads per CTA, LES closure wall-normal chunks.  Shapes change
 * how work is split, never the arithmetic: results are bit-identical for
 * every setting.  Use values db_get_tuning reported after db_autotune; a
 * shape a kernel cannot launch with makes the next step return an error. */
#define DB_NTUNE 6
int db_get_tuning(db_ctx* ctx, int* shapes, int n);
int db_set_tuning(db_ctx* ctx, const int* shapes, int n);

/* Record CUDA events between the stages of every substep (the step graph is
 * re-captured with event nodes).  Off by default. */
int db_set_timing(db_ctx* ctx, int enable);

/* Device milliseconds per stage of the most recent full step, summed over
 * its three substeps; ms must hold DB_NSTAGES values. */
int db_stage_times(db_ctx* ctx, double* ms, int nstages);

/* Number of this library's kernels issued on the context so far. */
int db_kernel_launches(db_ctx* ctx, long long* count);

/* Failure-handling hook for tests (no counterpart in the reference): the
 * number of non-blocking checks the first wait on each TMA copy in the
 * products and x-pass kernels makes before it gives up (0 restores the
 * built-in bound of about 1.7e7 blocking polls).  With a small value those
 * waits give up before their
 * copies land: the kernel records DB_FLAG_WAIT_TIMEOUT, waits (within the
 * built-in bound) for every copy it issued, and returns, so the context
 * stays usable and the next db_get_status reports the flag; the data of
 * that step are invalid.  Captured step graphs are dropped. */
int db_set_wait_limit(db_ctx* ctx, uint32_t polls);

#ifdef __cplusplus
}
#endif

#endif /* DIABLO_B200_H */
