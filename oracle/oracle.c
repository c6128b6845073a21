/*
 * oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * Literal CPU restatement of DIABLO 3.0's channel substep (wienkers/diablo3)
 * in FP64, on the reference's own aliased (x, z, y) arrays with ghost cells,
 * for one rank (NprocY = NprocZ = 1) and one scalar (N_th = 1).  Each
 * routine cites the Fortran lines it follows.  It is the checker for the
 * CUDA path and the CPU baseline of bench.py; it is never linked into the
 * product.  Parity against the reference binary is UNPINNED (see oracle.h).
 *
 * Literal details kept on purpose because they change results:
 *  - pi = 4.*atan(1.0) is evaluated in single precision in the reference
 *    (for/fft.f90:147), so wavenumbers use (double)(float)pi.
 *  - 0.1 and (1. - 0.025) in courant are single-precision literals
 *    (for/flow.f90:772, 831).
 *  - The Thomas systems span rows 0..Nyp+1 (real) and 1..Nyp (complex).
 *  - Rows outside each equation's j-range keep the values the reference
 *    leaves there (physical ghost planes are carried through the transforms).
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

static char g_err[256] = "";

struct orc_ctx {
  db_params p;
  int Nx, Nyp, Nz, Nxp, Nzp, Nkx, Nkz, twoNkz;
  long NX2, NZ2, NXP1, plane_r, len;
  double nu, pi, Ro_inv, dTHdX, dTHdZ;
  double w_bc_ymin_c1, w_bc_ymax_c1, w_bc_ymax_c1_transient;
  double *gx, *dx, *gz, *dz;    /* 0..Nx+1 / 0..Nz+1 */
  double *gy, *gyf, *dy, *dyf;  /* 0..Nyp+1 */
  double *kx, *kx2;             /* 0..Nxp */
  double *kz, *kz2;             /* 0..twoNkz */
  cplx *cikx, *cikz;
  double h_bar[3], beta_bar[3], zeta_bar[3];
  double delta_t;
  int jstart, jend, jstart_th, jend_th;
  double time, save_stats_time, save_flow_time;
  int time_step;
  double* arr[16];
  double* les[30];    /* LES work arrays, indexed by the L_* enum */
  cplx *twx, *twz;
  int *revx, *revz;
};

/* ---------------------------------------------------------------------- */
/* indexing into the reference layout                                      */

#define RV(c, a, i, k, j) ((a)[(long)(j) * (c)->plane_r + (long)(k) * (c)->NX2 + (i)])
#define CV(c, a, i, k, j) \
  (((cplx*)(a))[(long)(j) * ((c)->plane_r / 2) + (long)(k) * (c)->NXP1 + (i)])

enum { A_R1 = 11, A_R2 = 12, A_R3 = 13, A_RTH = 14, A_S1 = 15 };

static double* arr_of(orc_ctx* c, int id) {
  if (id >= 0 && id <= DB_KAPPA_T) return c->arr[id];
  if (id >= 100 && id <= 104) return c->arr[A_R1 + (id - 100)];
  return NULL;
}

/* ---------------------------------------------------------------------- */
/* FFT: radix-2 complex transform with long-double twiddles (FFTW-quality   */
/* accuracy), plus an O(N^2) long-double DFT used to pin it.               */

static const long double PI_L = 3.141592653589793238462643383279502884L;

static int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return ((1 << l) == n) ? l : -1;
}

static void make_fft_tables(int n, cplx** tw, int** rev) {
  int lg = ilog2i(n);
  *tw = (cplx*)malloc(sizeof(cplx) * (size_t)n);
  *rev = (int*)malloc(sizeof(int) * (size_t)n);
  for (int k = 0; k < n; ++k) {
    long double a = 2.0L * PI_L * (long double)k / (long double)n;
    (*tw)[k] = (double)cosl(a) - I * (double)sinl(a);
    int r = 0;
    for (int b = 0; b < lg; ++b)
      if (k & (1 << b)) r |= 1 << (lg - 1 - b);
    (*rev)[k] = r;
  }
}

/* in-place; sign -1: forward (exp(-2 pi i nk/N)), +1: backward; unnormalised */
static void fft_r2(cplx* x, int n, const cplx* tw, const int* rev, int sign) {
  for (int i = 0; i < n; ++i) {
    int j = rev[i];
    if (i < j) {
      cplx t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1, step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int k = 0; k < half; ++k) {
        cplx w = tw[k * step];
        if (sign > 0) w = conj(w);
        cplx a = x[i + k], b = x[i + k + half] * w;
        x[i + k] = a + b;
        x[i + k + half] = a - b;
      }
    }
  }
}

int orc_fft_c2c(double* data, int n, int sign) {
  if (ilog2i(n) < 0) return -1;
  cplx* tw;
  int* rev;
  make_fft_tables(n, &tw, &rev);
  fft_r2((cplx*)data, n, tw, rev, sign);
  free(tw);
  free(rev);
  return 0;
}

void orc_dft_c2c_ld(double* data, int n, int sign) {
  long double* out = (long double*)malloc(sizeof(long double) * 2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    long double sr = 0, si = 0;
    for (int m = 0; m < n; ++m) {
      long double a = (long double)sign * 2.0L * PI_L * (long double)((long)m * k % n) / n;
      long double cr = cosl(a), ci = sinl(a);
      long double xr = data[2 * m], xi = data[2 * m + 1];
      sr += xr * cr - xi * ci;
      si += xr * ci + xi * cr;
    }
    out[2 * k] = sr;
    out[2 * k + 1] = si;
  }
  for (int k = 0; k < 2 * n; ++k) data[k] = (double)out[k];
  free(out);
}

/* ---------------------------------------------------------------------- */
/* fft_xz_to_fourier / fft_xz_to_physical (for/fft.f90:242-374)             */

/* x r2c of rows ka, kb of plane j into tmp rows (two real rows per complex
 * FFT); tmp is (0:Nx/2, 0:Nz-1) complex, scaled by 1/Nx, zero for i > Nkx
 * (for/fft.f90:253-263). */
static void x_r2c_pair(orc_ctx* c, const double* buf, int j, int ka, int kb,
                       cplx* z, cplx* tmp) {
  int N = c->Nx, H = c->Nx / 2;
  for (int i = 0; i < N; ++i) z[i] = RV(c, buf, i, ka, j) + I * RV(c, buf, i, kb, j);
  fft_r2(z, N, c->twx, c->revx, -1);
  for (int m = 0; m <= H; ++m) {
    cplx zm = z[m], zn = conj(z[(N - m) % N]);
    cplx xa = 0.5 * (zm + zn);
    cplx xb = -0.5 * I * (zm - zn);
    tmp[(long)ka * (H + 1) + m] = (m <= c->Nkx) ? xa / (double)N : 0.0;
    tmp[(long)kb * (H + 1) + m] = (m <= c->Nkx) ? xb / (double)N : 0.0;
  }
}

/* x c2r of tmp rows ka, kb into rows ka, kb of plane j (FFTW c2r semantics:
 * Im of DC and Nyquist ignored; for/fft.f90:364-372). */
static void x_c2r_pair(orc_ctx* c, double* buf, int j, int ka, int kb,
                       const cplx* tmp, cplx* z) {
  int N = c->Nx, H = c->Nx / 2;
  const cplx* A = tmp + (long)ka * (H + 1);
  const cplx* B = tmp + (long)kb * (H + 1);
  for (int m = 0; m <= H; ++m) {
    cplx a = A[m], b = B[m];
    if (m == 0 || m == H) {
      a = creal(a);
      b = creal(b);
    }
    z[m] = a + I * b;
    if (m > 0 && m < H) z[N - m] = conj(a) + I * conj(b);
  }
  fft_r2(z, N, c->twx, c->revx, +1);
  for (int i = 0; i < N; ++i) {
    RV(c, buf, i, ka, j) = creal(z[i]);
    RV(c, buf, i, kb, j) = cimag(z[i]);
  }
}

void orc_fft_xz_to_fourier(orc_ctx* c, double* buf) {
  int Nz = c->Nz, Nxp = c->Nxp, Nkz = c->Nkz, H = c->Nx / 2;
  int nplanes = c->Nyp + 2;
#pragma omp parallel
  {
    cplx* z = (cplx*)malloc(sizeof(cplx) * (size_t)(c->Nx > Nz ? c->Nx : Nz));
    cplx* tmp = (cplx*)malloc(sizeof(cplx) * (size_t)(H + 1) * (size_t)Nz);
#pragma omp for schedule(static)
    for (int j = 0; j < nplanes; ++j) {
      for (int k = 0; k < Nz; k += 2) x_r2c_pair(c, buf, j, k, k + 1, z, tmp);
      /* transpose (single rank: the alltoall is a copy), for/fft.f90:283 */
      for (int k = 0; k < Nz; ++k)
        for (int i = 0; i < Nxp; ++i) CV(c, buf, i, k, j) = tmp[(long)k * (H + 1) + i];
      /* z c2c forward on columns i < Nxp, for/fft.f90:290 */
      for (int i = 0; i < Nxp; ++i) {
        for (int k = 0; k < Nz; ++k) z[k] = CV(c, buf, i, k, j);
        fft_r2(z, Nz, c->twz, c->revz, -1);
        for (int k = 0; k < Nz; ++k) CV(c, buf, i, k, j) = z[k];
      }
      /* scale and pack, for/fft.f90:293-305 */
      for (int k = 0; k <= Nkz; ++k)
        for (int i = 0; i < Nxp; ++i) CV(c, buf, i, k, j) = CV(c, buf, i, k, j) / (double)Nz;
      for (int k = 1; k <= Nkz; ++k)
        for (int i = 0; i < Nxp; ++i)
          CV(c, buf, i, Nkz + k, j) = CV(c, buf, i, Nz - 1 + k - Nkz, j) / (double)Nz;
    }
    free(z);
    free(tmp);
  }
}

void orc_fft_xz_to_physical(orc_ctx* c, double* buf) {
  int Nz = c->Nz, Nxp = c->Nxp, Nkz = c->Nkz, Nkx = c->Nkx, H = c->Nx / 2;
  int nplanes = c->Nyp + 2;
#pragma omp parallel
  {
    cplx* z = (cplx*)malloc(sizeof(cplx) * (size_t)(c->Nx > Nz ? c->Nx : Nz));
    cplx* tmp = (cplx*)malloc(sizeof(cplx) * (size_t)(H + 1) * (size_t)Nz);
#pragma omp for schedule(static)
    for (int j = 0; j < nplanes; ++j) {
      /* unpack and de-alias in z, for/fft.f90:322-333 */
      for (int k = Nkz; k >= 1; --k)
        for (int i = 0; i < Nxp; ++i) CV(c, buf, i, Nz - 1 + k - Nkz, j) = CV(c, buf, i, Nkz + k, j);
      for (int k = Nkz + 1; k <= Nz - Nkz - 1; ++k)
        for (int i = 0; i < Nxp; ++i) CV(c, buf, i, k, j) = 0.0;
      /* z c2c backward, for/fft.f90:337 */
      for (int i = 0; i < Nxp; ++i) {
        for (int k = 0; k < Nz; ++k) z[k] = CV(c, buf, i, k, j);
        fft_r2(z, Nz, c->twz, c->revz, +1);
        for (int k = 0; k < Nz; ++k) CV(c, buf, i, k, j) = z[k];
      }
      /* transpose back and de-alias in x, for/fft.f90:358-370 */
      for (int k = 0; k < Nz; ++k) {
        for (int i = 0; i < Nxp; ++i) tmp[(long)k * (H + 1) + i] = CV(c, buf, i, k, j);
        for (int i = Nxp; i <= H; ++i) tmp[(long)k * (H + 1) + i] = 0.0;
        for (int i = Nkx + 1; i <= H; ++i) tmp[(long)k * (H + 1) + i] = 0.0;
      }
      for (int k = 0; k < Nz; k += 2) x_c2r_pair(c, buf, j, k, k + 1, tmp, z);
    }
    free(z);
    free(tmp);
  }
}

/* ---------------------------------------------------------------------- */
/* Thomas solvers (for/solver.f90:1691-1896), NprocY = 1                    */

/* real: rows 0..ny+1, a,b,c,g laid out (0:inx-1, 0:ny+1) */
void orc_thomas_real(double* a, double* b, double* cc, double* g, int ny, int inx) {
#define T2(arr, i, j) arr[(long)(j) * inx + (i)]
  for (int j = 1; j <= ny + 1; ++j)
    for (int i = 0; i < inx; ++i) {
      T2(a, i, j) = -T2(a, i, j) / T2(b, i, j - 1);
      T2(b, i, j) = T2(b, i, j) + T2(a, i, j) * T2(cc, i, j - 1);
      T2(g, i, j) = T2(g, i, j) + T2(a, i, j) * T2(g, i, j - 1);
    }
  for (int i = 0; i < inx; ++i) {
    T2(g, i, ny + 1) = T2(g, i, ny + 1) / T2(b, i, ny + 1);
    for (int j = ny; j >= 0; --j)
      T2(g, i, j) = (T2(g, i, j) - T2(cc, i, j) * T2(g, i, j + 1)) / T2(b, i, j);
  }
#undef T2
}

/* complex rhs, real matrix: rows 1..ny (for/solver.f90:1764-1813, 1855-1896)
 * for a single column (arrays indexed 0..ny+1). */
static void thomas_complex_col(double* a, double* b, const double* cc, cplx* g, int ny) {
  for (int j = 2; j <= ny; ++j) {
    a[j] = -a[j] / b[j - 1];
    b[j] = b[j] + a[j] * cc[j - 1];
    g[j] = g[j] + a[j] * g[j - 1];
  }
  g[ny] = g[ny] / b[ny];
  for (int j = ny - 1; j >= 1; --j) g[j] = (g[j] - cc[j] * g[j + 1]) / b[j];
}

/* ---------------------------------------------------------------------- */
/* context                                                                  */

const char* orc_error(void) { return g_err; }

static int check_params(const db_params* p) {
  if (p->nx < 8 || p->nz < 8 || ilog2i(p->nx) < 0 || ilog2i(p->nz) < 0) {
    snprintf(g_err, sizeof g_err, "oracle: nx, nz must be powers of two >= 8");
    return -1;
  }
  if (p->ny < 4) {
    snprintf(g_err, sizeof g_err, "oracle: ny must be >= 4");
    return -1;
  }
  if (p->n_th != 1) {
    snprintf(g_err, sizeof g_err, "oracle: n_th must be 1");
    return -1;
  }
  int bcs[8] = {p->u_bc_ymin, p->v_bc_ymin, p->w_bc_ymin, p->th_bc_ymin,
                p->u_bc_ymax, p->v_bc_ymax, p->w_bc_ymax, p->th_bc_ymax};
  for (int b = 0; b < 8; ++b)
    if (bcs[b] != 0 && bcs[b] != 1) {
      snprintf(g_err, sizeof g_err, "oracle: boundary types must be 0 or 1");
      return -1;
    }
  return 0;
}

orc_ctx* orc_create(const db_params* p, const double* gy_in) {
  if (!p || !gy_in || check_params(p)) return NULL;
  orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
  c->p = *p;
  c->Nx = p->nx;
  c->Nyp = p->ny;
  c->Nz = p->nz;
  c->Nxp = c->Nx / 2;
  c->Nzp = c->Nz;
  c->Nkx = c->Nx / 3;
  c->Nkz = c->Nz / 3;
  c->twoNkz = 2 * c->Nkz;
  c->NX2 = c->Nx + 2;
  c->NZ2 = c->Nz + 2;
  c->NXP1 = c->Nxp + 1;
  c->plane_r = c->NX2 * c->NZ2;
  c->len = c->plane_r * (c->Nyp + 2);
  /* for/fft.f90:147: pi = 4.*atan(1.0) in default (single) precision */
  c->pi = (double)(4.0f * atanf(1.0f));
  c->nu = 1.0 / p->re; /* for/parameters.f90:102 */
  c->Ro_inv = 1.0 / p->ro; /* for/parameters.f90:221 */

  int Nyp = c->Nyp, Nx = c->Nx, Nz = c->Nz;
  c->gx = (double*)calloc(Nx + 2, sizeof(double));
  c->dx = (double*)calloc(Nx + 2, sizeof(double));
  c->gz = (double*)calloc(Nz + 2, sizeof(double));
  c->dz = (double*)calloc(Nz + 2, sizeof(double));
  c->gy = (double*)calloc(Nyp + 2, sizeof(double));
  c->gyf = (double*)calloc(Nyp + 2, sizeof(double));
  c->dy = (double*)calloc(Nyp + 2, sizeof(double));
  c->dyf = (double*)calloc(Nyp + 2, sizeof(double));
  /* create_grid_chan, for/domain.f90:253-300 */
  for (int i = 0; i <= Nx; ++i) {
    c->gx[i] = (i * p->lx) / Nx;
    c->dx[i] = p->lx / Nx;
  }
  for (int k = 0; k <= Nz; ++k) {
    c->gz[k] = (k * p->lz) / Nz;
    c->dz[k] = p->lz / Nz;
  }
  for (int j = 1; j <= Nyp + 1; ++j) c->gy[j] = gy_in[j - 1]; /* domain.f90:517 */
  for (int j = 1; j <= Nyp; ++j) c->gyf[j] = 0.5 * (c->gy[j] + c->gy[j + 1]);
  c->gyf[0] = 2.0 * c->gyf[1] - c->gyf[2];
  c->gyf[Nyp + 1] = 2.0 * c->gyf[Nyp] - c->gyf[Nyp - 1];
  for (int j = 1; j <= Nyp + 1; ++j) c->dy[j] = c->gyf[j] - c->gyf[j - 1];
  for (int j = 1; j <= Nyp; ++j) c->dyf[j] = c->gy[j + 1] - c->gy[j];
  c->dyf[0] = c->dyf[1];
  c->dyf[Nyp + 1] = c->dyf[Nyp];

  /* wavenumbers, for/fft.f90:208-225 */
  c->kx = (double*)calloc(c->Nxp + 1, sizeof(double));
  c->kx2 = (double*)calloc(c->Nxp + 1, sizeof(double));
  c->cikx = (cplx*)calloc(c->Nxp + 1, sizeof(cplx));
  c->kz = (double*)calloc(c->twoNkz + 1, sizeof(double));
  c->kz2 = (double*)calloc(c->twoNkz + 1, sizeof(double));
  c->cikz = (cplx*)calloc(c->twoNkz + 1, sizeof(cplx));
  for (int i = 0; i < c->Nxp; ++i) {
    c->kx[i] = i * (2. * c->pi) / p->lx;
    c->kx2[i] = c->kx[i] * c->kx[i];
    c->cikx[i] = I * c->kx[i];
  }
  for (int k = 0; k <= c->Nkz; ++k) c->kz[k] = k * (2. * c->pi) / p->lz;
  for (int k = 1; k <= c->Nkz; ++k) c->kz[c->twoNkz + 1 - k] = -k * (2. * c->pi) / p->lz;
  for (int k = 0; k <= c->twoNkz; ++k) {
    c->kz2[k] = c->kz[k] * c->kz[k];
    c->cikz[k] = I * c->kz[k];
  }

  /* input_chan thermal-wind compensation, for/parameters.f90:255-279 */
  c->w_bc_ymin_c1 = p->w_bc_ymin_c1;
  c->w_bc_ymax_c1 = p->w_bc_ymax_c1;
  c->dTHdX = 0.0;
  c->dTHdZ = 0.0;
  if (p->ic_type == 4 || p->ic_type == 5) {
    double m2 = isnan(p->dthdx_override) ? c->Ro_inv / p->delta : p->dthdx_override;
    double shear = m2 * p->delta / c->Ro_inv; /* == 1 under the reference tie */
    if (p->w_bc_ymin == 1) c->w_bc_ymin_c1 -= shear;
    if (p->w_bc_ymax == 1) c->w_bc_ymax_c1 -= shear;
    c->dTHdX = m2;
  } else if (p->ic_type == 6 || p->ic_type == 7 || p->ic_type == 8) {
    if (p->w_bc_ymin == 1) c->w_bc_ymin_c1 -= 2.0 * p->delta / p->lx;
    if (p->w_bc_ymax == 1) c->w_bc_ymax_c1 -= 2.0 * p->delta / p->lx;
    c->dTHdX = isnan(p->dthdx_override) ? 2.0 / p->lx * c->Ro_inv : p->dthdx_override;
  }
  c->w_bc_ymax_c1_transient = c->w_bc_ymax_c1;

  /* init_chan_mpi, for/domain.f90:321-340 with one rank in y: rankY == 0
   * takes the first branch of the if / else if chain, so jstart follows the
   * lower BC and jend = jend_th = Nyp whatever the upper BC (the upper
   * branch, 341-361, runs only on the top rank of several). */
  c->jstart = (p->u_bc_ymin == 1) ? 1 : 2;
  c->jend = Nyp;
  c->jstart_th = (p->th_bc_ymin == 1) ? 1 : 2;
  c->jend_th = Nyp;

  /* RKW3, for/parameters.f90:176-184 */
  c->delta_t = p->delta_t;
  c->h_bar[0] = c->delta_t * (8.0 / 15.0);
  c->h_bar[1] = c->delta_t * (2.0 / 15.0);
  c->h_bar[2] = c->delta_t * (5.0 / 15.0);
  c->beta_bar[0] = 1.0;
  c->beta_bar[1] = 25.0 / 8.0;
  c->beta_bar[2] = 9.0 / 4.0;
  c->zeta_bar[0] = 0.0;
  c->zeta_bar[1] = -17.0 / 8.0;
  c->zeta_bar[2] = -5.0 / 4.0;

  for (int a = 0; a < 16; ++a) c->arr[a] = (double*)calloc((size_t)c->len, sizeof(double));
  if (p->use_les)
    for (int a = 0; a < 30; ++a) c->les[a] = (double*)calloc((size_t)c->len, sizeof(double));
  make_fft_tables(Nx, &c->twx, &c->revx);
  make_fft_tables(Nz, &c->twz, &c->revz);
  c->save_stats_time = 1e300;
  c->save_flow_time = 1e300;
  return c;
}

void orc_destroy(orc_ctx* c) {
  if (!c) return;
  for (int a = 0; a < 16; ++a) free(c->arr[a]);
  for (int a = 0; a < 30; ++a) free(c->les[a]);
  free(c->gx); free(c->dx); free(c->gz); free(c->dz);
  free(c->gy); free(c->gyf); free(c->dy); free(c->dyf);
  free(c->kx); free(c->kx2); free(c->cikx);
  free(c->kz); free(c->kz2); free(c->cikz);
  free(c->twx); free(c->twz); free(c->revx); free(c->revz);
  free(c);
}

long orc_array_len(const orc_ctx* c) { return c->len; }
double* orc_array(orc_ctx* c, int id) { return arr_of(c, id); }

const double* orc_metric(const orc_ctx* c, int which) {
  switch (which) {
    case 0: return c->gy;
    case 1: return c->gyf;
    case 2: return c->dy;
    case 3: return c->dyf;
    case 4: return c->kx;
    case 5: return c->kz;
    default: return NULL;
  }
}

void orc_set_clock(orc_ctx* c, double time, int time_step, double sst, double sft) {
  c->time = time;
  c->time_step = time_step;
  c->save_stats_time = sst;
  c->save_flow_time = sft;
}

void orc_get_clock(const orc_ctx* c, double* time, int* time_step, double* dt) {
  if (time) *time = c->time;
  if (time_step) *time_step = c->time_step;
  if (dt) *dt = c->delta_t;
}

/* ---------------------------------------------------------------------- */
/* boundary conditions on the implicit systems (for/solver.f90:1901-2324)   */

typedef struct { double *l, *d, *u, *v; int nx; } tri_t;
#define TL(t, i, j) (t).l[(long)(j) * (t).nx + (i)]
#define TD(t, i, j) (t).d[(long)(j) * (t).nx + (i)]
#define TU(t, i, j) (t).u[(long)(j) * (t).nx + (i)]
#define TVv(t, i, j) (t).v[(long)(j) * (t).nx + (i)]

static void set_row(tri_t t, int j, double l, double d, double u, double v) {
  for (int i = 0; i < t.nx; ++i) {
    TL(t, i, j) = l;
    TD(t, i, j) = d;
    TU(t, i, j) = u;
    TVv(t, i, j) = v;
  }
}

/* apply_BC_1_lower/upper and apply_BC_3_lower/upper share this form */
static void bc_horizontal(orc_ctx* c, tri_t t, int bmin, double c1min, int bmax, double c1max) {
  int Nyp = c->Nyp;
  if (bmin == 0) {
    set_row(t, 0, 0., 1., 0., 0.);
    set_row(t, 1, 0., 1., 0., c1min);
  } else {
    set_row(t, 0, 0., 1., 0., 0.);
    set_row(t, 1, 0., -1., 1., c->dy[2] * c1min);
  }
  if (bmax == 0) {
    set_row(t, Nyp + 1, 0., 1., 0., 0.);
    set_row(t, Nyp, 0., 1., 0., c1max);
  } else {
    set_row(t, Nyp, -1., 1., 0., c->dy[Nyp] * c1max);
    set_row(t, Nyp + 1, 0., 1., 0., 0.);
  }
}

static void bc_u2(orc_ctx* c, tri_t t) { /* apply_BC_2_lower/upper */
  const db_params* p = &c->p;
  int Nyp = c->Nyp;
  if (p->v_bc_ymin == 0) {
    set_row(t, 1, 0., 1., 0., p->v_bc_ymin_c1);
    set_row(t, 2, 0., 1., 0., p->v_bc_ymin_c1);
  } else {
    set_row(t, 1, 0., -1., 1., c->dyf[1] * p->v_bc_ymin_c1);
  }
  set_row(t, 0, 0., 1., 0., 0.);
  if (p->v_bc_ymax == 0) {
    set_row(t, Nyp + 1, 0., 1., 0., p->v_bc_ymax_c1);
    set_row(t, Nyp, 0., 1., 0., p->v_bc_ymax_c1);
  } else {
    set_row(t, Nyp + 1, -1., 1., 0., c->dyf[Nyp] * p->v_bc_ymax_c1);
  }
}

/* ---------------------------------------------------------------------- */
/* user_rhs_chan_fourier: thermal-wind advection (for/solver.f90:35-111)    */

static void user_rhs_chan_fourier(orc_ctx* c) {
  const db_params* p = &c->p;
  if (!(p->flavor_front && c->Ro_inv != 0.0)) return;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  double* cth = c->arr[DB_CTH];
  double* cf1 = c->arr[DB_CF1]; double* cf2 = c->arr[DB_CF2]; double* cf3 = c->arr[DB_CF3];
  double* cfth = c->arr[DB_CFTH];
  double dX = c->dTHdX, dZ = c->dTHdZ, del = p->delta, Ro = c->Ro_inv, Ly = p->ly;
  for (int j = c->jstart; j <= c->jend; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        double y = c->gyf[j] - 0.5 * Ly;
        cplx v2 = 0.5 * (CV(c, cu2, i, k, j) + CV(c, cu2, i, k, j + 1));
        CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j)
            - (dX * y * del / Ro) * c->cikz[k] * CV(c, cu1, i, k, j)
            - (-1.0 * dZ * y * del / Ro) * c->cikx[i] * CV(c, cu1, i, k, j)
            - (-1.0 * dZ * del / Ro) * v2;
        CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j)
            - (dX * y * del / Ro) * c->cikz[k] * CV(c, cu3, i, k, j)
            - (-1.0 * dZ * y * del / Ro) * c->cikx[i] * CV(c, cu3, i, k, j)
            - (dX * del / Ro) * v2;
      }
  for (int j = 2; j <= c->Nyp; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        double y = c->gy[j] - 0.5 * Ly;
        CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j)
            - (dX * y * del / Ro) * c->cikz[k] * CV(c, cu2, i, k, j)
            - (-1.0 * dZ * y * del / Ro) * c->cikx[i] * CV(c, cu2, i, k, j);
      }
  for (int j = c->jstart_th; j <= c->jend_th; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        double y = c->gyf[j] - 0.5 * Ly;
        CV(c, cfth, i, k, j) = CV(c, cfth, i, k, j)
            - (del / Ro) * dX * y * c->cikz[k] * CV(c, cth, i, k, j)
            - (del / Ro) * (-1.0) * dZ * y * c->cikx[i] * CV(c, cth, i, k, j);
      }
}

/* ---------------------------------------------------------------------- */
/* rem_div_chan (for/solver.f90:1302-1379), phi left in cr1 (array r1)      */

void orc_rem_div_chan(orc_ctx* c) {
  int Nyp = c->Nyp;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  double* cr1 = c->arr[A_R1];
#pragma omp parallel
  {
    double* a = (double*)malloc(sizeof(double) * (size_t)(Nyp + 2));
    double* b = (double*)malloc(sizeof(double) * (size_t)(Nyp + 2));
    double* u = (double*)malloc(sizeof(double) * (size_t)(Nyp + 2));
    cplx* g = (cplx*)malloc(sizeof(cplx) * (size_t)(Nyp + 2));
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        for (int j = 0; j <= Nyp + 1; ++j) { a[j] = 0.; b[j] = 1.; u[j] = 0.; g[j] = 0.; }
        for (int j = 1; j <= Nyp; ++j) {
          a[j] = 1. / (c->dy[j] * c->dyf[j]);
          b[j] = -c->kx2[i] - c->kz2[k] - 1. / (c->dy[j + 1] * c->dyf[j]) - 1. / (c->dy[j] * c->dyf[j]);
          u[j] = 1. / (c->dy[j + 1] * c->dyf[j]);
          g[j] = c->cikx[i] * CV(c, cu1, i, k, j)
               + (CV(c, cu2, i, k, j + 1) - CV(c, cu2, i, k, j)) / c->dyf[j]
               + c->cikz[k] * CV(c, cu3, i, k, j);
        }
        /* apply_BC_rem_div_mpi, for/solver.f90:2341-2368 */
        if (k == 0 && i == 0) { a[1] = 0.; b[1] = 1.; u[1] = 0.; g[1] = 0.; }
        else { a[1] = 0.; b[1] = 1.; u[1] = -1.; g[1] = 0.; }
        a[Nyp] = 1.; b[Nyp] = -1.; u[Nyp] = 0.; g[Nyp] = 0.;
        thomas_complex_col(a, b, u, g, Nyp);
        for (int j = 1; j <= Nyp; ++j) CV(c, cr1, i, k, j) = g[j];
      }
    free(a); free(b); free(u); free(g);
  }
  for (int j = 1; j <= Nyp; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        CV(c, cu1, i, k, j) = CV(c, cu1, i, k, j) - c->cikx[i] * CV(c, cr1, i, k, j);
        CV(c, cu3, i, k, j) = CV(c, cu3, i, k, j) - c->cikz[k] * CV(c, cr1, i, k, j);
      }
  for (int j = 2; j <= Nyp; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i)
        CV(c, cu2, i, k, j) = CV(c, cu2, i, k, j) - (CV(c, cr1, i, k, j) - CV(c, cr1, i, k, j - 1)) / c->dy[j];
}

/* ---------------------------------------------------------------------- */
/* poisson_p_chan (for/solver.f90:1382-1590): cp from the velocity and      */
/* buoyancy, for restarts without pressure.  The right-hand side is the sum */
/* of (dui/dxj)(duj/dxi) over the three diagonal and the three off-diagonal */
/* pairs, each formed in physical space from spectral derivatives and sent  */
/* back, plus the y-derivative of the buoyancy (the (0,0) mode skipped);    */
/* then one complex Thomas per (kx, kz) with apply_BC_poisson_mpi's rows    */
/* (2375-2411).  The reference uses cf1..cf3 as its work arrays; here they  */
/* are separate buffers.                                                    */

static void pp_product(orc_ctx* c, double* w1, double* w2, double fac, int square, cplx* cs) {
  int Nyp = c->Nyp;
  orc_fft_xz_to_physical(c, w1);
  if (!square) orc_fft_xz_to_physical(c, w2);
  for (int j = 2; j <= Nyp; ++j)
    for (int k = 0; k < c->Nzp; ++k)
      for (int i = 0; i < c->Nx; ++i) {
        const double a = RV(c, w1, i, k, j);
        RV(c, w1, i, k, j) = square ? a * a : fac * a * RV(c, w2, i, k, j);
      }
  orc_fft_xz_to_fourier(c, w1);
  for (int j = 2; j <= Nyp; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) cs[(long)j * (c->plane_r / 2) + (long)k * c->NXP1 + i] += CV(c, w1, i, k, j);
}

void orc_poisson_p_chan(orc_ctx* c) {
  int Nyp = c->Nyp;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  double* cth = c->arr[DB_CTH]; double* cp = c->arr[DB_CP];
  double* w1 = (double*)calloc((size_t)c->len, sizeof(double));
  double* w2 = (double*)calloc((size_t)c->len, sizeof(double));
  cplx* cs = (cplx*)calloc((size_t)c->len / 2, sizeof(cplx));
  /* the diagonal terms (dui/dxi)^2 */
  for (int t = 0; t < 3; ++t) {
    memset(w1, 0, sizeof(double) * (size_t)c->len);
    for (int j = 2; j <= Nyp; ++j)
      for (int k = 0; k <= c->twoNkz; ++k)
        for (int i = 0; i < c->Nxp; ++i)
          CV(c, w1, i, k, j) = t == 0 ? c->cikx[i] * CV(c, cu1, i, k, j)
                             : t == 1 ? (CV(c, cu2, i, k, j + 1) - CV(c, cu2, i, k, j)) / c->dyf[j]
                                      : c->cikz[k] * CV(c, cu3, i, k, j);
    pp_product(c, w1, NULL, 1.0, 1, cs);
  }
  /* the off-diagonal terms 2 (du1/dy)(du2/dx), 2 (du3/dy)(du2/dz), 2 (du1/dz)(du3/dx) */
  for (int t = 0; t < 3; ++t) {
    memset(w1, 0, sizeof(double) * (size_t)c->len);
    memset(w2, 0, sizeof(double) * (size_t)c->len);
    for (int j = 2; j <= Nyp; ++j)
      for (int k = 0; k <= c->twoNkz; ++k)
        for (int i = 0; i < c->Nxp; ++i) {
          const cplx v = 0.5 * (CV(c, cu2, i, k, j) + CV(c, cu2, i, k, j + 1));
          if (t == 0) {
            CV(c, w1, i, k, j) = (CV(c, cu1, i, k, j + 1) - CV(c, cu1, i, k, j - 1)) / (2. * c->dyf[j]);
            CV(c, w2, i, k, j) = c->cikx[i] * v;
          } else if (t == 1) {
            CV(c, w1, i, k, j) = (CV(c, cu3, i, k, j + 1) - CV(c, cu3, i, k, j - 1)) / (2. * c->dyf[j]);
            CV(c, w2, i, k, j) = c->cikz[k] * v;
          } else {
            CV(c, w1, i, k, j) = c->cikz[k] * CV(c, cu1, i, k, j);
            CV(c, w2, i, k, j) = c->cikx[i] * CV(c, cu3, i, k, j);
          }
        }
    pp_product(c, w1, w2, 2.0, 0, cs);
  }
  /* buoyancy, the (0,0) mode skipped (its hydrostatic part was cancelled) */
  for (int j = 2; j <= Nyp; ++j)
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i)
        if (i != 0 || k != 0)
          cs[(long)j * (c->plane_r / 2) + (long)k * c->NXP1 + i] +=
              (CV(c, cth, i, k, j + 1) - CV(c, cth, i, k, j - 1)) / (c->gyf[j + 1] - c->gyf[j - 1]);
  /* the Poisson solve per (kx, kz) */
  double* a = (double*)malloc(sizeof(double) * (size_t)(Nyp + 2));
  double* b = (double*)malloc(sizeof(double) * (size_t)(Nyp + 2));
  double* u = (double*)malloc(sizeof(double) * (size_t)(Nyp + 2));
  cplx* g = (cplx*)malloc(sizeof(cplx) * (size_t)(Nyp + 2));
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      for (int j = 0; j <= Nyp + 1; ++j) { a[j] = 0.; b[j] = 1.; u[j] = 0.; g[j] = 0.; }
      for (int j = 2; j <= Nyp; ++j) {
        a[j] = 1. / (c->dy[j] * c->dyf[j]);
        b[j] = -c->kx2[i] - c->kz2[k] - 1. / (c->dy[j + 1] * c->dyf[j]) - 1. / (c->dy[j] * c->dyf[j]);
        u[j] = 1. / (c->dy[j + 1] * c->dyf[j]);
        g[j] = -1. * cs[(long)j * (c->plane_r / 2) + (long)k * c->NXP1 + i];
      }
      /* apply_BC_poisson_mpi: row 1 Dirichlet for (0,0), Neumann otherwise; row Nyp Neumann */
      if (i == 0 && k == 0) { b[1] = 1.; u[1] = 0.; g[1] = 0.; }
      else { b[1] = 1.; u[1] = -1.; g[1] = 0.; }
      b[Nyp] = -1.; a[Nyp] = 1.; g[Nyp] = 0.;
      thomas_complex_col(a, b, u, g, Nyp);
      for (int j = 1; j <= Nyp; ++j) CV(c, cp, i, k, j) = g[j];
    }
  free(a); free(b); free(u); free(g);
  free(w1); free(w2); free(cs);
}

/* ---------------------------------------------------------------------- */
/* apply_BC_vel_mpi_post (for/flow.f90:1161-1360)                            */

void orc_apply_bc_vel_post(orc_ctx* c) {
  const db_params* p = &c->p;
  int Nyp = c->Nyp;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  /* lower, for/flow.f90:1170-1255 */
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->u_bc_ymin == 0) { CV(c, cu1, i, k, 0) = 0.; CV(c, cu1, i, k, 1) = 0.; }
      else { CV(c, cu1, i, k, 1) = CV(c, cu1, i, k, 2); CV(c, cu1, i, k, 0) = CV(c, cu1, i, k, 1); }
    }
  if (p->u_bc_ymin == 0) { CV(c, cu1, 0, 0, 1) = p->u_bc_ymin_c1; CV(c, cu1, 0, 0, 0) = p->u_bc_ymin_c1; }
  else {
    CV(c, cu1, 0, 0, 1) = CV(c, cu1, 0, 0, 2) - c->dy[2] * p->u_bc_ymin_c1;
    CV(c, cu1, 0, 0, 0) = CV(c, cu1, 0, 0, 1) - c->dy[1] * p->u_bc_ymin_c1;
  }
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->w_bc_ymin == 0) { CV(c, cu3, i, k, 0) = 0.; CV(c, cu3, i, k, 1) = 0.; }
      else { CV(c, cu3, i, k, 1) = CV(c, cu3, i, k, 2); CV(c, cu3, i, k, 0) = CV(c, cu3, i, k, 1); }
    }
  if (p->w_bc_ymin == 0) { CV(c, cu3, 0, 0, 1) = c->w_bc_ymin_c1; CV(c, cu3, 0, 0, 0) = c->w_bc_ymin_c1; }
  else {
    CV(c, cu3, 0, 0, 1) = CV(c, cu3, 0, 0, 2) - c->dy[2] * c->w_bc_ymin_c1;
    CV(c, cu3, 0, 0, 0) = CV(c, cu3, 0, 0, 1) - c->dy[1] * c->w_bc_ymin_c1;
  }
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->v_bc_ymin == 0) {
        CV(c, cu2, i, k, 1) = 2.0 * p->v_bc_ymin_c1 - CV(c, cu2, i, k, 2);
        CV(c, cu2, i, k, 0) = CV(c, cu2, i, k, 1);
      } else {
        CV(c, cu2, i, k, 1) = CV(c, cu2, i, k, 2);
        CV(c, cu2, i, k, 0) = CV(c, cu2, i, k, 1);
      }
    }
  if (p->v_bc_ymin == 1) {
    CV(c, cu2, 0, 0, 1) = CV(c, cu2, 0, 0, 2) - c->dyf[1] * p->v_bc_ymin_c1;
    CV(c, cu2, 0, 0, 0) = CV(c, cu2, 0, 0, 1) - c->dyf[1] * p->v_bc_ymin_c1;
  }
  /* upper, for/flow.f90:1270-1357 */
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->u_bc_ymax == 0) { CV(c, cu1, i, k, Nyp) = 0.; CV(c, cu1, i, k, Nyp + 1) = 0.; }
      else { CV(c, cu1, i, k, Nyp) = CV(c, cu1, i, k, Nyp - 1); CV(c, cu1, i, k, Nyp + 1) = CV(c, cu1, i, k, Nyp); }
    }
  if (p->u_bc_ymax == 0) { CV(c, cu1, 0, 0, Nyp) = p->u_bc_ymax_c1; CV(c, cu1, 0, 0, Nyp + 1) = p->u_bc_ymax_c1; }
  else {
    CV(c, cu1, 0, 0, Nyp) = CV(c, cu1, 0, 0, Nyp - 1) + c->dy[Nyp] * p->u_bc_ymax_c1;
    CV(c, cu1, 0, 0, Nyp + 1) = CV(c, cu1, 0, 0, Nyp) + c->dy[Nyp] * p->u_bc_ymax_c1;
  }
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->w_bc_ymax == 0) { CV(c, cu3, i, k, Nyp) = 0.; CV(c, cu3, i, k, Nyp + 1) = 0.; }
      else { CV(c, cu3, i, k, Nyp) = CV(c, cu3, i, k, Nyp - 1); CV(c, cu3, i, k, Nyp + 1) = CV(c, cu3, i, k, Nyp); }
    }
  if (p->w_bc_ymax == 0) {
    CV(c, cu3, 0, 0, Nyp) = c->w_bc_ymax_c1;
    CV(c, cu3, 0, 0, Nyp + 1) = c->w_bc_ymax_c1;
    CV(c, cu3, 0, 0, Nyp + 1) = 0.; /* "Ghost cell not used", flow.f90:1316 */
  } else {
    if (p->f_type == 4)
      c->w_bc_ymax_c1_transient = c->w_bc_ymax_c1 + p->amp_omega0 *
          sin(p->omega0 * (c->Ro_inv / p->delta * c->time - p->force_start));
    CV(c, cu3, 0, 0, Nyp) = CV(c, cu3, 0, 0, Nyp - 1) + c->dy[Nyp] * c->w_bc_ymax_c1_transient;
    CV(c, cu3, 0, 0, Nyp + 1) = CV(c, cu3, 0, 0, Nyp) + c->dy[Nyp] * c->w_bc_ymax_c1_transient;
  }
  if (p->v_bc_ymax == 0) {
    /* the reference loop writes only the (0,0) mode, flow.f90:1338-1342 */
    CV(c, cu2, 0, 0, Nyp + 1) = 2.0 * p->v_bc_ymax_c1 - CV(c, cu2, 0, 0, Nyp);
  } else {
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        CV(c, cu2, i, k, Nyp) = CV(c, cu2, i, k, Nyp - 1);
        CV(c, cu2, i, k, Nyp + 1) = CV(c, cu2, i, k, Nyp);
      }
    CV(c, cu2, 0, 0, Nyp + 1) = CV(c, cu2, 0, 0, Nyp) + c->dy[Nyp] * p->v_bc_ymax_c1;
  }
}

/* ---------------------------------------------------------------------- */
/* courant (for/flow.f90:746-857) on physical u1..u3                        */

static double fmin3(double a, double b, double c) { return fmin(a, fmin(b, c)); }

double orc_courant_physical(orc_ctx* c) {
  const db_params* p = &c->p;
  double* u1 = c->arr[DB_CU1]; double* u2 = c->arr[DB_CU2]; double* u3 = c->arr[DB_CU3];
  double dt = 1.0;
  dt = fmin(dt, 0.5 * pow(fmin(c->dx[1], c->dz[1]), 2.0 * p->beta) / c->nu);
  dt = fmin(dt, dt * c->nu / (c->nu / p->pr));
  if (c->Ro_inv != 0.0) dt = fmin(dt, 2.0 * c->pi / fabs(c->Ro_inv / p->delta) / 20.0);
  {
    double Nmax = sqrt(fabs(p->th_bc_ymin_c1));
    dt = fmin(dt, (double)0.1f * 2.0 * c->pi / Nmax);
  }
  if (p->flavor_front) {
    double f = c->Ro_inv / p->delta;
    for (int j = c->jstart; j <= c->jend; ++j)
      for (int k = 0; k < c->Nzp; ++k)
        for (int i = 0; i < c->Nx; ++i) {
          double dt_x = p->cfl * c->dx[i] / fabs(RV(c, u1, i, k, j) - c->dTHdZ * c->gyf[j] / f);
          double dt_y = p->cfl * c->dy[j] / fabs(RV(c, u2, i, k, j));
          double dt_z = p->cfl * c->dz[k] /
              fabs(RV(c, u3, i, k, j) + (1.0 / f) * c->dTHdX * (c->gyf[j] - 0.5 * p->ly));
          dt = fmin(dt, fmin3(dt_x, dt_y, dt_z));
        }
  } else {
    for (int j = 1; j <= c->Nyp; ++j)
      for (int k = 0; k < c->Nzp; ++k)
        for (int i = 0; i < c->Nx; ++i) {
          double dt_x = p->cfl * c->dx[i] / fabs(RV(c, u1, i, k, j));
          double dt_y = p->cfl * c->dy[j] / fabs(RV(c, u2, i, k, j));
          double dt_z = p->cfl * c->dz[k] / fabs(RV(c, u3, i, k, j));
          dt = fmin(dt, fmin3(dt_x, dt_y, dt_z));
        }
  }
  if (dt <= 0) c->delta_t = 0.00001;
  else if (dt >= 1000.) c->delta_t = 1000.0;
  else c->delta_t = dt;
  double tl = p->time_limit;
  double next = fmin(fmin(tl, c->save_stats_time - c->time), fmin(c->save_flow_time - c->time, tl - c->time));
  double r_max = (double)(1.0f - 0.025f);
  if (next < dt) c->delta_t = next + 1.e-14;
  else if (next < (1. + r_max) * dt) c->delta_t = 1. / (1. + r_max) * next;
  else c->delta_t = dt;
  c->h_bar[0] = c->delta_t * (8.0 / 15.0);
  c->h_bar[1] = c->delta_t * (2.0 / 15.0);
  c->h_bar[2] = c->delta_t * (5.0 / 15.0);
  return c->delta_t;
}

#define LOOP_SPEC(jlo, jhi) \
  for (int j = (jlo); j <= (jhi); ++j) \
    for (int k = 0; k <= c->twoNkz; ++k) \
      for (int i = 0; i < c->Nxp; ++i)
#define LOOP_PHYS(jlo, jhi) \
  for (int j = (jlo); j <= (jhi); ++j) \
    for (int k = 0; k < c->Nzp; ++k) \
      for (int i = 0; i < c->Nx; ++i)

/* ---------------------------------------------------------------------- */
/* LES, les_model_type 5: anisotropic minimum dissipation, Verstappen form   */
/* (for/les.f90:3-1068 model-5 branch, 1072-1435, 1443-1746, 1980-2079,      */
/* 2086-2249; BCs for/flow.f90:1161-1360, 1596-1732).                        */

enum { L_S1 = 0, L_S2, L_S3, L_S4, L_S5, L_S6,          /* Sij (strain)          */
       L_SI1, L_SI2, L_SI3, L_SI4, L_SI5, L_SI6,        /* SIij (scaled strain)  */
       L_O4, L_O5, L_O6,                                /* Oij (scaled rotation) */
       L_DU1DX, L_DU2DY, L_DU3DZ, L_DU2DX, L_DU3DX, L_DU1DZ, L_DU2DZ, L_DU1DY, L_DU3DY,
       L_DTHX, L_DTHY, L_DTHZ, L_TEMP, L_TEMP_TH, L_S1_TH };

static const double C_AMD = 0.2887;   /* les.f90:25 */
static const double BETA_SGS = 3.0;   /* les.f90:43 */

/* apply_BC_th_mpi_post (for/flow.f90:1596-1689) */
static void apply_bc_th_post(orc_ctx* c) {
  const db_params* p = &c->p;
  int Nyp = c->Nyp;
  double* cth = c->arr[DB_CTH];
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->th_bc_ymin == 0) { CV(c, cth, i, k, 0) = 0.; CV(c, cth, i, k, 1) = 0.; }
      else { CV(c, cth, i, k, 1) = CV(c, cth, i, k, 2); CV(c, cth, i, k, 0) = CV(c, cth, i, k, 1); }
    }
  if (p->th_bc_ymin == 0) { CV(c, cth, 0, 0, 1) = p->th_bc_ymin_c1; CV(c, cth, 0, 0, 0) = p->th_bc_ymin_c1; }
  else {
    CV(c, cth, 0, 0, 1) = CV(c, cth, 0, 0, 2) - c->dy[2] * p->th_bc_ymin_c1;
    CV(c, cth, 0, 0, 0) = CV(c, cth, 0, 0, 1) - c->dy[1] * p->th_bc_ymin_c1;
  }
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->th_bc_ymax == 0) { CV(c, cth, i, k, Nyp) = 0.; CV(c, cth, i, k, Nyp + 1) = 0.; }
      else { CV(c, cth, i, k, Nyp) = CV(c, cth, i, k, Nyp - 1); CV(c, cth, i, k, Nyp + 1) = CV(c, cth, i, k, Nyp); }
    }
  if (p->th_bc_ymax == 0) { CV(c, cth, 0, 0, Nyp) = p->th_bc_ymax_c1; CV(c, cth, 0, 0, Nyp + 1) = p->th_bc_ymax_c1; }
  else {
    CV(c, cth, 0, 0, Nyp) = CV(c, cth, 0, 0, Nyp - 1) + c->dy[Nyp] * p->th_bc_ymax_c1;
    CV(c, cth, 0, 0, Nyp + 1) = CV(c, cth, 0, 0, Nyp) + c->dy[Nyp] * p->th_bc_ymax_c1;
  }
}

/* apply_BC_les and apply_BC_th_les (for/les.f90:1980-2079) */
static void apply_bc_les(orc_ctx* c) {
  const db_params* p = &c->p;
  int Nyp = c->Nyp;
  double* cu1 = c->arr[DB_CU1]; double* cu3 = c->arr[DB_CU3]; double* cth = c->arr[DB_CTH];
  for (int k = 0; k <= c->twoNkz; ++k)
    for (int i = 0; i < c->Nxp; ++i) {
      if (p->u_bc_ymax == 1) { CV(c, cu1, i, k, Nyp) = CV(c, cu1, i, k, Nyp - 1); CV(c, cu1, i, k, Nyp + 1) = CV(c, cu1, i, k, Nyp); }
      if (p->w_bc_ymax == 1) { CV(c, cu3, i, k, Nyp) = CV(c, cu3, i, k, Nyp - 1); CV(c, cu3, i, k, Nyp + 1) = CV(c, cu3, i, k, Nyp); }
      if (p->u_bc_ymin == 1) { CV(c, cu1, i, k, 1) = CV(c, cu1, i, k, 2); CV(c, cu1, i, k, 0) = CV(c, cu1, i, k, 1); }
      if (p->w_bc_ymin == 1) { CV(c, cu3, i, k, 1) = CV(c, cu3, i, k, 2); CV(c, cu3, i, k, 0) = CV(c, cu3, i, k, 1); }
      if (p->th_bc_ymax == 1) { CV(c, cth, i, k, Nyp) = CV(c, cth, i, k, Nyp - 1); CV(c, cth, i, k, Nyp + 1) = CV(c, cth, i, k, Nyp); }
      if (p->th_bc_ymin == 1) { CV(c, cth, i, k, 1) = CV(c, cth, i, k, 2); CV(c, cth, i, k, 0) = CV(c, cth, i, k, 1); }
    }
}

/* the spectral tensors of compute_strain_chan, compute_strain_chan_invariant,
 * compute_rotation_chan_invariant and compute_all_gradients_chan
 * (les.f90:1443-1746), then all of them to physical space */
static void les_tensors(orc_ctx* c) {
  int Nyp = c->Nyp;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  double* cth = c->arr[DB_CTH];
  double** L = c->les;
  const double deltax = c->dx[1] * BETA_SGS, deltaz = c->dz[1] * BETA_SGS;
  for (int j = 0; j <= Nyp + 1; ++j) {
    for (int k = 0; k <= c->twoNkz; ++k)
      for (int i = 0; i < c->Nxp; ++i) {
        cplx ikx = c->cikx[i], ikz = c->cikz[k];
        cplx a1 = CV(c, cu1, i, k, j), a2 = CV(c, cu2, i, k, j), a3 = CV(c, cu3, i, k, j);
        CV(c, L[L_S1], i, k, j) = ikx * a1;
        CV(c, L[L_S3], i, k, j) = ikz * a3;
        CV(c, L[L_S5], i, k, j) = 0.5 * (ikz * a1 + ikx * a3);
        CV(c, L[L_SI1], i, k, j) = ikx * a1;
        CV(c, L[L_SI3], i, k, j) = ikz * a3;
        CV(c, L[L_SI5], i, k, j) = 0.5 * (ikz * a1 * (deltaz / deltax) + ikx * a3 * (deltax / deltaz));
        CV(c, L[L_O5], i, k, j) = 0.5 * (ikz * a1 * (deltaz / deltax) - ikx * a3 * (deltax / deltaz));
        CV(c, L[L_DU1DX], i, k, j) = ikx * a1;
        CV(c, L[L_DU1DZ], i, k, j) = ikz * a1;
        CV(c, L[L_DU2DX], i, k, j) = ikx * a2;
        CV(c, L[L_DU2DZ], i, k, j) = ikz * a2;
        CV(c, L[L_DU3DX], i, k, j) = ikx * a3;
        CV(c, L[L_DU3DZ], i, k, j) = ikz * a3;
        if (j != Nyp + 1) {
          cplx d2 = (CV(c, cu2, i, k, j + 1) - a2) / c->dyf[j];
          CV(c, L[L_S2], i, k, j) = d2;
          CV(c, L[L_SI2], i, k, j) = d2;
          CV(c, L[L_DU2DY], i, k, j) = d2;
        } else {
          /* ghost_CS2_mpi with one rank (les.f90:2505-2512) */
          CV(c, L[L_S2], i, k, j) = -10000.0;
          CV(c, L[L_SI2], i, k, j) = -10000.0;
          /* the reference reads cu2(Nyp+2), outside its array; the value
           * only reaches rows the model never uses (les.f90:1679, 1266) */
          CV(c, L[L_DU2DY], i, k, j) = 0.0;
        }
        if (j >= 1) {
          const double deltay = c->dy[j] * 2.0;
          cplx d1 = (a1 - CV(c, cu1, i, k, j - 1)) / c->dy[j];
          cplx d3 = (a3 - CV(c, cu3, i, k, j - 1)) / c->dy[j];
          CV(c, L[L_S4], i, k, j) = 0.5 * (d1 + ikx * a2);
          CV(c, L[L_S6], i, k, j) = 0.5 * (ikz * a2 + d3);
          CV(c, L[L_SI4], i, k, j) = 0.5 * (d1 * (deltay / deltax) + ikx * a2 * (deltax / deltay));
          CV(c, L[L_SI6], i, k, j) = 0.5 * (ikz * a2 * (deltaz / deltay) + d3 * (deltay / deltaz));
          CV(c, L[L_O4], i, k, j) = 0.5 * (d1 * (deltay / deltax) - ikx * a2 * (deltax / deltay));
          CV(c, L[L_O6], i, k, j) = 0.5 * (ikz * a2 * (deltaz / deltay) - d3 * (deltay / deltaz));
          CV(c, L[L_DU1DY], i, k, j) = d1;
          CV(c, L[L_DU3DY], i, k, j) = d3;
          cplx t = CV(c, cth, i, k, j);
          CV(c, L[L_DTHX], i, k, j) = ikx * t;
          CV(c, L[L_DTHZ], i, k, j) = ikz * t;
          CV(c, L[L_DTHY], i, k, j) = (t - CV(c, cth, i, k, j - 1)) / c->dy[j];
        }
      }
  }
  for (int a = L_S1; a <= L_DTHZ; ++a) orc_fft_xz_to_physical(c, L[a]);
}

/* AMD eddy viscosity and SGS stress divergence (les.f90:551-900) */
static void les_chan(orc_ctx* c, int rk_step) {
  (void)rk_step;
  int Nyp = c->Nyp, js = c->jstart, je = c->jend;
  double** L = c->les;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  double* cf1 = c->arr[DB_CF1]; double* cf2 = c->arr[DB_CF2]; double* cf3 = c->arr[DB_CF3];
  double* nu_t = c->arr[DB_NU_T];
  double *u1 = cu1, *u2 = cu2, *u3 = cu3;
  /* j1, j2 with one rank: the "upper wall" branch (les.f90:46-49) */
  const int j1 = js, j2 = Nyp - 1;
  orc_apply_bc_vel_post(c);           /* les.f90:63 */
  apply_bc_th_post(c);                /* les.f90:64 */
  apply_bc_les(c);                    /* les.f90:74-75 */
  les_tensors(c);                     /* les.f90:555-564 */
  orc_fft_xz_to_physical(c, cu1);     /* les.f90:567-569 */
  orc_fft_xz_to_physical(c, cu2);
  orc_fft_xz_to_physical(c, cu3);
#define SI(n, i, k, j) RV(c, L[L_SI##n], i, k, j)
#define OO(n, i, k, j) RV(c, L[L_O##n], i, k, j)
  double* s1 = c->arr[A_S1];
  double* temp = L[L_TEMP];
  /* max{0, -(I3-I4)}/(I1-I2) at GYF points (les.f90:574-623) */
  LOOP_PHYS(js, je) {
    double s4 = 0.5 * (SI(4, i, k, j + 1) + SI(4, i, k, j)), s6 = 0.5 * (SI(6, i, k, j + 1) + SI(6, i, k, j));
    double o4 = 0.5 * (OO(4, i, k, j + 1) + OO(4, i, k, j)), o6 = 0.5 * (OO(6, i, k, j + 1) + OO(6, i, k, j));
    double s1v = SI(1, i, k, j), s2v = SI(2, i, k, j), s3v = SI(3, i, k, j), s5 = SI(5, i, k, j), o5 = OO(5, i, k, j);
    double v = s1v * s1v * s1v + s2v * s2v * s2v + s3v * s3v * s3v
             + 3.0 * s1v * s4 * s4 + 3.0 * s1v * s5 * s5 + 3.0 * s2v * s4 * s4 + 3.0 * s2v * s6 * s6
             + 3.0 * s3v * s5 * s5 + 3.0 * s3v * s6 * s6 + 6.0 * s4 * s5 * s6;
    v = (-v - s1v * o4 * o4 - s1v * o5 * o5 - s2v * o4 * o4 - s2v * o6 * o6 - s3v * o5 * o5 - s3v * o6 * o6
         - 2.0 * s4 * o5 * o6 + 2.0 * s5 * o4 * o6 - 2.0 * s6 * o4 * o5);
    if (v <= 0.0) v = 0.0;
    else v = v / (s1v * s1v + s2v * s2v + s3v * s3v + 2.0 * s4 * s4 + 2.0 * o4 * o4 + 2.0 * s5 * s5
                  + 2.0 * o5 * o5 + 2.0 * s6 * s6 + 2.0 * o6 * o6);
    RV(c, s1, i, k, j) = v;
  }
  /* the same at GY points (les.f90:628-719) */
  LOOP_PHYS(2, Nyp) {
    double w = 1.0 / (2.0 * c->dy[j]);
#define GI(X) ((X(i, k, j) * c->dyf[j - 1] + X(i, k, j - 1) * c->dyf[j]) * w)
#define SIA1(i, k, j) SI(1, i, k, j)
#define SIA2(i, k, j) SI(2, i, k, j)
#define SIA3(i, k, j) SI(3, i, k, j)
#define SIA5(i, k, j) SI(5, i, k, j)
#define OA5(i, k, j) OO(5, i, k, j)
    double s1v = GI(SIA1), s2v = GI(SIA2), s3v = GI(SIA3), s5 = GI(SIA5), o5 = GI(OA5);
    double s4 = SI(4, i, k, j), s6 = SI(6, i, k, j), o4 = OO(4, i, k, j), o6 = OO(6, i, k, j);
    double v = s1v * s1v * s1v + s2v * s2v * s2v + s3v * s3v * s3v
             + 3.0 * s1v * s4 * s4 + 3.0 * s1v * s5 * s5 + 3.0 * s2v * s4 * s4 + 3.0 * s2v * s6 * s6
             + 3.0 * s3v * s5 * s5 + 3.0 * s3v * s6 * s6 + 6.0 * s4 * s6 * s5;
    v = -v - s1v * o4 * o4 - s1v * o5 * o5 - s2v * o4 * o4 - s2v * o6 * o6 - s3v * o5 * o5 - s3v * o6 * o6
        - 2.0 * s4 * o5 * o6 + 2.0 * s5 * o4 * o6 - 2.0 * s6 * o4 * o5;
    if (v <= 0.0) v = 0.0;
    else v = v / (s1v * s1v + s2v * s2v + s3v * s3v + 2.0 * s4 * s4 + 2.0 * o4 * o4 + 2.0 * s5 * s5
                  + 2.0 * o5 * o5 + 2.0 * s6 * s6 + 2.0 * o6 * o6);
    RV(c, temp, i, k, j) = v;
  }
#undef GI
  /* les.f90:724-750 */
  LOOP_PHYS(js, je) {
    double f = RV(c, s1, i, k, j);
    RV(c, L[L_S1], i, k, j) = f * RV(c, L[L_S1], i, k, j);
    RV(c, L[L_S5], i, k, j) = f * RV(c, L[L_S5], i, k, j);
    RV(c, L[L_S2], i, k, j) = 0.0;
    RV(c, L[L_S3], i, k, j) = f * RV(c, L[L_S3], i, k, j);
  }
  LOOP_PHYS(2, Nyp + 1) {
    double f = RV(c, temp, i, k, j);
    RV(c, L[L_S4], i, k, j) = f * (RV(c, L[L_S4], i, k, j) - 0.5 * (RV(c, u1, i, k, j) - RV(c, u1, i, k, j - 1)) / c->dy[j]);
    RV(c, L[L_S6], i, k, j) = f * (RV(c, L[L_S6], i, k, j) - 0.5 * (RV(c, u3, i, k, j) - RV(c, u3, i, k, j - 1)) / c->dy[j]);
  }
  /* filter widths with -2 C^2 absorbed (les.f90:756-780) */
  double* dyf_w = (double*)calloc(Nyp + 2, sizeof(double));
  double* dy_w = (double*)calloc(Nyp + 2, sizeof(double));
  for (int j = 1; j <= Nyp + 1; ++j) {
    dyf_w[j] = -2.0 * C_AMD * C_AMD * 3.0 /
        (1.0 / pow(c->dx[1] * BETA_SGS, 2.0) + 1.0 / pow(c->dyf[j] * 2.0, 2.0) + 1.0 / pow(c->dz[1] * BETA_SGS, 2.0));
    dy_w[j] = -2.0 * C_AMD * C_AMD * 3.0 /
        (1.0 / pow(c->dx[1] * BETA_SGS, 2.0) + 1.0 / pow(c->dy[j] * 2.0, 2.0) + 1.0 / pow(c->dz[1] * BETA_SGS, 2.0));
  }
  LOOP_PHYS(2, Nyp + 1) RV(c, nu_t, i, k, j) = -0.5 * dy_w[j] * RV(c, temp, i, k, j);
  /* ghost_les_mpi with one rank: nu_t = 0 at both walls (les.f90:2229-2244) */
  for (int k = 0; k < c->Nzp; ++k)
    for (int i = 0; i < c->Nx; ++i) {
      RV(c, nu_t, i, k, 1) = 0.0; RV(c, nu_t, i, k, 2) = 0.0;
      RV(c, nu_t, i, k, Nyp) = 0.0; RV(c, nu_t, i, k, Nyp + 1) = 0.0;
    }
  /* stress to Fourier space and its divergence (les.f90:800-866) */
  orc_fft_xz_to_fourier(c, L[L_S1]);
  orc_fft_xz_to_fourier(c, L[L_S3]);
  orc_fft_xz_to_fourier(c, L[L_S4]);
  orc_fft_xz_to_fourier(c, L[L_S5]);
  orc_fft_xz_to_fourier(c, L[L_S6]);
  LOOP_SPEC(1, Nyp) {
    CV(c, L[L_S1], i, k, j) = dyf_w[j] * CV(c, L[L_S1], i, k, j);
    CV(c, L[L_S5], i, k, j) = dyf_w[j] * CV(c, L[L_S5], i, k, j);
    CV(c, L[L_S3], i, k, j) = dyf_w[j] * CV(c, L[L_S3], i, k, j);
  }
  LOOP_SPEC(1, Nyp + 1) {
    CV(c, L[L_S4], i, k, j) = dy_w[j] * CV(c, L[L_S4], i, k, j);
    CV(c, L[L_S6], i, k, j) = dy_w[j] * CV(c, L[L_S6], i, k, j);
  }
  LOOP_SPEC(j1, j2) {
    CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j) - c->cikx[i] * CV(c, L[L_S1], i, k, j)
        - (CV(c, L[L_S4], i, k, j + 1) - CV(c, L[L_S4], i, k, j)) / c->dyf[j] - c->cikz[k] * CV(c, L[L_S5], i, k, j);
    CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j) - c->cikx[i] * CV(c, L[L_S5], i, k, j)
        - (CV(c, L[L_S6], i, k, j + 1) - CV(c, L[L_S6], i, k, j)) / c->dyf[j] - c->cikz[k] * CV(c, L[L_S3], i, k, j);
  }
  LOOP_SPEC(2, Nyp)
    CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) - c->cikx[i] * CV(c, L[L_S4], i, k, j) - c->cikz[k] * CV(c, L[L_S6], i, k, j);
  /* explicit cross terms nu_t d(u1,u3)/dy (les.f90:871-900) */
  LOOP_PHYS(2, Nyp) RV(c, temp, i, k, j) = RV(c, nu_t, i, k, j) * (RV(c, u1, i, k, j) - RV(c, u1, i, k, j - 1)) / c->dy[j];
  orc_fft_xz_to_fourier(c, temp);
  LOOP_SPEC(2, Nyp) CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) + c->cikx[i] * CV(c, temp, i, k, j);
  LOOP_PHYS(2, Nyp) RV(c, temp, i, k, j) = RV(c, nu_t, i, k, j) * (RV(c, u3, i, k, j) - RV(c, u3, i, k, j - 1)) / c->dy[j];
  orc_fft_xz_to_fourier(c, temp);
  LOOP_SPEC(2, Nyp) CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) + c->cikz[k] * CV(c, temp, i, k, j);
  free(dyf_w);
  free(dy_w);
}

/* scalar AMD eddy diffusivity and SGS flux divergence (les.f90:1201-1395) */
static void les_chan_th(orc_ctx* c) {
  int Nyp = c->Nyp, jst = c->jstart_th, jet = c->jend_th;
  double** L = c->les;
  double* cth = c->arr[DB_CTH];
  double* cfth = c->arr[DB_CFTH];
  double* kappa_t = c->arr[DB_KAPPA_T];
  orc_fft_xz_to_physical(c, cth);
  const double dxs = c->dx[1] * BETA_SGS, dzs = c->dz[1] * BETA_SGS;
#define G(a, i, k, j) RV(c, L[a], i, k, j)
  LOOP_PHYS(jst, jet) {
    const double dys = c->dyf[j] * 2.0;
    const double ty = 0.5 * (G(L_DTHY, i, k, j + 1) + G(L_DTHY, i, k, j));
    const double tx = G(L_DTHX, i, k, j), tz = G(L_DTHZ, i, k, j);
    double v = -(dxs * dxs * G(L_DU1DX, i, k, j) * tx * tx
                 + dys * dys * G(L_DU2DY, i, k, j) * ty * ty
                 + dzs * dzs * G(L_DU3DZ, i, k, j) * tz * tz
                 + (dys * dys * 0.5 * (G(L_DU1DY, i, k, j + 1) + G(L_DU1DY, i, k, j))
                    + dxs * dxs * 0.5 * (G(L_DU2DX, i, k, j + 1) + G(L_DU2DX, i, k, j))) * tx * ty
                 + (dzs * dzs * G(L_DU1DZ, i, k, j) + dxs * dxs * G(L_DU3DX, i, k, j)) * tx * tz
                 + (dzs * dzs * 0.5 * (G(L_DU2DZ, i, k, j + 1) + G(L_DU2DZ, i, k, j))
                    + dys * dys * 0.5 * (G(L_DU3DY, i, k, j + 1) + G(L_DU3DY, i, k, j))) * ty * tz);
    if (v <= 0.0) v = 0.0;
    else v = v / ((dxs * tx) * (dxs * tx) + (dys * ty) * (dys * ty) + (dzs * tz) * (dzs * tz));
    RV(c, L[L_S1_TH], i, k, j) = v;
  }
  LOOP_PHYS(2, Nyp) {   /* temp_th at GY; row Nyp+1 of the reference is never used */
    const double dys = c->dy[j] * 2.0, w = 1.0 / (2.0 * c->dy[j]);
#define GY(a) ((G(a, i, k, j) * c->dyf[j - 1] + G(a, i, k, j - 1) * c->dyf[j]) * w)
    const double tx = GY(L_DTHX), tz = GY(L_DTHZ), ty = G(L_DTHY, i, k, j);
    double v = -(dxs * dxs * GY(L_DU1DX) * tx * tx
                 + dys * dys * GY(L_DU2DY) * ty * ty
                 + dzs * dzs * GY(L_DU3DZ) * tz * tz
                 + (dys * dys * G(L_DU1DY, i, k, j) + dxs * dxs * G(L_DU2DX, i, k, j)) * tx * ty
                 + (dzs * dzs * GY(L_DU1DZ) + dxs * dxs * GY(L_DU3DX)) * tx * tz
                 + (dzs * dzs * G(L_DU2DZ, i, k, j) + dys * dys * G(L_DU3DY, i, k, j)) * ty * tz);
#undef GY
    if (v <= 0.0) v = 0.0;
    else v = v / ((dxs * tx) * (dxs * tx) + (dys * ty) * (dys * ty) + (dzs * tz) * (dzs * tz));
    RV(c, L[L_TEMP_TH], i, k, j) = v;
  }
  LOOP_PHYS(jst, jet) {
    RV(c, L[L_DTHX], i, k, j) = RV(c, L[L_S1_TH], i, k, j) * RV(c, L[L_DTHX], i, k, j);
    RV(c, L[L_DTHZ], i, k, j) = RV(c, L[L_S1_TH], i, k, j) * RV(c, L[L_DTHZ], i, k, j);
  }
  double* dyf_w = (double*)calloc(Nyp + 2, sizeof(double));
  double* dy_w = (double*)calloc(Nyp + 2, sizeof(double));
  for (int j = 1; j <= Nyp + 1; ++j) {
    dyf_w[j] = -2.0 * C_AMD * C_AMD * 3.0 /
        (1.0 / pow(c->dx[1] * BETA_SGS, 2.0) + 1.0 / pow(c->dyf[j] * 2.0, 2.0) + 1.0 / pow(c->dz[1] * BETA_SGS, 2.0));
    dy_w[j] = -2.0 * C_AMD * C_AMD * 3.0 /
        (1.0 / pow(c->dx[1] * BETA_SGS, 2.0) + 1.0 / pow(c->dy[j] * 2.0, 2.0) + 1.0 / pow(c->dz[1] * BETA_SGS, 2.0));
  }
  LOOP_PHYS(2, Nyp) RV(c, kappa_t, i, k, j) = -0.5 * dy_w[j] * RV(c, L[L_TEMP_TH], i, k, j);
  /* ghost_les_th_mpi with one rank (les.f90:2396-2411) */
  for (int k = 0; k < c->Nzp; ++k)
    for (int i = 0; i < c->Nx; ++i) {
      RV(c, kappa_t, i, k, 1) = 0.0; RV(c, kappa_t, i, k, 2) = 0.0;
      RV(c, kappa_t, i, k, Nyp) = 0.0; RV(c, kappa_t, i, k, Nyp + 1) = 0.0;
    }
  orc_fft_xz_to_fourier(c, L[L_DTHX]);
  orc_fft_xz_to_fourier(c, L[L_DTHZ]);
  LOOP_SPEC(1, Nyp + 1) {
    CV(c, L[L_DTHX], i, k, j) = 0.5 * dyf_w[j] * CV(c, L[L_DTHX], i, k, j);
    CV(c, L[L_DTHZ], i, k, j) = 0.5 * dyf_w[j] * CV(c, L[L_DTHZ], i, k, j);
  }
  LOOP_SPEC(jst, jet)
    CV(c, cfth, i, k, j) = CV(c, cfth, i, k, j) - c->cikx[i] * CV(c, L[L_DTHX], i, k, j)
                           - c->cikz[k] * CV(c, L[L_DTHZ], i, k, j);
  free(dyf_w);
  free(dy_w);
#undef G
}

/* ---------------------------------------------------------------------- */
/* rk_chan_1 (for/solver.f90:366-1273), DNS path                            */

int orc_rk_chan_1(orc_ctx* c, int rk_step) {
  const db_params* p = &c->p;
  if (rk_step < 1 || rk_step > 3) return -1;
  if (p->use_les && p->les_model_type != 5) {
    snprintf(g_err, sizeof g_err, "oracle: only LES model 5 (AMD, Verstappen) is restated");
    return -1;
  }
  int Nyp = c->Nyp, js = c->jstart, je = c->jend, jst = c->jstart_th, jet = c->jend_th;
  double nu = c->nu, beta = p->beta, nvs = p->nu_v_scale, Pr = p->pr;
  double* cu1 = c->arr[DB_CU1]; double* cu2 = c->arr[DB_CU2]; double* cu3 = c->arr[DB_CU3];
  double* cp = c->arr[DB_CP]; double* cth = c->arr[DB_CTH];
  double* cf1 = c->arr[DB_CF1]; double* cf2 = c->arr[DB_CF2]; double* cf3 = c->arr[DB_CF3];
  double* cfth = c->arr[DB_CFTH];
  double* cr1 = c->arr[A_R1]; double* cr2 = c->arr[A_R2]; double* cr3 = c->arr[A_R3];
  double* crth = c->arr[A_RTH]; double* cs1 = c->arr[A_S1];
  /* physical aliases */
  double *u1 = cu1, *u2 = cu2, *u3 = cu3, *th = cth, *r1 = cr1, *r2 = cr2, *r3 = cr3, *rth = crth, *s1 = cs1;

  /* :385-389 */
  int rk = rk_step - 1;
  double temp1 = 0.5 * nu * c->h_bar[rk];
  double temp2 = 0.5 * c->h_bar[rk];
  double temp3 = c->zeta_bar[rk] * c->h_bar[rk];
  double temp4 = c->h_bar[rk];
  double temp5 = c->beta_bar[rk] * c->h_bar[rk];

  /* :396-410 */
  LOOP_SPEC(js, je) { CV(c, cr1, i, k, j) = CV(c, cu1, i, k, j); CV(c, cr3, i, k, j) = CV(c, cu3, i, k, j); }
  LOOP_SPEC(2, Nyp) CV(c, cr2, i, k, j) = CV(c, cu2, i, k, j);
  /* :413-429 */
  if (rk_step > 1) {
    LOOP_SPEC(js, je) {
      CV(c, cr1, i, k, j) = CV(c, cr1, i, k, j) + temp3 * CV(c, cf1, i, k, j);
      CV(c, cr3, i, k, j) = CV(c, cr3, i, k, j) + temp3 * CV(c, cf3, i, k, j);
    }
    LOOP_SPEC(2, Nyp) CV(c, cr2, i, k, j) = CV(c, cr2, i, k, j) + temp3 * CV(c, cf2, i, k, j);
  }
  /* :432-456 */
  LOOP_SPEC(2, Nyp) CV(c, cs1, i, k, j) = (CV(c, cp, i, k, j) - CV(c, cp, i, k, j - 1)) / c->dy[j];
  LOOP_SPEC(js, je) {
    CV(c, cr1, i, k, j) = CV(c, cr1, i, k, j) - temp4 * (c->cikx[i] * CV(c, cp, i, k, j));
    CV(c, cr3, i, k, j) = CV(c, cr3, i, k, j) - temp4 * (c->cikz[k] * CV(c, cp, i, k, j));
  }
  LOOP_SPEC(2, Nyp) CV(c, cr2, i, k, j) = CV(c, cr2, i, k, j) - temp4 * CV(c, cs1, i, k, j);
  /* :464-476 */
  if (p->f_type == 1) {
    for (int j = js; j <= je; ++j) CV(c, cr1, 0, 0, j) = CV(c, cr1, 0, 0, j) - temp4 * p->px0;
  } else if (p->f_type == 2) {
    for (int j = js; j <= je; ++j)
      CV(c, cr1, 0, 0, j) = CV(c, cr1, 0, 0, j) - temp4 * (p->px0 + p->amp_omega0 * cos(p->omega0 * c->time));
  }
  /* :484-498 */
  LOOP_SPEC(js, je) {
    double kk = pow(c->kx2[i] + c->kz2[k], beta);
    CV(c, cf1, i, k, j) = -nu * kk * CV(c, cu1, i, k, j);
    CV(c, cf3, i, k, j) = -nu * kk * CV(c, cu3, i, k, j);
  }
  LOOP_SPEC(2, Nyp) CV(c, cf2, i, k, j) = -nu * pow(c->kx2[i] + c->kz2[k], beta) * CV(c, cu2, i, k, j);
  /* Coriolis :502-509 */
  LOOP_SPEC(js, je) {
    CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j) + (c->Ro_inv / p->delta) * CV(c, cu3, i, k, j);
    CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j) - (c->Ro_inv / p->delta) * CV(c, cu1, i, k, j);
  }
  /* buoyancy :518-554, skipping the (0,0) mode */
  LOOP_SPEC(2, Nyp) {
    if (k == 0 && i == 0) continue;
    CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) + p->grav_y *
        (CV(c, cth, i, k, j) * c->dyf[j - 1] + CV(c, cth, i, k, j - 1) * c->dyf[j]) / (2.0 * c->dy[j]);
  }
  LOOP_SPEC(js, je) CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j) + p->grav_x * CV(c, cth, i, k, j);
  LOOP_SPEC(js, je) CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j) + p->grav_z * CV(c, cth, i, k, j);
  /* scalar RHS :565-602 */
  LOOP_SPEC(jst, jet) CV(c, crth, i, k, j) = CV(c, cth, i, k, j);
  if (rk_step > 1) LOOP_SPEC(jst, jet) CV(c, crth, i, k, j) = CV(c, crth, i, k, j) + temp3 * CV(c, cfth, i, k, j);
  LOOP_SPEC(jst, jet) CV(c, cfth, i, k, j) = -(nu / Pr) * pow(c->kx2[i] + c->kz2[k], beta) * CV(c, cth, i, k, j);
  LOOP_SPEC(jst, jet)
    CV(c, cfth, i, k, j) = CV(c, cfth, i, k, j) - CV(c, cu1, i, k, j) * c->dTHdX - CV(c, cu3, i, k, j) * c->dTHdZ;
  /* :609 */
  user_rhs_chan_fourier(c);
  /* :615-645 */
  if (p->use_les && (!p->create_new_flow || c->time_step > 100)) {
    les_chan(c, rk_step);
    les_chan_th(c);
  } else {
    orc_fft_xz_to_physical(c, cu1);
    orc_fft_xz_to_physical(c, cu2);
    orc_fft_xz_to_physical(c, cu3);
    orc_fft_xz_to_physical(c, cth);
  }

  /* nonlinear terms :655-815 */
  LOOP_PHYS(js, je) RV(c, s1, i, k, j) = RV(c, u3, i, k, j) * RV(c, u1, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(js, je) {
    CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j) - c->cikz[k] * CV(c, cs1, i, k, j);
    CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j) - c->cikx[i] * CV(c, cs1, i, k, j);
  }
  LOOP_PHYS(js, je) RV(c, s1, i, k, j) = RV(c, u1, i, k, j) * RV(c, u1, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(js, je) CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j) - c->cikx[i] * CV(c, cs1, i, k, j);
  LOOP_PHYS(js, je) RV(c, s1, i, k, j) = RV(c, u3, i, k, j) * RV(c, u3, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(js, je) CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j) - c->cikz[k] * CV(c, cs1, i, k, j);
  LOOP_PHYS(2, Nyp)
    RV(c, s1, i, k, j) = ((c->dyf[j] * RV(c, u1, i, k, j) + c->dyf[j - 1] * RV(c, u1, i, k, j - 1)) /
                          (2. * c->dy[j])) * RV(c, u2, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(2, Nyp) CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) - c->cikx[i] * CV(c, cs1, i, k, j);
  LOOP_PHYS(2, Nyp)
    RV(c, s1, i, k, j) = ((c->dyf[j] * RV(c, u3, i, k, j) + c->dyf[j - 1] * RV(c, u3, i, k, j - 1)) /
                          (2. * c->dy[j])) * RV(c, u2, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(2, Nyp) CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) - c->cikz[k] * CV(c, cs1, i, k, j);
  LOOP_PHYS(js, je)
    RV(c, s1, i, k, j) = (RV(c, u1, i, k, j + 1) * RV(c, u2, i, k, j + 1) + RV(c, u1, i, k, j) * RV(c, u2, i, k, j + 1)
                          - RV(c, u1, i, k, j) * RV(c, u2, i, k, j) - RV(c, u1, i, k, j - 1) * RV(c, u2, i, k, j)) /
                         (2.0 * c->dyf[j]);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(js, je) CV(c, cf1, i, k, j) = CV(c, cf1, i, k, j) - CV(c, cs1, i, k, j);
  LOOP_PHYS(js, je)
    RV(c, s1, i, k, j) = (RV(c, u3, i, k, j + 1) * RV(c, u2, i, k, j + 1) + RV(c, u3, i, k, j) * RV(c, u2, i, k, j + 1)
                          - RV(c, u3, i, k, j) * RV(c, u2, i, k, j) - RV(c, u3, i, k, j - 1) * RV(c, u2, i, k, j)) /
                         (2.0 * c->dyf[j]);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(js, je) CV(c, cf3, i, k, j) = CV(c, cf3, i, k, j) - CV(c, cs1, i, k, j);
  LOOP_PHYS(2, Nyp) {
    double a = RV(c, u2, i, k, j) + RV(c, u2, i, k, j + 1);
    double b = RV(c, u2, i, k, j) + RV(c, u2, i, k, j - 1);
    RV(c, s1, i, k, j) = (0.25 * (a * a) - 0.25 * (b * b)) / c->dy[j];
  }
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(2, Nyp) CV(c, cf2, i, k, j) = CV(c, cf2, i, k, j) - CV(c, cs1, i, k, j);

  /* :824-838 */
  LOOP_SPEC(js, je) {
    CV(c, cr1, i, k, j) = CV(c, cr1, i, k, j) + temp5 * CV(c, cf1, i, k, j);
    CV(c, cr3, i, k, j) = CV(c, cr3, i, k, j) + temp5 * CV(c, cf3, i, k, j);
  }
  LOOP_SPEC(2, Nyp) CV(c, cr2, i, k, j) = CV(c, cr2, i, k, j) + temp5 * CV(c, cf2, i, k, j);
  /* :841-843 */
  orc_fft_xz_to_physical(c, cr1);
  orc_fft_xz_to_physical(c, cr2);
  orc_fft_xz_to_physical(c, cr3);
  /* CN explicit :850-870 */
  LOOP_PHYS(js, je) {
    RV(c, r1, i, k, j) = RV(c, r1, i, k, j) + temp1 * nvs *
        (((RV(c, u1, i, k, j + 1) - RV(c, u1, i, k, j)) / c->dy[j + 1] -
          (RV(c, u1, i, k, j) - RV(c, u1, i, k, j - 1)) / c->dy[j]) / c->dyf[j]);
    RV(c, r3, i, k, j) = RV(c, r3, i, k, j) + temp1 * nvs *
        (((RV(c, u3, i, k, j + 1) - RV(c, u3, i, k, j)) / c->dy[j + 1] -
          (RV(c, u3, i, k, j) - RV(c, u3, i, k, j - 1)) / c->dy[j]) / c->dyf[j]);
  }
  LOOP_PHYS(2, Nyp)
    RV(c, r2, i, k, j) = RV(c, r2, i, k, j) + temp1 * nvs *
        (((RV(c, u2, i, k, j + 1) - RV(c, u2, i, k, j)) / c->dyf[j] -
          (RV(c, u2, i, k, j) - RV(c, u2, i, k, j - 1)) / c->dyf[j - 1]) / c->dy[j]);
  if (p->use_les) { /* :875-903, nu_t at GY points */
    double* nt = c->arr[DB_NU_T];
    LOOP_PHYS(js, je) {
      RV(c, r1, i, k, j) = RV(c, r1, i, k, j) + temp2 *
          ((RV(c, nt, i, k, j + 1) * (RV(c, u1, i, k, j + 1) - RV(c, u1, i, k, j)) / c->dy[j + 1]
            - RV(c, nt, i, k, j) * (RV(c, u1, i, k, j) - RV(c, u1, i, k, j - 1)) / c->dy[j]) / c->dyf[j]);
      RV(c, r3, i, k, j) = RV(c, r3, i, k, j) + temp2 *
          ((RV(c, nt, i, k, j + 1) * (RV(c, u3, i, k, j + 1) - RV(c, u3, i, k, j)) / c->dy[j + 1]
            - RV(c, nt, i, k, j) * (RV(c, u3, i, k, j) - RV(c, u3, i, k, j - 1)) / c->dy[j]) / c->dyf[j]);
    }
    LOOP_PHYS(2, Nyp)
      RV(c, r2, i, k, j) = RV(c, r2, i, k, j) + temp2 *
          ((0.5 * (RV(c, nt, i, k, j) + RV(c, nt, i, k, j + 1))) * (RV(c, u2, i, k, j + 1) - RV(c, u2, i, k, j))
               / c->dyf[j]
           - 0.5 * (RV(c, nt, i, k, j) + RV(c, nt, i, k, j - 1)) * (RV(c, u2, i, k, j) - RV(c, u2, i, k, j - 1))
               / c->dyf[j - 1]) / c->dy[j];
  }

  /* scalar :914-973 */
  LOOP_PHYS(jst, jet) RV(c, s1, i, k, j) = RV(c, th, i, k, j) * RV(c, u1, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(jst, jet) CV(c, cfth, i, k, j) = CV(c, cfth, i, k, j) - c->cikx[i] * CV(c, cs1, i, k, j);
  LOOP_PHYS(jst, jet) RV(c, s1, i, k, j) = RV(c, th, i, k, j) * RV(c, u3, i, k, j);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(jst, jet) CV(c, cfth, i, k, j) = CV(c, cfth, i, k, j) - c->cikz[k] * CV(c, cs1, i, k, j);
  LOOP_PHYS(jst, jet)
    RV(c, s1, i, k, j) = (RV(c, th, i, k, j + 1) * RV(c, u2, i, k, j + 1) + RV(c, th, i, k, j) * RV(c, u2, i, k, j + 1)
                          - RV(c, th, i, k, j) * RV(c, u2, i, k, j) - RV(c, th, i, k, j - 1) * RV(c, u2, i, k, j)) /
                         (2.0 * c->dyf[j]);
  orc_fft_xz_to_fourier(c, s1);
  LOOP_SPEC(jst, jet) CV(c, cfth, i, k, j) = CV(c, cfth, i, k, j) - CV(c, cs1, i, k, j);
  LOOP_SPEC(jst, jet) CV(c, crth, i, k, j) = CV(c, crth, i, k, j) + temp5 * CV(c, cfth, i, k, j);
  /* :977 */
  orc_fft_xz_to_physical(c, crth);
  /* :981-989 */
  LOOP_PHYS(jst, jet)
    RV(c, rth, i, k, j) = RV(c, rth, i, k, j) + (temp1 / Pr) * nvs *
        (((RV(c, th, i, k, j + 1) - RV(c, th, i, k, j)) / c->dy[j + 1] -
          (RV(c, th, i, k, j) - RV(c, th, i, k, j - 1)) / c->dy[j]) / c->dyf[j]);
  if (p->use_les) { /* :992-1002, kappa_t at GY points */
    double* kt = c->arr[DB_KAPPA_T];
    LOOP_PHYS(jst, jet)
      RV(c, rth, i, k, j) = RV(c, rth, i, k, j) + temp2 *
          ((RV(c, kt, i, k, j + 1) * (RV(c, th, i, k, j + 1) - RV(c, th, i, k, j)) / c->dy[j + 1]
            - RV(c, kt, i, k, j) * (RV(c, th, i, k, j) - RV(c, th, i, k, j - 1)) / c->dy[j]) / c->dyf[j]);
  }

  /* implicit solves, one z-plane k at a time (every row 0..Nyp+1 of the
   * system is rewritten each k by the interior loop or the BC routines, so
   * planes are independent). */
  int Nx = c->Nx, NR = Nyp + 2;
#pragma omp parallel
  {
    tri_t t;
    t.nx = Nx;
    t.l = (double*)malloc(sizeof(double) * (size_t)Nx * NR);
    t.d = (double*)malloc(sizeof(double) * (size_t)Nx * NR);
    t.u = (double*)malloc(sizeof(double) * (size_t)Nx * NR);
    t.v = (double*)malloc(sizeof(double) * (size_t)Nx * NR);
    double tth = temp1 / Pr * nvs, tv = temp1 * nvs;
#pragma omp for schedule(static)
    for (int k = 0; k < c->Nzp; ++k) {
      /* TH :1013-1060 */
      for (int j = 0; j < NR; ++j) set_row(t, j, 0., 1., 0., 0.);
      for (int j = jst; j <= jet; ++j)
        for (int i = 0; i < Nx; ++i) {
          TL(t, i, j) = -(tth) / (c->dy[j] * c->dyf[j]);
          TD(t, i, j) = 1. + (tth) / (c->dy[j + 1] * c->dyf[j]) + (tth) / (c->dy[j] * c->dyf[j]);
          TU(t, i, j) = -(tth) / (c->dy[j + 1] * c->dyf[j]);
          TVv(t, i, j) = RV(c, rth, i, k, j);
        }
      if (p->use_les) { /* :1032-1045 */
        double* kt = c->arr[DB_KAPPA_T];
        for (int j = jst; j <= jet; ++j)
          for (int i = 0; i < Nx; ++i) {
            TL(t, i, j) = TL(t, i, j) - temp2 * RV(c, kt, i, k, j) / (c->dy[j] * c->dyf[j]);
            TD(t, i, j) = TD(t, i, j) + temp2 * RV(c, kt, i, k, j + 1) / (c->dy[j + 1] * c->dyf[j])
                          + temp2 * RV(c, kt, i, k, j) / (c->dy[j] * c->dyf[j]);
            TU(t, i, j) = TU(t, i, j) - temp2 * RV(c, kt, i, k, j + 1) / (c->dy[j + 1] * c->dyf[j]);
          }
      }
      bc_horizontal(c, t, p->th_bc_ymin, p->th_bc_ymin_c1, p->th_bc_ymax, p->th_bc_ymax_c1);
      orc_thomas_real(t.l, t.d, t.u, t.v, Nyp, Nx);
      for (int j = jst - 1; j <= jet + 1; ++j)
        for (int i = 0; i < Nx; ++i) RV(c, th, i, k, j) = TVv(t, i, j);
      /* U2 :1072-1121 */
      for (int j = 0; j < NR; ++j) set_row(t, j, 0., 1., 0., 0.);
      for (int j = 2; j <= Nyp; ++j)
        for (int i = 0; i < Nx; ++i) {
          TL(t, i, j) = -tv / (c->dyf[j - 1] * c->dy[j]);
          TD(t, i, j) = 1. + tv / (c->dyf[j] * c->dy[j]) + tv / (c->dyf[j - 1] * c->dy[j]);
          TU(t, i, j) = -tv / (c->dyf[j] * c->dy[j]);
          TVv(t, i, j) = RV(c, r2, i, k, j);
        }
      if (p->use_les) { /* :1092-1105 */
        double* nt = c->arr[DB_NU_T];
        for (int j = 2; j <= Nyp; ++j)
          for (int i = 0; i < Nx; ++i) {
            TL(t, i, j) = TL(t, i, j) - temp2 * 0.5 * (RV(c, nt, i, k, j) + RV(c, nt, i, k, j - 1)) / (c->dyf[j - 1] * c->dy[j]);
            TD(t, i, j) = TD(t, i, j) + temp2 * 0.5 * (RV(c, nt, i, k, j) + RV(c, nt, i, k, j + 1)) / (c->dyf[j] * c->dy[j])
                          + temp2 * 0.5 * (RV(c, nt, i, k, j) + RV(c, nt, i, k, j - 1)) / (c->dyf[j - 1] * c->dy[j]);
            TU(t, i, j) = TU(t, i, j) - temp2 * 0.5 * (RV(c, nt, i, k, j) + RV(c, nt, i, k, j + 1)) / (c->dyf[j] * c->dy[j]);
          }
      }
      bc_u2(c, t);
      orc_thomas_real(t.l, t.d, t.u, t.v, Nyp, Nx);
      for (int j = 1; j <= Nyp + 1; ++j)
        for (int i = 0; i < Nx; ++i) RV(c, u2, i, k, j) = TVv(t, i, j);
      /* U1 :1127-1178 */
      for (int j = 0; j < NR; ++j) set_row(t, j, 0., 1., 0., 0.);
      for (int j = js; j <= je; ++j)
        for (int i = 0; i < Nx; ++i) {
          TL(t, i, j) = -tv / (c->dy[j] * c->dyf[j]);
          TD(t, i, j) = 1. - tv * (-1. / (c->dy[j + 1] * c->dyf[j]) - 1. / (c->dy[j] * c->dyf[j]));
          TU(t, i, j) = -tv / (c->dy[j + 1] * c->dyf[j]);
          TVv(t, i, j) = RV(c, r1, i, k, j);
        }
      if (p->use_les) { /* :1148-1161, 1204-1217 */
        double* nt = c->arr[DB_NU_T];
        for (int j = js; j <= je; ++j)
          for (int i = 0; i < Nx; ++i) {
            TL(t, i, j) = TL(t, i, j) - temp2 * RV(c, nt, i, k, j) / (c->dy[j] * c->dyf[j]);
            TD(t, i, j) = TD(t, i, j) + temp2 * RV(c, nt, i, k, j + 1) / (c->dy[j + 1] * c->dyf[j])
                          + temp2 * RV(c, nt, i, k, j) / (c->dy[j] * c->dyf[j]);
            TU(t, i, j) = TU(t, i, j) - temp2 * RV(c, nt, i, k, j + 1) / (c->dy[j + 1] * c->dyf[j]);
          }
      }
      bc_horizontal(c, t, p->u_bc_ymin, p->u_bc_ymin_c1, p->u_bc_ymax, p->u_bc_ymax_c1);
      orc_thomas_real(t.l, t.d, t.u, t.v, Nyp, Nx);
      for (int j = js - 1; j <= je + 1; ++j)
        for (int i = 0; i < Nx; ++i) RV(c, u1, i, k, j) = TVv(t, i, j);
      /* U3 :1181-1233 */
      for (int j = 0; j < NR; ++j) set_row(t, j, 0., 1., 0., 0.);
      for (int j = js; j <= je; ++j)
        for (int i = 0; i < Nx; ++i) {
          TL(t, i, j) = -tv / (c->dy[j] * c->dyf[j]);
          TD(t, i, j) = 1. - tv * (-1. / (c->dy[j + 1] * c->dyf[j]) - 1. / (c->dy[j] * c->dyf[j]));
          TU(t, i, j) = -tv / (c->dy[j + 1] * c->dyf[j]);
          TVv(t, i, j) = RV(c, r3, i, k, j);
        }
      if (p->use_les) { /* :1148-1161, 1204-1217 */
        double* nt = c->arr[DB_NU_T];
        for (int j = js; j <= je; ++j)
          for (int i = 0; i < Nx; ++i) {
            TL(t, i, j) = TL(t, i, j) - temp2 * RV(c, nt, i, k, j) / (c->dy[j] * c->dyf[j]);
            TD(t, i, j) = TD(t, i, j) + temp2 * RV(c, nt, i, k, j + 1) / (c->dy[j + 1] * c->dyf[j])
                          + temp2 * RV(c, nt, i, k, j) / (c->dy[j] * c->dyf[j]);
            TU(t, i, j) = TU(t, i, j) - temp2 * RV(c, nt, i, k, j + 1) / (c->dy[j + 1] * c->dyf[j]);
          }
      }
      {
        double wmax = c->w_bc_ymax_c1;
        if (p->w_bc_ymax == 1) {
          if (p->f_type == 4)
            c->w_bc_ymax_c1_transient = c->w_bc_ymax_c1 + p->amp_omega0 *
                sin(p->omega0 * (c->Ro_inv / p->delta * c->time - p->force_start));
          wmax = c->w_bc_ymax_c1_transient;
        }
        bc_horizontal(c, t, p->w_bc_ymin, c->w_bc_ymin_c1, p->w_bc_ymax, wmax);
      }
      orc_thomas_real(t.l, t.d, t.u, t.v, Nyp, Nx);
      for (int j = js - 1; j <= je + 1; ++j)
        for (int i = 0; i < Nx; ++i) RV(c, u3, i, k, j) = TVv(t, i, j);
    }
    free(t.l); free(t.d); free(t.u); free(t.v);
  }

  /* :1241-1244 */
  if (p->variable_dt && rk_step == 3 && (c->time_step % p->update_dt) == 0) orc_courant_physical(c);
  /* :1247-1252 */
  orc_fft_xz_to_fourier(c, u1);
  orc_fft_xz_to_fourier(c, u2);
  orc_fft_xz_to_fourier(c, u3);
  orc_fft_xz_to_fourier(c, th);
  /* :1257 */
  orc_rem_div_chan(c);
  /* :1261-1267 */
  LOOP_SPEC(js, je) CV(c, cp, i, k, j) = CV(c, cp, i, k, j) + CV(c, cr1, i, k, j) / temp4;
  return 0;
}

int orc_step(orc_ctx* c) {
  c->time_step += 1; /* for/diablo.f90:59 */
  for (int rk = 1; rk <= 3; ++rk)
    if (orc_rk_chan_1(c, rk)) return -1;
  c->time += c->delta_t; /* for/diablo.f90:68 (dt possibly updated by courant) */
  return 0;
}
