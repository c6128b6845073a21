// db_api.cu -- C-ABI of include/diablo_b200.h: context, state transfer
// between the reference layout and the device layout, and the substep
// orchestration (one CUDA graph per RK step).
#include <cuda_runtime.h>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "../../include/diablo_b200.h"
#include "db_kernels.cuh"
#include "les_feat.cuh"
#include "mlp.cuh"

using namespace db;

struct db_ctx {
  db_params p;
  db_sgs_net* sgs = nullptr;     // learned closure (les_model_type 6)
  Geom g;
  Phys ph;
  State s;
  cudaStream_t st = nullptr;
  // side stream of the substep: the tridiagonal rows are factored there
  // while the transforms and products run (a branch of the captured graph)
  cudaStream_t st_side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool own_stream = false;
  int device = 0;
  std::vector<void*> allocs;
  double* stats = nullptr;        // db_stats rows (device), allocated on first use
  // db_budget / db_bpe scratch (device, first use): FP64 physical u1, u2,
  // u3, th, one FP64 x-half field, the z-means, the rows, the PDF
  double* bud_phys[4] = {nullptr, nullptr, nullptr, nullptr};
  double2* bud_xh = nullptr;
  double* bud_mxy = nullptr;
  double* bud_out = nullptr;
  double* bud_pdf = nullptr;
  int bud_nbin = 0;
  double* zs_field = nullptr;    // a caller's physical field for db_bin_ystar
  double* d_tab = nullptr;       // gy, gyf, dy, dyf, kx, kz tables
  double2* d_tw = nullptr;       // twiddles (Nx then Nz)
  float2* d_twf = nullptr;       // the same in FP32
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // [LES model active]
  int time_step = 0;             // host mirror of time_step (for/diablo.f90:59)
  std::string err;
  double* h_stage = nullptr;     // pinned staging, one physical field
  double2* d_ref = nullptr;       // one spectral field in the reference layout (device)
  size_t stage_doubles = 0;
  std::vector<double> gy, gyf, dy, dyf, kx, kz;
  double pi_ref = 0.0;
  double w_min_c1 = 0.0, w_max_c1 = 0.0;
  // stage timing: events between the kernels of each substep
  bool timing = false;
  cudaEvent_t ev[3][DB_NSTAGES + 1] = {};
  long long launches = 0;          // kernels issued so far
  long long graph_kernels[2] = {0, 0};   // kernel nodes in one captured step
  // nu_t / kappa_t may be non-zero: the LES model has run or they were
  // uploaded.  Until then (they start at zero, for/flow.f90:49-50) a substep
  // without the model has no eddy terms and takes the spectral CN solve.
  bool eddy_live = false;
  bool graph_eddy[2] = {false, false};   // eddy_live when each step graph was captured
};

static void drop_graphs(db_ctx* c);

static std::string g_init_err;

static void set_err(db_ctx* c, const char* a, const char* b) noexcept {
  if (!c) return;
  try {
    c->err = b ? std::string(a) + ": " + b : std::string(a);
  } catch (...) {
  }
}

static void mark(db_ctx* c, int rk, int stage) {
  if (c->timing) cudaEventRecordWithFlags(c->ev[rk][stage], c->st, cudaEventRecordExternal);
}

// error text of a context; recording it never throws (nothing may throw
// past the C-ABI)
static void set_err(db_ctx* c, const char* a, const char* b = nullptr) noexcept;

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_err(c, #call, cudaGetErrorString(e_));                                         \
      return DB_ERR_CUDA;                                                                \
    }                                                                                    \
  } while (0)

static int fail(db_ctx* c, int code, const char* msg) {
  set_err(c, msg);
  return code;
}

// an entry point whose body allocates host memory: an allocation failure
// becomes an error code
template <typename F>
static int guarded(F&& body) noexcept {
  try {
    return body();
  } catch (...) {
    return DB_ERR_CUDA;
  }
}

static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

extern "C" int db_abi_version(void) { return DB_ABI_VERSION; }

extern "C" const char* db_last_error(const db_ctx* c) {
  if (!c) return g_init_err.c_str();
  return c->err.c_str();
}

// ---------------------------------------------------------------------------
// init

static int validate(const db_params* p, std::string& why) {
  if (!pow2(p->nx) || p->nx < 16 || p->nx > 1024) { why = "nx must be a power of two in [16, 1024]"; return DB_ERR_SIZE; }
  if (!pow2(p->nz) || p->nz < 16 || p->nz > 1024) { why = "nz must be a power of two in [16, 1024]"; return DB_ERR_SIZE; }
  if (p->ny < 4) { why = "ny must be >= 4"; return DB_ERR_SIZE; }
  if (p->n_th != 1) { why = "n_th must be 1 (one scalar)"; return DB_ERR_UNSUPPORTED; }
  if (p->time_ad_meth != 1) { why = "time_ad_meth 2 (rk_chan_2) stops in the reference (solver.f90:1289-1293)"; return DB_ERR_UNSUPPORTED; }
  if (p->use_les && p->les_model_type != 5 && p->les_model_type != 6) {
    why = "LES: les_model_type 5 (AMD) and 6 (learned closure) are built";
    return DB_ERR_UNSUPPORTED;
  }
  if (p->precision != 0 && p->precision != 1) {
    why = "precision must be 0 (FP64) or 1 (mixed: FP32 transforms, products and SGS)";
    return DB_ERR_ARG;
  }
  const int b[8] = {p->u_bc_ymin, p->v_bc_ymin, p->w_bc_ymin, p->th_bc_ymin,
                    p->u_bc_ymax, p->v_bc_ymax, p->w_bc_ymax, p->th_bc_ymax};
  for (int i = 0; i < 8; ++i)
    if (b[i] != 0 && b[i] != 1) { why = "boundary types must be 0 (Dirichlet) or 1 (Neumann)"; return DB_ERR_ARG; }
  if (p->variable_dt && p->update_dt < 1) { why = "update_dt must be >= 1"; return DB_ERR_ARG; }
  if (p->re <= 0 || p->pr <= 0 || p->lx <= 0 || p->lz <= 0) { why = "re, pr, lx, lz must be positive"; return DB_ERR_ARG; }
  return DB_OK;
}

static void twiddles(int n, std::vector<double2>& out) {
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; ++k) {
    long double a = 2.0L * PI * (long double)k / (long double)n;
    out.push_back(make_double2((double)cosl(a), -(double)sinl(a)));
  }
}

static void twiddles_f(int n, std::vector<float2>& out) {
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; ++k) {
    long double a = 2.0L * PI * (long double)k / (long double)n;
    out.push_back(make_float2((float)cosl(a), -(float)sinl(a)));
  }
}

// bytes of one physical / x-half element at the context's precision
static size_t phys_elem(const db_ctx* c) { return c->p.precision ? sizeof(float) : sizeof(double); }
static size_t xh_elem(const db_ctx* c) { return c->p.precision ? sizeof(float2) : sizeof(double2); }

static int balloc(db_ctx* c, void** ptr, size_t bytes) {
  void* q = nullptr;
  CK(cudaMalloc(&q, bytes));
  CK(cudaMemset(q, 0, bytes));
  c->allocs.push_back(q);
  *ptr = q;
  return DB_OK;
}

template <typename T>
static int dalloc(db_ctx* c, T** ptr, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, count * sizeof(T)));
  CK(cudaMemset(q, 0, count * sizeof(T)));
  c->allocs.push_back(q);
  *ptr = (T*)q;
  return DB_OK;
}

static int init_impl(const db_params* p, const double* gy_in, void* stream, db_ctx** out) {
  if (!p || !gy_in || !out) { g_init_err = "db_init: NULL argument"; return DB_ERR_ARG; }
  *out = nullptr;
  std::string why;
  int v = validate(p, why);
  if (v) { g_init_err = "db_init: " + why; return v; }
  db_ctx* c = new db_ctx();
  c->p = *p;
  cudaGetDevice(&c->device);
  if (stream) c->st = (cudaStream_t)stream;
  else {
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
      g_init_err = "db_init: no CUDA device";
      delete c;
      return DB_ERR_CUDA;
    }
    c->own_stream = true;
  }
  if (cudaStreamCreateWithFlags(&c->st_side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    g_init_err = "db_init: no CUDA device";
    db_finalize(c);
    return DB_ERR_CUDA;
  }
  const int Nx = p->nx, Nyp = p->ny, Nz = p->nz, np = Nyp + 2;
  Geom& g = c->g;
  g.nx = Nx; g.ny = Nyp; g.nz = Nz; g.np = np;
  g.nkx = Nx / 3; g.nkz = Nz / 3; g.nkzp = 2 * g.nkz + 1;
  g.kxs = round_up(g.nkx + 1, KT);
  g.sp = (long long)g.nkzp * g.kxs;
  g.hp = (long long)Nz * g.kxs;
  g.pp = (long long)Nz * Nx;
  // init_chan_mpi, for/domain.f90:321-340 with one rank in y: rankY == 0
  // takes the first branch, so jstart follows the lower BC and jend =
  // jend_th = Nyp whatever the upper BC (the upper branch, 341-361, runs
  // only on the top rank of several)
  g.jstart = (p->u_bc_ymin == 1) ? 1 : 2;
  g.jend = Nyp;
  g.jstart_th = (p->th_bc_ymin == 1) ? 1 : 2;
  g.jend_th = Nyp;
  g.prec = p->precision;

  // grid metrics, for/domain.f90:276-300, 538-565
  c->gy.assign(np, 0.0); c->gyf.assign(np, 0.0); c->dy.assign(np, 0.0); c->dyf.assign(np, 0.0);
  for (int j = 1; j <= Nyp + 1; ++j) c->gy[j] = gy_in[j - 1];
  for (int j = 1; j <= Nyp; ++j) c->gyf[j] = 0.5 * (c->gy[j] + c->gy[j + 1]);
  c->gyf[0] = 2.0 * c->gyf[1] - c->gyf[2];
  c->gyf[Nyp + 1] = 2.0 * c->gyf[Nyp] - c->gyf[Nyp - 1];
  for (int j = 1; j <= Nyp + 1; ++j) c->dy[j] = c->gyf[j] - c->gyf[j - 1];
  for (int j = 1; j <= Nyp; ++j) c->dyf[j] = c->gy[j + 1] - c->gy[j];
  c->dyf[0] = c->dyf[1];
  c->dyf[Nyp + 1] = c->dyf[Nyp];
  // wavenumbers with the reference's single-precision pi (for/fft.f90:147, 208-225)
  c->pi_ref = (double)(4.0f * atanf(1.0f));
  c->kx.assign(g.kxs, 0.0);
  c->kz.assign(g.nkzp, 0.0);
  for (int i = 0; i <= g.nkx; ++i) c->kx[i] = i * (2. * c->pi_ref) / p->lx;
  for (int k = 0; k <= g.nkz; ++k) c->kz[k] = k * (2. * c->pi_ref) / p->lz;
  for (int k = 1; k <= g.nkz; ++k) c->kz[2 * g.nkz + 1 - k] = -k * (2. * c->pi_ref) / p->lz;

  // physics constants, thermal-wind compensation (for/parameters.f90:255-279)
  Phys& ph = c->ph;
  memset(&ph, 0, sizeof(ph));
  ph.nu = 1.0 / p->re; ph.beta = p->beta; ph.nu_v_scale = p->nu_v_scale; ph.pr = p->pr;
  ph.ro_inv = 1.0 / p->ro; ph.delta = p->delta;
  ph.grav_x = p->grav_x; ph.grav_y = p->grav_y; ph.grav_z = p->grav_z;
  ph.ly = p->ly;
  ph.lx = p->lx;
  ph.front = p->flavor_front ? 1 : 0;
  ph.front_tw = (p->flavor_front && ph.ro_inv != 0.0) ? 1 : 0;
  ph.f_type = p->f_type; ph.px0 = p->px0; ph.omega0 = p->omega0;
  ph.amp_omega0 = p->amp_omega0; ph.force_start = p->force_start; ph.ic_type = p->ic_type;
  double wmin = p->w_bc_ymin_c1, wmax = p->w_bc_ymax_c1;
  ph.dthdx = 0.0; ph.dthdz = 0.0;
  if (p->ic_type == 4 || p->ic_type == 5) {
    double m2 = isnan(p->dthdx_override) ? ph.ro_inv / p->delta : p->dthdx_override;
    double shear = m2 * p->delta / ph.ro_inv;
    if (p->w_bc_ymin == 1) wmin -= shear;
    if (p->w_bc_ymax == 1) wmax -= shear;
    ph.dthdx = m2;
  } else if (p->ic_type >= 6 && p->ic_type <= 8) {
    if (p->w_bc_ymin == 1) wmin -= 2.0 * p->delta / p->lx;
    if (p->w_bc_ymax == 1) wmax -= 2.0 * p->delta / p->lx;
    ph.dthdx = isnan(p->dthdx_override) ? 2.0 / p->lx * ph.ro_inv : p->dthdx_override;
  }
  c->w_min_c1 = wmin; c->w_max_c1 = wmax;
  const int bt[8] = {p->u_bc_ymin, p->v_bc_ymin, p->w_bc_ymin, p->th_bc_ymin,
                     p->u_bc_ymax, p->v_bc_ymax, p->w_bc_ymax, p->th_bc_ymax};
  const double bv[8] = {p->u_bc_ymin_c1, p->v_bc_ymin_c1, wmin, p->th_bc_ymin_c1,
                        p->u_bc_ymax_c1, p->v_bc_ymax_c1, wmax, p->th_bc_ymax_c1};
  for (int i = 0; i < 8; ++i) { ph.bc_type[i] = bt[i]; ph.bc_c1[i] = bv[i]; }
  ph.dx = p->lx / Nx; ph.dz = p->lz / Nz;
  ph.pi_ref = c->pi_ref;

  // device memory
  int rc;
  size_t S = (size_t)np * g.sp, H = (size_t)np * g.hp, Pn = (size_t)np * g.pp;
  double2* sp[11];
  for (int i = 0; i < 11; ++i)
    if ((rc = dalloc(c, &sp[i], S))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
  State& s = c->s;
  s.cu1 = sp[0]; s.cu2 = sp[1]; s.cu3 = sp[2]; s.cp = sp[3]; s.cth = sp[4];
  s.cf1 = sp[5]; s.cf2 = sp[6]; s.cf3 = sp[7]; s.cfth = sp[8];
  s.phi_g = sp[9]; s.pfac = sp[10];
  for (int i = 0; i < 4; ++i)   // NL (or Z(N)) and the forward sweep of the spectral CN solve
    if ((rc = dalloc(c, &s.crs[i], S))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
  // FP64: Z(M) of the spectral solve's z-pass (nls[4..7]); the FP64 LES
  // z-pass (three stages) uses all 8, the first 4 shared with the spectral
  // solve, which never runs in the same substep
  if (!p->precision) {
    for (int i = 4; i < 8; ++i)
      if ((rc = dalloc(c, &s.nls[i], S))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
    if (p->use_les)
      for (int i = 0; i < 4; ++i) s.nls[i] = s.crs[i];
  }
  const size_t eP = phys_elem(c), eH = xh_elem(c);
  for (int i = 0; i < 8; ++i)
    if ((rc = balloc(c, (void**)&s.xh[i], H * eH))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
  double* ph_[8];
  for (int i = 0; i < 8; ++i)
    if ((rc = balloc(c, (void**)&ph_[i], Pn * eP))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
  s.u1 = ph_[0]; s.u2 = ph_[1]; s.u3 = ph_[2]; s.th = ph_[3];
  s.r1 = ph_[4]; s.r2 = ph_[5]; s.r3 = ph_[6]; s.rth = ph_[7];
  if (p->use_les) {
    double** lf[21] = {&s.gx[0], &s.gx[1], &s.gx[2], &s.gx[3], &s.gz[0], &s.gz[1], &s.gz[2], &s.gz[3],
                       &s.les[0], &s.les[1], &s.les[2], &s.les[3], &s.les[4], &s.les[5], &s.les[6],
                       &s.les[7], &s.les[8], &s.les[9], &s.les[10], &s.nu_t, &s.kappa_t};
    for (int i = 0; i < 21; ++i)
      if ((rc = balloc(c, (void**)lf[i], Pn * eP))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
    if ((rc = dalloc(c, &s.ghost, 16 * (size_t)g.sp))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
    if ((rc = dalloc(c, &s.umean, 4 * (size_t)np))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
    // the mixed path's FP64 x-pass of the solve's increments writes its
    // x-half field over one physical FP64 field of the solve scratch
    if (p->precision && 2 * g.kxs > Nx) { db_finalize(c); g_init_err = "db_init: Nx too small for the mixed LES path"; return DB_ERR_ARG; }
    if ((rc = dalloc(c, &s.tscr, 8 * Pn))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
    if ((rc = balloc(c, (void**)&s.sgs_feat, Pn * 16 * sizeof(float))) ||
        (rc = balloc(c, (void**)&s.sgs_out, Pn * 2 * sizeof(float)))) {
      db_finalize(c); g_init_err = "db_init: out of device memory"; return rc;
    }
    LesRow* lr = nullptr;
    if ((rc = dalloc(c, &lr, (size_t)np))) { db_finalize(c); g_init_err = "db_init: out of device memory"; return rc; }
    s.lrow = lr;
  }
  if ((rc = dalloc(c, &s.tri, (size_t)4 * np))) { db_finalize(c); g_init_err = c->err; return rc; }
  if ((rc = dalloc(c, &s.sc, 1))) { db_finalize(c); g_init_err = c->err; return rc; }
  g.flags = &s.sc->flags;
  size_t ntab = 4 * (size_t)np + g.kxs + g.nkzp;
  if ((rc = dalloc(c, &c->d_tab, ntab))) { db_finalize(c); g_init_err = c->err; return rc; }
  std::vector<double> tab;
  tab.insert(tab.end(), c->gy.begin(), c->gy.end());
  tab.insert(tab.end(), c->gyf.begin(), c->gyf.end());
  tab.insert(tab.end(), c->dy.begin(), c->dy.end());
  tab.insert(tab.end(), c->dyf.begin(), c->dyf.end());
  tab.insert(tab.end(), c->kx.begin(), c->kx.end());
  tab.insert(tab.end(), c->kz.begin(), c->kz.end());
  std::vector<double2> tw;
  twiddles(Nx, tw);
  twiddles(Nz, tw);
  std::vector<float2> twf;
  twiddles_f(Nx, twf);
  twiddles_f(Nz, twf);
  if ((rc = dalloc(c, &c->d_tw, tw.size()))) { db_finalize(c); g_init_err = c->err; return rc; }
  if ((rc = dalloc(c, &c->d_twf, twf.size()))) { db_finalize(c); g_init_err = c->err; return rc; }
  if (cudaMemcpy(c->d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_twf, twf.data(), twf.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
    db_finalize(c);
    g_init_err = "db_init: table upload failed";
    return DB_ERR_CUDA;
  }
  g.gy = c->d_tab; g.gyf = c->d_tab + np; g.dy = c->d_tab + 2 * np; g.dyf = c->d_tab + 3 * np;
  if (p->use_les) {   // AMD per-row constants (les.f90:756-780, 1213-1222)
    const double dxs = ph.dx * 3.0, dzs = ph.dz * 3.0, C = 0.2887;
    auto dcoef = [&](double h) {
      return -2.0 * C * C * 3.0 / (1.0 / (dxs * dxs) + 1.0 / ((h * 2.0) * (h * 2.0)) + 1.0 / (dzs * dzs));
    };
    std::vector<LesRow> rows(np);
    for (int j = 0; j < np; ++j) {
      LesRow& r = rows[j];
      memset(&r, 0, sizeof(r));
      const double dyj = c->dy[j], dyfj = c->dyf[j];
      r.idy = dyj != 0.0 ? 1.0 / dyj : 0.0;
      r.idyf = dyfj != 0.0 ? 1.0 / dyfj : 0.0;
      r.dgy = dyj != 0.0 ? dcoef(dyj) : 0.0;
      r.dgyf = dcoef(dyfj);
      const double dly = 2.0 * dyj;
      r.ryx = dly / dxs; r.rxy = dly != 0.0 ? dxs / dly : 0.0;
      r.rzy = dly != 0.0 ? dzs / dly : 0.0; r.ryz = dly / dzs;
      r.wa = (j >= 1 && dyj != 0.0) ? c->dyf[j - 1] / (2.0 * dyj) : 0.0;
      r.wb = dyj != 0.0 ? dyfj / (2.0 * dyj) : 0.0;
      r.dys_f = 2.0 * dyfj;
      r.dys_y = dly;
    }
    if (cudaMemcpy((void*)s.lrow, rows.data(), np * sizeof(LesRow), cudaMemcpyHostToDevice) != cudaSuccess) {
      db_finalize(c);
      g_init_err = "db_init: LES table upload failed";
      return DB_ERR_CUDA;
    }
  }
  g.kx = c->d_tab + 4 * np; g.kz = c->d_tab + 4 * np + g.kxs;
  g.twx = c->d_tw; g.twz = c->d_tw + Nx;
  g.twxf = c->d_twf; g.twzf = c->d_twf + Nx;

  // run scalars (for/parameters.f90:176-178)
  DevScalars h{};
  h.delta_t = p->delta_t;
  h.h_bar[0] = p->delta_t * (8.0 / 15.0);
  h.h_bar[1] = p->delta_t * (2.0 / 15.0);
  h.h_bar[2] = p->delta_t * (5.0 / 15.0);
  h.time = 0.0; h.time_step = 0;
  h.save_stats_time = 1e300; h.save_flow_time = 1e300;
  h.w_bc_ymax_c1_transient = wmax;
  union { double d; unsigned long long u; } inf;
  inf.d = INFINITY;
  h.dt_min_bits = inf.u;
  if (cudaMemcpy(s.sc, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) {
    db_finalize(c);
    g_init_err = "db_init: scalar upload failed";
    return DB_ERR_CUDA;
  }
  c->stage_doubles = std::max(Pn, 2 * S);
  if (cudaMallocHost(&c->h_stage, c->stage_doubles * sizeof(double)) != cudaSuccess) {
    db_finalize(c);
    g_init_err = "db_init: pinned staging allocation failed";
    return DB_ERR_CUDA;
  }
  if (launch_pfac(g, s, c->st) != cudaSuccess || cudaStreamSynchronize(c->st) != cudaSuccess) {
    g_init_err = std::string("db_init: ") + cudaGetErrorString(cudaGetLastError());
    db_finalize(c);
    return DB_ERR_CUDA;
  }
  *out = c;
  return DB_OK;
}

extern "C" int db_init(const db_params* p, const double* gy_in, void* stream, db_ctx** out) {
  try {
    return init_impl(p, gy_in, stream, out);
  } catch (...) {   // a host allocation failed
    try {
      g_init_err = "db_init: host allocation failed";
    } catch (...) {
    }
    if (out) *out = nullptr;
    return DB_ERR_CUDA;
  }
}

extern "C" int db_finalize(db_ctx* c) {
  if (!c) return DB_ERR_ARG;
  for (int i = 0; i < 2; ++i)
    if (c->graph[i]) cudaGraphExecDestroy(c->graph[i]);
  if (c->st) cudaStreamSynchronize(c->st);
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k <= DB_NSTAGES; ++k)
      if (c->ev[r][k]) cudaEventDestroy(c->ev[r][k]);
  for (void* q : c->allocs) cudaFree(q);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  if (c->st_side) {
    cudaStreamSynchronize(c->st_side);
    cudaStreamDestroy(c->st_side);
  }
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->own_stream && c->st) cudaStreamDestroy(c->st);
  delete c;
  return DB_OK;
}

// ---------------------------------------------------------------------------
// layout conversion (host side, into the pinned staging buffer)

static double2* spec_field(db_ctx* c, int id) {
  State& s = c->s;
  switch (id) {
    case DB_CU1: return s.cu1;
    case DB_CU2: return s.cu2;
    case DB_CU3: return s.cu3;
    case DB_CP: return s.cp;
    case DB_CTH: return s.cth;
    case DB_CF1: return s.cf1;
    case DB_CF2: return s.cf2;
    case DB_CF3: return s.cf3;
    case DB_CFTH: return s.cfth;
    default: return nullptr;
  }
}

// reference complex (0:Nxp, 0:Nz+1, 0:Nyp+1) -> compact [j][kzp][kx]
static void ref_to_compact(const db_ctx* c, const double* ref, double2* dst) {
  const Geom& g = c->g;
  const int nxp1 = c->p.nx / 2 + 1, nz2 = c->p.nz + 2;
  for (int j = 0; j < g.np; ++j)
    for (int k = 0; k < g.nkzp; ++k) {
      const double* row = ref + 2 * ((long long)(j * nz2 + k) * nxp1);
      double2* d = dst + (long long)j * g.sp + (long long)k * g.kxs;
      for (int i = 0; i <= g.nkx; ++i) d[i] = make_double2(row[2 * i], row[2 * i + 1]);
      for (int i = g.nkx + 1; i < g.kxs; ++i) d[i] = make_double2(0.0, 0.0);
    }
}

static void compact_to_ref(const db_ctx* c, const double2* src, double* ref) {
  const Geom& g = c->g;
  const int nxp1 = c->p.nx / 2 + 1, nz2 = c->p.nz + 2;
  for (int j = 0; j < g.np; ++j)
    for (int k = 0; k < nz2; ++k) {
      double* row = ref + 2 * ((long long)(j * nz2 + k) * nxp1);
      if (k < g.nkzp) {
        const double2* s = src + (long long)j * g.sp + (long long)k * g.kxs;
        for (int i = 0; i <= g.nkx; ++i) { row[2 * i] = s[i].x; row[2 * i + 1] = s[i].y; }
        for (int i = g.nkx + 1; i < nxp1; ++i) { row[2 * i] = 0.0; row[2 * i + 1] = 0.0; }
      } else {
        for (int i = 0; i < 2 * nxp1; ++i) row[i] = 0.0;
      }
    }
}

static void phys_ref_to_compact(const db_ctx* c, const double* ref, double* dst) {
  const Geom& g = c->g;
  const int nx2 = c->p.nx + 2, nz2 = c->p.nz + 2;
  for (int j = 0; j < g.np; ++j)
    for (int k = 0; k < g.nz; ++k)
      memcpy(dst + (long long)j * g.pp + (long long)k * g.nx, ref + (long long)(j * nz2 + k) * nx2,
             sizeof(double) * g.nx);
}

static void compact_to_phys_ref(const db_ctx* c, const double* src, double* ref) {
  const Geom& g = c->g;
  const int nx2 = c->p.nx + 2, nz2 = c->p.nz + 2;
  for (int j = 0; j < g.np; ++j)
    for (int k = 0; k < g.nz; ++k)
      memcpy(ref + (long long)(j * nz2 + k) * nx2, src + (long long)j * g.pp + (long long)k * g.nx,
             sizeof(double) * g.nx);
}

// one physical field between the reference layout on the host and the
// device at the context's precision (FP32 on the mixed path)
static int phys_upload(db_ctx* c, const double* ref, void* dev) {
  const size_t n = (size_t)c->g.np * c->g.pp;
  phys_ref_to_compact(c, ref, c->h_stage);
  if (c->p.precision) {
    float* f = (float*)c->h_stage;
    for (size_t i = 0; i < n; ++i) f[i] = (float)c->h_stage[i];
  }
  CK(cudaMemcpyAsync(dev, c->h_stage, n * phys_elem(c), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

static int phys_download(db_ctx* c, const void* dev, double* ref) {
  const size_t n = (size_t)c->g.np * c->g.pp;
  CK(cudaMemcpyAsync(c->h_stage, dev, n * phys_elem(c), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (c->p.precision) {
    const float* f = (const float*)c->h_stage;
    for (size_t i = n; i-- > 0;) c->h_stage[i] = (double)f[i];
  }
  compact_to_phys_ref(c, c->h_stage, ref);
  return DB_OK;
}

// spectral fields cross PCIe in the reference layout as one DMA of the
// caller's array; the layout change runs on the device (k_layout.cu)
static size_t ref_spec_bytes(const db_ctx* c) {
  return (size_t)(c->p.nx / 2 + 1) * (c->p.nz + 2) * c->g.np * sizeof(double2);
}
static int ensure_ref(db_ctx* c) {
  if (!c->d_ref && balloc(c, (void**)&c->d_ref, ref_spec_bytes(c)))
    return fail(c, DB_ERR_CUDA, "out of device memory for the layout buffer");
  return DB_OK;
}

// The retained block of a reference-layout array (kx <= Nkx of the first
// 2 Nkz + 1 rows of every plane) between d_ref and a host array, as one 3D
// copy on the context's stream.
static cudaError_t copy_retained(const db_ctx* c, double* host, cudaMemcpyKind kind) {
  const size_t nxh = (size_t)(c->p.nx / 2 + 1), rows = (size_t)(c->p.nz + 2), pitch = nxh * sizeof(double2);
  cudaMemcpy3DParms cp = {};
  cudaPitchedPtr h = make_cudaPitchedPtr(host, pitch, nxh, rows);
  cudaPitchedPtr d = make_cudaPitchedPtr(c->d_ref, pitch, nxh, rows);
  cp.srcPtr = kind == cudaMemcpyHostToDevice ? h : d;
  cp.dstPtr = kind == cudaMemcpyHostToDevice ? d : h;
  cp.extent = make_cudaExtent((size_t)(c->g.nkx + 1) * sizeof(double2), (size_t)c->g.nkzp, (size_t)c->g.np);
  cp.kind = kind;
  return cudaMemcpy3DAsync(&cp, c->st);
}

// n complex zeros from p (16-byte aligned): non-temporal stores, so the
// lines are not read before being overwritten (x86-64), else memset
static void zero_c16(double2* p, size_t n) {
#if defined(__x86_64__)
  const __m128i z = _mm_setzero_si128();
  __m128i* q = reinterpret_cast<__m128i*>(p);
  for (size_t i = 0; i < n; ++i) _mm_stream_si128(q + i, z);
#else
  memset(p, 0, n * sizeof(double2));
#endif
}

// Zero everything of a reference-layout host array outside the retained
// block (the reference keeps those entries zero), planes split over host
// threads.
static void zero_ref_padding(const db_ctx* c, double* host) {
  const size_t nxh = (size_t)(c->p.nx / 2 + 1), rows = (size_t)(c->p.nz + 2);
  const size_t keep = (size_t)(c->g.nkx + 1), krows = (size_t)c->g.nkzp, plane = nxh * rows;
  const int np = c->g.np;
  auto work = [=](int j0, int j1) {
    for (int j = j0; j < j1; ++j) {
      double2* pl = reinterpret_cast<double2*>(host) + (size_t)j * plane;
      for (size_t r = 0; r < krows; ++r) zero_c16(pl + r * nxh + keep, nxh - keep);
      zero_c16(pl + krows * nxh, (rows - krows) * nxh);
    }
#if defined(__x86_64__)
    _mm_sfence();   // the streamed zeros are visible before the thread is joined
#endif
  };
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = std::max(1, std::min({(int)(hw ? hw : 1), 16, np}));
  std::thread th[16];
  bool started[16] = {};
  for (int k = 1; k < nt; ++k) {
    const int a = (int)((long long)np * k / nt), b = (int)((long long)np * (k + 1) / nt);
    try {   // a thread that cannot be created: its planes run here (nothing may throw past the C-ABI)
      th[k] = std::thread(work, a, b);
      started[k] = true;
    } catch (...) {
      work(a, b);
    }
  }
  work(0, (int)((long long)np / nt));
  for (int k = 1; k < nt; ++k)
    if (started[k]) th[k].join();
}

static int upload_spec(db_ctx* c, int id, const double* ref) {
  double2* d = spec_field(c, id);
  if (!d) return fail(c, DB_ERR_ARG, "bad spectral field id");
  const size_t n = (size_t)c->g.np * c->g.sp;
  if (!ref) {
    CK(cudaMemsetAsync(d, 0, n * sizeof(double2), c->st));
  } else {
    if (int rc = ensure_ref(c)) return rc;
    // only the retained modes cross PCIe; the rest of the reference array
    // is never read
    CK(copy_retained(c, const_cast<double*>(ref), cudaMemcpyHostToDevice));
    CK(launch_ref_to_spec(c->g, c->p.nx, c->p.nz, c->d_ref, d, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

static int download_spec(db_ctx* c, int id, double* ref) {
  double2* d = spec_field(c, id);
  if (!d) return fail(c, DB_ERR_ARG, "bad spectral field id");
  if (!ref) return DB_OK;
  if (int rc = ensure_ref(c)) return rc;
  // only the retained modes cross PCIe; the host threads write the zero
  // padding while the copy runs (disjoint parts of the array)
  CK(launch_spec_to_ref(c->g, c->p.nx, c->p.nz, d, c->d_ref, c->st));
  CK(copy_retained(c, ref, cudaMemcpyDeviceToHost));
  zero_ref_padding(c, ref);
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

extern "C" int db_upload_state(db_ctx* c, const double* cu1, const double* cu2, const double* cu3,
                               const double* cp, const double* cth, const double* cf1, const double* cf2,
                               const double* cf3, const double* cfth) {
  if (!c) return DB_ERR_ARG;
  const double* a[9] = {cu1, cu2, cu3, cp, cth, cf1, cf2, cf3, cfth};
  for (int i = 0; i < 9; ++i) {
    int rc = upload_spec(c, i, a[i]);
    if (rc) return rc;
  }
  return DB_OK;
}

extern "C" int db_download_state(db_ctx* c, double* cu1, double* cu2, double* cu3, double* cp, double* cth,
                                 double* cf1, double* cf2, double* cf3, double* cfth) {
  if (!c) return DB_ERR_ARG;
  double* a[9] = {cu1, cu2, cu3, cp, cth, cf1, cf2, cf3, cfth};
  for (int i = 0; i < 9; ++i) {
    int rc = download_spec(c, i, a[i]);
    if (rc) return rc;
  }
  return DB_OK;
}

static double* les_field(db_ctx* c, int id) {
  if (!c->p.use_les) return nullptr;
  return id == DB_NU_T ? c->s.nu_t : c->s.kappa_t;
}

extern "C" int db_upload_field(db_ctx* c, int field, const double* host) {
  if (!c || !host) return DB_ERR_ARG;
  if (field >= DB_CU1 && field <= DB_CFTH) return upload_spec(c, field, host);
  if (field == DB_NU_T || field == DB_KAPPA_T) {
    double* d = les_field(c, field);
    if (!d) return fail(c, DB_ERR_STATE, "nu_t / kappa_t exist only with use_les");
    // a substep without the model now has eddy terms: drop the step graph
    // captured with the spectral CN solve
    if (!c->eddy_live) drop_graphs(c);
    c->eddy_live = true;
    return phys_upload(c, host, d);
  }
  return fail(c, DB_ERR_ARG, "bad field id");
}

extern "C" int db_download_field(db_ctx* c, int field, double* host) {
  if (!c || !host) return DB_ERR_ARG;
  if (field >= DB_CU1 && field <= DB_CFTH) return download_spec(c, field, host);
  if (field == DB_NU_T || field == DB_KAPPA_T) {
    double* d = les_field(c, field);
    if (!d) return fail(c, DB_ERR_STATE, "nu_t / kappa_t exist only with use_les");
    // the reference array's padding (x >= Nx, z >= Nz) reads as zero
    const int nx2 = c->p.nx + 2, nz2 = c->p.nz + 2;
    memset(host, 0, sizeof(double) * (size_t)c->g.np * nz2 * nx2);
    return phys_download(c, d, host);
  }
  return fail(c, DB_ERR_ARG, "bad field id");
}

// ---------------------------------------------------------------------------
// clock / status

extern "C" int db_set_clock(db_ctx* c, double time, int32_t time_step, double sst, double sft) {
  if (!c) return DB_ERR_ARG;
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->s.sc, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  h.time = time; h.time_step = time_step; h.save_stats_time = sst; h.save_flow_time = sft;
  CK(cudaMemcpyAsync(c->s.sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->time_step = time_step;
  return DB_OK;
}

extern "C" int db_get_status(db_ctx* c, db_status* out) {
  if (!c || !out) return DB_ERR_ARG;
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->s.sc, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  out->flags = h.flags; out->time_step = h.time_step; out->time = h.time;
  out->delta_t = h.delta_t; out->max_div = h.max_div;
  return DB_OK;
}

extern "C" int db_clear_status(db_ctx* c) {
  if (!c) return DB_ERR_ARG;
  CK(cudaMemsetAsync(&c->s.sc->flags, 0, sizeof(int), c->st));
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

// ---------------------------------------------------------------------------
// transforms of one host array

extern "C" int db_fft_xz_to_fourier(db_ctx* c, double* buf) {
  if (!c || !buf) return DB_ERR_ARG;
  const Geom& g = c->g;
  int rc = phys_upload(c, buf, c->s.r1);
  if (rc) return rc;
  CK(launch_fwd_x(g, fset(c->s.r1), fset(c->s.xh[0]), 1, c->st));
  CK(launch_fwd_z(g, fset(c->s.xh[0]), fset(c->s.phi_g), 1, c->st));
  CK(cudaMemcpyAsync(c->h_stage, c->s.phi_g, (size_t)g.np * g.sp * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  compact_to_ref(c, (double2*)c->h_stage, buf);
  return DB_OK;
}

extern "C" int db_fft_xz_to_physical(db_ctx* c, double* buf) {
  if (!c || !buf) return DB_ERR_ARG;
  const Geom& g = c->g;
  ref_to_compact(c, buf, (double2*)c->h_stage);
  CK(cudaMemcpyAsync(c->s.phi_g, c->h_stage, (size_t)g.np * g.sp * sizeof(double2), cudaMemcpyHostToDevice, c->st));
  CK(launch_inv_z(g, fset(c->s.phi_g), fset(c->s.xh[0]), 1, c->st));
  CK(launch_inv_x(g, fset(c->s.xh[0]), fset(c->s.r1), 1, c->st));
  return phys_download(c, c->s.r1, buf);
}

// device-resident forms: the same transforms on a device array in the
// reference layout, every layout change on the device, stream-ordered on
// the context's stream (no host synchronisation)
extern "C" int db_fft_xz_to_fourier_dev(db_ctx* c, double* d) {
  if (!c || !d) return DB_ERR_ARG;
  const Geom& g = c->g;
  CK(launch_phys_from_ref(g, c->p.nx, c->p.nz, d, c->s.r1, c->st));
  CK(launch_fwd_x(g, fset(c->s.r1), fset(c->s.xh[0]), 1, c->st));
  CK(launch_fwd_z(g, fset(c->s.xh[0]), fset(c->s.phi_g), 1, c->st));
  CK(launch_spec_to_ref(g, c->p.nx, c->p.nz, c->s.phi_g, reinterpret_cast<double2*>(d), c->st));
  c->launches += 4;
  return DB_OK;
}

extern "C" int db_fft_xz_to_physical_dev(db_ctx* c, double* d) {
  if (!c || !d) return DB_ERR_ARG;
  const Geom& g = c->g;
  CK(launch_ref_to_spec(g, c->p.nx, c->p.nz, reinterpret_cast<const double2*>(d), c->s.phi_g, c->st));
  CK(launch_inv_z(g, fset(c->s.phi_g), fset(c->s.xh[0]), 1, c->st));
  CK(launch_inv_x(g, fset(c->s.xh[0]), fset(c->s.r1), 1, c->st));
  CK(launch_phys_to_ref(g, c->p.nx, c->p.nz, c->s.r1, d, c->st));
  c->launches += 4;
  return DB_OK;
}

// ---------------------------------------------------------------------------
// the substep

// the learned closure's feature source: the physical fields and x/z
// derivatives the LES part of the substep has just formed
static LesFeatSrc les_feat_src(const db_ctx* c) {
  const State& s = c->s;
  LesFeatSrc f{};
  f.f[0] = s.u1; f.f[1] = s.u2; f.f[2] = s.u3; f.f[3] = s.th;
  for (int i = 0; i < 4; ++i) {
    f.f[4 + i] = s.gx[i];
    f.f[8 + i] = s.gz[i];
  }
  f.lrow = s.lrow;
  f.pp = c->g.pp;
  f.ny = c->g.ny;
  f.dxs = c->ph.dx * BETA_SGS;
  f.dzs = c->ph.dz * BETA_SGS;
  f.mean = s.pmean;
  return f;
}

// the LES model runs on a substep of driver step time_step (solver.f90:615)
static bool les_active(const db_ctx* c, int time_step) {
  return c->p.use_les && (!c->p.create_new_flow || time_step > 100);
}

// the plane-mean split of the physical fields holds for the kernels of one
// substep only
struct MeanSplit {
  State& s;
  MeanSplit(State& s_, bool on) : s(s_) { s.pmean = on ? s.umean : nullptr; }
  ~MeanSplit() { s.pmean = nullptr; }
};

static cudaError_t substep(db_ctx* c, int rk /* 0-based */, bool les) {
  const Geom& g = c->g;
  State& s = c->s;
  cudaStream_t st = c->st;
  cudaError_t e;
  long long n = 0;
  // mixed path with LES: the physical fields hold fluctuations about their
  // plane means (FP64), which the closure walk, the features and the
  // eddy-viscosity solves add back
  const MeanSplit split(s, les && g.prec != 0);
  if (les) c->eddy_live = true;
  // without eddy terms the CN matrices are the same in every column
  const bool spectral = !c->p.use_les || (!les && !c->eddy_live);
  mark(c, rk, 0);
  // the implicit systems' rows (dt and rk only) on the side stream, joined
  // before the solves
  if ((e = cudaEventRecord(c->ev_fork, st))) return e;
  if ((e = cudaStreamWaitEvent(c->st_side, c->ev_fork, 0))) return e;
  if ((e = launch_tri_coef(g, c->ph, s, rk, c->st_side))) return e;
  if ((e = cudaEventRecord(c->ev_join, c->st_side))) return e;
  if (les) {
    // les_chan / les_chan_th: ghost rows, then the state and its x and z
    // derivatives to physical space (les.f90:63-75, 555-569, 1209-1211)
    if ((e = launch_les_bc(g, c->ph, s, st))) return e;
    if ((e = launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3, s.cth, s.cu1, s.cu2, s.cu3, s.cth),
                          fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[4], s.xh[5], s.xh[6], s.xh[7]), 8, st,
                          0xF0u, s.ghost, s.pmean ? s.umean : nullptr))) return e;
    mark(c, rk, 1);
    FieldSet in = fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[0], s.xh[1], s.xh[2], s.xh[3]);
    FieldSet out = fset(s.u1, s.u2, s.u3, s.th, s.gx[0], s.gx[1], s.gx[2], s.gx[3]);
    for (int i = 0; i < 4; ++i) { in.p[8 + i] = s.xh[4 + i]; out.p[8 + i] = s.gz[i]; }
    if ((e = launch_inv_x(g, in, out, 12, st, 0xF0u))) return e;
    mark(c, rk, 2);
    if (c->p.les_model_type == 6) {   // learned closure (features formed in the inference kernel), AMD outside its range
      if (sgs_forward_les_async(c->sgs, les_feat_src(c), g.prec != 0, s.sgs_out, (long long)g.np * g.pp, st))
        return cudaErrorLaunchFailure;
      if ((e = launch_les_amd(g, c->ph, s, st, 2))) return e;
      n += 1;
    } else {
      if ((e = launch_les_amd(g, c->ph, s, st))) return e;
    }
    n += 2;
  } else {
    // velocity and buoyancy to physical space (solver.f90:635-643)
    if ((e = launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3, s.cth), fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]), 4, st))) return e;
    mark(c, rk, 1);
    if ((e = launch_inv_x(g, fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]), fset(s.u1, s.u2, s.u3, s.th), 4, st))) return e;
    mark(c, rk, 2);
  }
  // nonlinear products (+ SGS forcing) + x-FFT
  if ((e = launch_products(g, s, st, les))) return e;
  mark(c, rk, 3);
  const bool cfl_step = rk == 2 && c->p.variable_dt;
  if (spectral) {
    // without eddy viscosity the CN matrices are the same in every column:
    // z-FFT of the products, then the spectral RHS and the CN solves on the
    // retained modes (FP64), no transforms of cr or u
    if ((e = launch_zpass_spec(g, s, st))) return e;
    mark(c, rk, 4);
    mark(c, rk, 5);
    if ((e = cudaStreamWaitEvent(st, c->ev_join, 0))) return e;
    if ((e = launch_rhs_cn(g, c->ph, s, rk, st))) return e;
    mark(c, rk, 6);
    n += 4;
    // CFL on the last substep from the new velocity before the projection
    // (solver.f90:1241-1244): u1..u3 to physical space for it
    if (cfl_step) {
      CflCtl ctl{c->p.cfl, c->p.time_limit, c->p.variable_dt, c->p.update_dt, 0};
      if ((e = launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3), fset(s.xh[0], s.xh[1], s.xh[2]), 3, st))) return e;
      if ((e = launch_inv_x_cfl(g, c->ph, s, ctl, fset(s.xh[0], s.xh[1], s.xh[2]), st))) return e;
      if ((e = launch_courant_final(c->ph, s, ctl, st))) return e;
      n += 3;
    }
    mark(c, rk, 7);
    mark(c, rk, 8);
  } else {
    // z-FFT + spectral RHS + inverse z of cr
    const double2* ov = les ? s.ghost : nullptr;   // ghost rows the transforms saw
    if ((e = cudaStreamWaitEvent(st, c->ev_join, 0))) return e;
    if ((e = launch_zpass_rhs(g, c->ph, s, rk, st, ov))) return e;
    mark(c, rk, 4);
    // cr1 = xh[0], cr3 = xh[2], cr2 = xh[4], crth = xh[6] -> physical r
    if ((e = launch_inv_x(g, fset(s.xh[0], s.xh[4], s.xh[2], s.xh[6]), fset(s.r1, s.r2, s.r3, s.rth), 4, st))) return e;
    mark(c, rk, 5);
    // implicit CN solves with the eddy terms (solver.f90:1012-1233); the
    // mixed path's solves store the new physical u only where the CFL below
    // reads it
    if ((e = launch_thomas_les(g, s, rk, st, cfl_step))) return e;
    mark(c, rk, 6);
    n += 7;
    // CFL on the last substep (solver.f90:1241-1244)
    if (cfl_step) {
      CflCtl ctl{c->p.cfl, c->p.time_limit, c->p.variable_dt, c->p.update_dt, 0};
      if ((e = launch_courant(g, c->ph, s, ctl, st))) return e;
      n += 2;
    }
    mark(c, rk, 7);
    // back to Fourier space (solver.f90:1247-1252) and projection
    if (c->p.precision != 0) {
      // mixed path: the solve left u's increment in FP64; transform it in
      // FP64 and add it to the state the substep started from (an FP32
      // increment's rounding is not divergence free, and the projection
      // would carry it into cp amplified by 1 / h_bar)
      double* dinc[4];
      double2* dxh[4];
      thomas_les_inc(g, s, dinc, dxh);
      Geom g64 = g;
      g64.prec = 0;
      if ((e = launch_fwd_x(g64, fset(dinc[0], dinc[1], dinc[2], dinc[3]), fset(dxh[0], dxh[1], dxh[2], dxh[3]), 4,
                            st))) return e;
      mark(c, rk, 8);
      if ((e = launch_fwd_z(g64, fset(dxh[0], dxh[1], dxh[2], dxh[3]), fset(s.cu1, s.cu2, s.cu3, s.cth), 4, st, 1,
                            ov))) return e;
    } else {
      if ((e = launch_fwd_x(g, fset(s.u1, s.u2, s.u3, s.th), fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]), 4, st)))
        return e;
      mark(c, rk, 8);
      if ((e = launch_fwd_z(g, fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]), fset(s.cu1, s.cu2, s.cu3, s.cth), 4, st, 0,
                            ov))) return e;
    }
  }
  mark(c, rk, 9);
  if ((e = launch_rem_div(g, s, rk, 1, st))) return e;
  if (rk == 2 && c->p.variable_dt) {
    if ((e = launch_apply_dt(s.sc, st))) return e;
    n += 1;
  }
  mark(c, rk, 10);
  n += 3;
  c->launches += n;
  return cudaSuccess;
}

static int need_net(db_ctx* c);

extern "C" int db_rk_substep(db_ctx* c, int rk_step) {
  if (!c) return DB_ERR_ARG;
  if (need_net(c)) return DB_ERR_STATE;
  if (rk_step < 1 || rk_step > 3) return fail(c, DB_ERR_ARG, "rk_step must be 1, 2 or 3");
  const bool t = c->timing;
  c->timing = false;  // stage events belong to whole steps
  cudaError_t e = substep(c, rk_step - 1, les_active(c, c->time_step));
  c->timing = t;
  CK(e);
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

static cudaError_t one_step(db_ctx* c, bool les) {
  cudaError_t e;
  if ((e = launch_step_begin(c->s.sc, c->st))) return e;
  for (int rk = 0; rk < 3; ++rk)
    if ((e = substep(c, rk, les))) return e;
  c->launches += 2;
  return launch_step_end(c->s.sc, c->st);
}

extern "C" int db_rk_steps(db_ctx* c, int nsteps) {
  if (!c) return DB_ERR_ARG;
  if (nsteps < 0) return fail(c, DB_ERR_ARG, "nsteps must be >= 0");
  if (need_net(c)) return DB_ERR_STATE;
  for (int i = 0; i < nsteps; ++i) {
    // time_step is incremented at the start of the step (diablo.f90:58-61)
    const int m = les_active(c, c->time_step + 1) ? 1 : 0;
    if (c->graph[m] && c->graph_eddy[m] != c->eddy_live) {   // captured for the other CN path
      cudaGraphExecDestroy(c->graph[m]);
      c->graph[m] = nullptr;
    }
    if (!c->graph[m]) {
      cudaGraph_t gr;
      const long long before = c->launches;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
      cudaError_t e = one_step(c, m == 1);
      c->graph_kernels[m] = c->launches - before;
      c->launches = before;
      cudaError_t e2 = cudaStreamEndCapture(c->st, &gr);
      if (e != cudaSuccess || e2 != cudaSuccess) {
        c->err = std::string("graph capture failed: ") + cudaGetErrorString(e != cudaSuccess ? e : e2);
        return DB_ERR_CUDA;
      }
      e = cudaGraphInstantiate(&c->graph[m], gr, 0);
      cudaGraphDestroy(gr);
      c->graph_eddy[m] = c->eddy_live;
      if (e != cudaSuccess) {
        c->graph[m] = nullptr;
        c->err = std::string("graph instantiate failed: ") + cudaGetErrorString(e);
        return DB_ERR_CUDA;
      }
    }
    CK(cudaGraphLaunch(c->graph[m], c->st));
    c->launches += c->graph_kernels[m];
    c->time_step += 1;
  }
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

// ---------------------------------------------------------------------------
// ensembles: one CUDA graph per time step.  Members of equal size without
// LES at a fixed dt are batched: each kernel of the step is launched once
// for all of them (launch_substep_batch, the members' arguments in a device
// table).  Otherwise the graph forks into every member's stream, runs its
// step there and joins back.

struct db_ensemble {
  std::vector<db_ctx*> members;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // [LES model active]
  std::vector<cudaEvent_t> ev;                     // fork event + one join event per member
  long long kernels[2] = {0, 0};
  bool graph_eddy[2] = {false, false};             // eddy terms when each graph was captured
  // batched form
  bool can_batch = false, batched = false;
  MemberArgs* tab = nullptr;                       // device table, one entry per member
  // the members split into groups of consecutive members, each group a
  // chain of batched kernels on its own branch of the graph (one group's
  // kernel boundaries overlap another's work)
  int groups = 1, groups_cap = 0;                  // requested; in bgraph
  static constexpr int kMaxGroups = 8;
  cudaStream_t gst[kMaxGroups] = {}, gside[kMaxGroups] = {};   // group streams, the implicit systems' rows
  cudaEvent_t gfork[kMaxGroups] = {}, gjoin[kMaxGroups] = {}, gdone[kMaxGroups] = {};
  cudaEvent_t ev_start = nullptr;
  cudaGraphExec_t bgraph = nullptr;
  Geom g_cap{};                                    // member 0's geometry when bgraph was captured
  long long bkernels = 0;
  std::string err;
};

// members that one batched launch per kernel can advance: the spectral
// substep (no LES), fixed dt, the same grid, solved planes and precision
static bool batch_eligible(const std::vector<db_ctx*>& m) {
  const db_ctx* a = m[0];
  if (a->g.nx > 512 || (long long)m.size() > 65535 / MAXF) return false;
  for (const db_ctx* c : m) {
    if (c->p.use_les || c->p.variable_dt) return false;
    if (c->g.nx != a->g.nx || c->g.ny != a->g.ny || c->g.nz != a->g.nz || c->g.prec != a->g.prec) return false;
    // the batched kernels take member 0's geometry (the planes each equation solves included)
    if (c->g.jstart != a->g.jstart || c->g.jend != a->g.jend || c->g.jstart_th != a->g.jstart_th ||
        c->g.jend_th != a->g.jend_th)
      return false;
    if (!c->s.crs[0] || (!c->g.prec && !c->s.nls[4])) return false;
  }
  return true;
}

static int ensemble_create_impl(db_ctx** members, int n, void* stream, db_ensemble** out) {
  if (!members || n < 1 || !out) return DB_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return DB_ERR_ARG;
    const db_params& a = members[0]->p;
    const db_params& b = members[i]->p;
    if (a.use_les != b.use_les || a.les_model_type != b.les_model_type || a.create_new_flow != b.create_new_flow ||
        a.precision != b.precision || members[i]->time_step != members[0]->time_step || members[i]->timing) {
      g_init_err = "db_ensemble_create: members must share use_les, les_model_type, create_new_flow, precision, "
                   "time_step, and have stage timing off";
      return DB_ERR_ARG;
    }
    for (int k = 0; k < i; ++k)
      if (members[k] == members[i] || members[k]->st == members[i]->st) {
        g_init_err = "db_ensemble_create: members must be distinct contexts on distinct streams";
        return DB_ERR_ARG;
      }
  }
  db_ensemble* e = new db_ensemble();
  e->members.assign(members, members + n);
  if (stream) e->st = (cudaStream_t)stream;
  else {
    if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
      delete e;
      g_init_err = "db_ensemble_create: stream creation failed";
      return DB_ERR_CUDA;
    }
    e->own_stream = true;
  }
  e->ev.resize(n + 1, nullptr);
  for (auto& v : e->ev)
    if (cudaEventCreateWithFlags(&v, cudaEventDisableTiming) != cudaSuccess) {
      db_ensemble_destroy(e);
      g_init_err = "db_ensemble_create: event creation failed";
      return DB_ERR_CUDA;
    }
  if (batch_eligible(e->members)) {
    const bool ok = cudaMalloc((void**)&e->tab, (size_t)n * sizeof(MemberArgs)) == cudaSuccess &&
                    cudaEventCreateWithFlags(&e->ev_start, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      db_ensemble_destroy(e);
      g_init_err = "db_ensemble_create: out of device memory";
      return DB_ERR_CUDA;
    }
    e->can_batch = e->batched = true;
    // one group: for 64 members of 128x65x128 four groups ran 31.5 ms per
    // step against 30.8 ms for one (the GPU is full either way)
    e->groups = 1;
  }
  *out = e;
  return DB_OK;
}

extern "C" int db_ensemble_create(db_ctx** members, int n, void* stream, db_ensemble** out) {
  return guarded([&] { return ensemble_create_impl(members, n, stream, out); });
}

extern "C" int db_ensemble_destroy(db_ensemble* e) {
  if (!e) return DB_ERR_ARG;
  if (e->st) cudaStreamSynchronize(e->st);
  for (int i = 0; i < 2; ++i)
    if (e->graph[i]) cudaGraphExecDestroy(e->graph[i]);
  if (e->bgraph) cudaGraphExecDestroy(e->bgraph);
  for (auto v : e->ev)
    if (v) cudaEventDestroy(v);
  for (int k = 0; k < db_ensemble::kMaxGroups; ++k) {
    for (cudaStream_t q : {e->gst[k], e->gside[k]})
      if (q) {
        cudaStreamSynchronize(q);
        cudaStreamDestroy(q);
      }
    for (cudaEvent_t v : {e->gfork[k], e->gjoin[k], e->gdone[k]})
      if (v) cudaEventDestroy(v);
  }
  if (e->ev_start) cudaEventDestroy(e->ev_start);
  if (e->tab) cudaFree(e->tab);
  if (e->own_stream && e->st) cudaStreamDestroy(e->st);
  delete e;
  return DB_OK;
}

extern "C" const char* db_ensemble_error(const db_ensemble* e) { return e ? e->err.c_str() : g_init_err.c_str(); }

extern "C" int db_ensemble_set_batched(db_ensemble* e, int groups) {
  if (!e || groups < 0 || (groups && !e->can_batch)) return DB_ERR_ARG;
  e->batched = groups != 0;
  if (groups) e->groups = std::min(std::min(groups, db_ensemble::kMaxGroups), (int)e->members.size());
  return DB_OK;
}

extern "C" int db_ensemble_info(const db_ensemble* e, int* groups, long long* kernels_per_step) {
  if (!e) return DB_ERR_ARG;
  if (groups) *groups = e->batched ? e->groups : 0;
  if (kernels_per_step) *kernels_per_step = e->batched ? e->bkernels : e->kernels[0];
  return DB_OK;
}

// the launch shapes of a captured batched graph follow member 0's tuning
static bool same_shapes(const Geom& a, const Geom& b) {
  return a.tune_xcps == b.tune_xcps && a.tune_xgrid == b.tune_xgrid && a.tune_zns == b.tune_zns &&
         a.tune_pgrid == b.tune_pgrid;
}

// the streams and events of groups 0..G-1, created on first use
static bool ensure_groups(db_ensemble* e, int G) {
  for (int k = 0; k < G; ++k) {
    for (cudaStream_t* q : {&e->gst[k], &e->gside[k]})
      if (!*q && cudaStreamCreateWithFlags(q, cudaStreamNonBlocking) != cudaSuccess) {
        *q = nullptr;
        return false;
      }
    for (cudaEvent_t* v : {&e->gfork[k], &e->gjoin[k], &e->gdone[k]})
      if (!*v && cudaEventCreateWithFlags(v, cudaEventDisableTiming) != cudaSuccess) {
        *v = nullptr;
        return false;
      }
  }
  return true;
}

static int ensemble_steps_batched(db_ensemble* e, int nsteps) {
  const int n = (int)e->members.size();
  db_ctx* c0 = e->members[0];
  if (!ensure_groups(e, e->groups)) {
    e->err = "ensemble stream creation failed";
    return DB_ERR_CUDA;
  }
  // the step stream follows whatever the members' own streams hold
  for (int i = 0; i < n; ++i) {
    if (cudaEventRecord(e->ev[1 + i], e->members[i]->st) != cudaSuccess ||
        cudaStreamWaitEvent(e->st, e->ev[1 + i], 0) != cudaSuccess) {
      e->err = "ensemble stream join failed";
      return DB_ERR_CUDA;
    }
  }
  if (e->bgraph && (!same_shapes(e->g_cap, c0->g) || e->groups_cap != e->groups)) {
    cudaGraphExecDestroy(e->bgraph);
    e->bgraph = nullptr;
  }
  if (!e->bgraph) {
    std::vector<MemberArgs> h(n);
    for (int i = 0; i < n; ++i) h[i] = member_args(e->members[i]->g, e->members[i]->ph, e->members[i]->s);
    if (cudaMemcpyAsync(e->tab, h.data(), (size_t)n * sizeof(MemberArgs), cudaMemcpyHostToDevice, e->st) !=
            cudaSuccess ||
        cudaStreamSynchronize(e->st) != cudaSuccess) {
      e->err = "ensemble member table upload failed";
      return DB_ERR_CUDA;
    }
    cudaGraph_t gr;
    if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
      e->err = "ensemble capture could not start";
      return DB_ERR_CUDA;
    }
    const int G = e->groups;
    cudaError_t er = cudaEventRecord(e->ev_start, e->st);
    for (int k = 0; k < G && er == cudaSuccess; ++k) {
      // group k: members [n k / G, n (k + 1) / G)
      const int m0 = (int)((long long)n * k / G), m1 = (int)((long long)n * (k + 1) / G);
      const Batch b{e->tab + m0, m1 - m0, 0, 0, 0};
      cudaStream_t q = e->gst[k];
      er = cudaStreamWaitEvent(q, e->ev_start, 0);
      if (er == cudaSuccess) er = launch_steps_batch(b, 0, q);
      for (int rk = 0; rk < 3 && er == cudaSuccess; ++rk)
        er = launch_substep_batch(c0->g, b, rk, q, e->gside[k], e->gfork[k], e->gjoin[k]);
      if (er == cudaSuccess) er = launch_steps_batch(b, 1, q);
      if (er == cudaSuccess) er = cudaEventRecord(e->gdone[k], q);
      if (er == cudaSuccess) er = cudaStreamWaitEvent(e->st, e->gdone[k], 0);
    }
    cudaError_t er2 = cudaStreamEndCapture(e->st, &gr);
    if (er != cudaSuccess || er2 != cudaSuccess) {
      e->err = std::string("ensemble capture failed: ") + cudaGetErrorString(er != cudaSuccess ? er : er2);
      return DB_ERR_CUDA;
    }
    er = cudaGraphInstantiate(&e->bgraph, gr, 0);
    cudaGraphDestroy(gr);
    if (er != cudaSuccess) {
      e->bgraph = nullptr;
      e->err = std::string("ensemble graph instantiate failed: ") + cudaGetErrorString(er);
      return DB_ERR_CUDA;
    }
    e->g_cap = c0->g;
    e->groups_cap = G;
    // step scalars twice; per substep tri_coef, the two inverse passes,
    // products, the z-pass, rhs_cn, cn_back and rem_div
    e->bkernels = (long long)G * (2 + 3 * 8);
  }
  for (int it = 0; it < nsteps; ++it) {
    if (cudaGraphLaunch(e->bgraph, e->st) != cudaSuccess) {
      e->err = "ensemble graph launch failed";
      return DB_ERR_CUDA;
    }
    for (db_ctx* c : e->members) c->time_step += 1;
  }
  if (cudaStreamSynchronize(e->st) != cudaSuccess) {
    e->err = std::string("ensemble step failed: ") + cudaGetErrorString(cudaGetLastError());
    return DB_ERR_CUDA;
  }
  return DB_OK;
}

extern "C" int db_ensemble_steps(db_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return DB_ERR_ARG;
  if (e->batched) return ensemble_steps_batched(e, nsteps);
  db_ctx* c0 = e->members[0];
  for (db_ctx* c : e->members)
    if (need_net(c)) { e->err = c->err; return DB_ERR_STATE; }
  const int n = (int)e->members.size();
  for (int it = 0; it < nsteps; ++it) {
    const int m = les_active(c0, c0->time_step + 1) ? 1 : 0;
    bool eddy = false;   // some member's substeps carry eddy terms
    for (db_ctx* c : e->members) eddy = eddy || c->eddy_live;
    if (e->graph[m] && e->graph_eddy[m] != eddy) {   // captured for the other CN path
      cudaGraphExecDestroy(e->graph[m]);
      e->graph[m] = nullptr;
    }
    if (!e->graph[m]) {
      cudaGraph_t gr;
      if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        e->err = "ensemble capture could not start";
        return DB_ERR_CUDA;
      }
      cudaError_t er = cudaEventRecord(e->ev[0], e->st);
      long long k0 = 0;
      for (int i = 0; i < n && er == cudaSuccess; ++i) {
        db_ctx* c = e->members[i];
        er = cudaStreamWaitEvent(c->st, e->ev[0], 0);   // fork: the member's stream joins the capture
        const long long before = c->launches;
        if (er == cudaSuccess) er = one_step(c, m == 1);
        k0 += c->launches - before;
        c->launches = before;
        if (er == cudaSuccess) er = cudaEventRecord(e->ev[1 + i], c->st);
        if (er == cudaSuccess) er = cudaStreamWaitEvent(e->st, e->ev[1 + i], 0);   // join
      }
      cudaError_t er2 = cudaStreamEndCapture(e->st, &gr);
      if (er != cudaSuccess || er2 != cudaSuccess) {
        e->err = std::string("ensemble capture failed: ") + cudaGetErrorString(er != cudaSuccess ? er : er2);
        return DB_ERR_CUDA;
      }
      er = cudaGraphInstantiate(&e->graph[m], gr, 0);
      cudaGraphDestroy(gr);
      if (er != cudaSuccess) {
        e->graph[m] = nullptr;
        e->err = std::string("ensemble graph instantiate failed: ") + cudaGetErrorString(er);
        return DB_ERR_CUDA;
      }
      e->kernels[m] = k0;
      eddy = false;
      for (db_ctx* c : e->members) eddy = eddy || c->eddy_live;
      e->graph_eddy[m] = eddy;
    }
    if (cudaGraphLaunch(e->graph[m], e->st) != cudaSuccess) {
      e->err = "ensemble graph launch failed";
      return DB_ERR_CUDA;
    }
    for (db_ctx* c : e->members) {
      c->time_step += 1;
      c->launches += e->kernels[m] / n;
    }
  }
  if (cudaStreamSynchronize(e->st) != cudaSuccess) {
    e->err = std::string("ensemble step failed: ") + cudaGetErrorString(cudaGetLastError());
    return DB_ERR_CUDA;
  }
  return DB_OK;
}

// ---------------------------------------------------------------------------
// autotuner: launch shapes timed on the context's own scratch buffers

template <typename F>
static float time_ms(db_ctx* c, F&& launch, int reps = 3) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch();   // warm-up (also sets kernel attributes)
  cudaEventRecord(a, c->st);
  for (int i = 0; i < reps; ++i) launch();
  cudaEventRecord(b, c->st);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

// the step graphs hold the launch shapes they were captured with
static void drop_graphs(db_ctx* c) {
  for (int i = 0; i < 2; ++i)
    if (c->graph[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph[i] = nullptr;
    }
}

extern "C" int db_get_tuning(db_ctx* c, int* shapes, int n) {
  if (!c || !shapes || n < DB_NTUNE) return DB_ERR_ARG;
  const Geom& g = c->g;
  const int v[DB_NTUNE] = {g.tune_xcps, g.tune_xgrid, g.tune_zns, g.tune_pgrid, g.tune_les_tb, g.tune_amd_ch};
  for (int i = 0; i < DB_NTUNE; ++i) shapes[i] = v[i];
  return DB_OK;
}

extern "C" int db_set_tuning(db_ctx* c, const int* shapes, int n) {
  if (!c || !shapes || n < DB_NTUNE) return DB_ERR_ARG;
  for (int i = 0; i < DB_NTUNE; ++i)
    if (shapes[i] < 0 || shapes[i] > 1024) return fail(c, DB_ERR_ARG, "launch shape out of range");
  Geom& g = c->g;
  g.tune_xcps = shapes[0];
  g.tune_xgrid = shapes[1];
  g.tune_zns = shapes[2];
  g.tune_pgrid = shapes[3];
  g.tune_les_tb = shapes[4];
  g.tune_amd_ch = shapes[5];
  drop_graphs(c);
  return DB_OK;
}

static int autotune_impl(db_ctx* c, char* report, int report_len) {
  if (!c) return DB_ERR_ARG;
  if (c->timing) return fail(c, DB_ERR_STATE, "turn stage timing off before db_autotune");
  Geom& g = c->g;
  State& s = c->s;
  std::string rep;
  char buf[160];
  const int T = g.nx / 8 > 0 ? g.nx / 8 : 1;     // threads per x sequence
  const int Tz = g.nz / 8 > 0 ? g.nz / 8 : 1;    // threads per z sequence
  // x-pass: sequences per staged item x persistent CTAs per SM (inverse x of 4 fields)
  {
    float best = 1e30f;
    int bc = 0, bg = 0;
    for (int cps = T >= 32 ? 1 : 32 / T; cps * T <= 256; cps *= 2)   // whole warps
      for (int gsm = 1; gsm <= 4; ++gsm) {
        g.tune_xcps = cps;
        g.tune_xgrid = gsm;
        const float ms = time_ms(c, [&] {
          launch_inv_x(g, fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]), fset(s.r1, s.r2, s.r3, s.rth), 4, c->st);
        });
        if (cudaGetLastError() != cudaSuccess) continue;
        snprintf(buf, sizeof buf, "x-pass cps %d ctas/SM %d: %.3f ms\n", cps, gsm, ms);
        rep += buf;
        if (ms < best) { best = ms; bc = cps; bg = gsm; }
      }
    g.tune_xcps = bc;
    g.tune_xgrid = bg;
  }
  // z-pass: sequences per CTA (inverse z of 4 fields)
  {
    float best = 1e30f;
    int bn = 0;
    for (int ns = Tz >= 32 ? 1 : 32 / Tz; ns * Tz <= 256; ns *= 2) {
      g.tune_zns = ns;
      const float ms = time_ms(c, [&] {
        launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3, s.cth), fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3]), 4, c->st);
      });
      if (cudaGetLastError() != cudaSuccess) continue;
      snprintf(buf, sizeof buf, "z-pass seqs/CTA %d: %.3f ms\n", ns, ms);
      rep += buf;
      if (ms < best) { best = ms; bn = ns; }
    }
    g.tune_zns = bn;
  }
  // products: persistent CTAs per SM (physical u in, x-half products out)
  {
    float best = 1e30f;
    int bg = 0;
    for (int gsm = 1; gsm <= 4; ++gsm) {
      g.tune_pgrid = gsm;
      const float ms = time_ms(c, [&] { launch_products(g, s, c->st, false); });
      if (cudaGetLastError() != cudaSuccess) continue;
      snprintf(buf, sizeof buf, "products ctas/SM %d: %.3f ms\n", gsm, ms);
      rep += buf;
      if (ms < best) { best = ms; bg = gsm; }
    }
    g.tune_pgrid = bg;
  }
  // LES Thomas: threads per CTA (matrices from the current dt)
  if (c->p.use_les) {
    CK(launch_tri_coef(g, c->ph, s, 0, c->st));
    float best = 1e30f;
    int bt = 0;
    for (int tb = 32; tb <= 128; tb *= 2) {   // kernel bound: 128 threads
      g.tune_les_tb = tb;
      const float ms = time_ms(c, [&] { launch_thomas_les(g, s, 0, c->st, true); });
      if (cudaGetLastError() != cudaSuccess) continue;
      snprintf(buf, sizeof buf, "LES Thomas threads/CTA %d: %.3f ms\n", tb, ms);
      rep += buf;
      if (ms < best) { best = ms; bt = tb; }
    }
    g.tune_les_tb = bt;
  }
  // LES closure walk: wall-normal chunks (nu_t, kappa_t kept: a substep
  // without the model reuses them)
  if (c->p.use_les) {
    const size_t pb = (size_t)g.np * g.pp * (g.prec ? sizeof(float) : sizeof(double));
    char* keep = reinterpret_cast<char*>(s.tscr);
    CK(cudaMemcpyAsync(keep, s.nu_t, pb, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(keep + pb, s.kappa_t, pb, cudaMemcpyDeviceToDevice, c->st));
    float best = 1e30f;
    int bch = 0;
    const int maxch = (g.ny + 1) / 8 > 1 ? (g.ny + 1) / 8 : 1;
    for (int ch = 1; ch <= maxch; ch *= 2) {
      g.tune_amd_ch = ch;
      const float ms = time_ms(c, [&] { launch_les_amd(g, c->ph, s, c->st); });
      if (cudaGetLastError() != cudaSuccess) continue;
      snprintf(buf, sizeof buf, "LES closure chunks %d: %.3f ms\n", ch, ms);
      rep += buf;
      if (ms < best) { best = ms; bch = ch; }
    }
    g.tune_amd_ch = bch;
    CK(cudaMemcpyAsync(s.nu_t, keep, pb, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(s.kappa_t, keep + pb, pb, cudaMemcpyDeviceToDevice, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  snprintf(buf, sizeof buf,
           "chosen: x-pass cps %d ctas/SM %d, z-pass seqs/CTA %d, products ctas/SM %d, LES Thomas %d, LES closure "
           "chunks %d\n",
           g.tune_xcps, g.tune_xgrid, g.tune_zns, g.tune_pgrid, g.tune_les_tb, g.tune_amd_ch);
  rep += buf;
  drop_graphs(c);   // captured steps hold the old launch shapes
  if (report && report_len > 0) {
    strncpy(report, rep.c_str(), (size_t)report_len - 1);
    report[report_len - 1] = 0;
  }
  return DB_OK;
}

extern "C" int db_autotune(db_ctx* c, char* report, int report_len) {
  return guarded([&] { return autotune_impl(c, report, report_len); });
}

extern "C" int db_set_timing(db_ctx* c, int enable) {
  if (!c) return DB_ERR_ARG;
  if (enable && !c->ev[0][0])
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k <= DB_NSTAGES; ++k) CK(cudaEventCreate(&c->ev[r][k]));
  if ((enable != 0) != c->timing)  // re-capture with/without event nodes
    for (int i = 0; i < 2; ++i)
      if (c->graph[i]) {
        cudaGraphExecDestroy(c->graph[i]);
        c->graph[i] = nullptr;
      }
  c->timing = enable != 0;
  return DB_OK;
}

extern "C" int db_stage_times(db_ctx* c, double* ms, int nstages) {
  if (!c || !ms || nstages < DB_NSTAGES) return DB_ERR_ARG;
  if (!c->timing) return fail(c, DB_ERR_STATE, "stage timing is off (db_set_timing)");
  CK(cudaStreamSynchronize(c->st));
  for (int k = 0; k < DB_NSTAGES; ++k) {
    double t = 0.0;
    for (int r = 0; r < 3; ++r) {
      float f = 0.f;
      CK(cudaEventElapsedTime(&f, c->ev[r][k], c->ev[r][k + 1]));
      t += f;
    }
    ms[k] = t;
  }
  return DB_OK;
}

extern "C" int db_set_sgs_net(db_ctx* c, db_sgs_net* net) {
  if (!c) return DB_ERR_ARG;
  c->sgs = net;
  c->s.sgs_range = net ? sgs_range_dev(net) : nullptr;
  for (int i = 0; i < 2; ++i)   // captured steps hold the old state pointers
    if (c->graph[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph[i] = nullptr;
    }
  return DB_OK;
}

extern "C" int db_les_eval(db_ctx* c, int model, double* nu_t, double* kappa_t, float* feat) {
  if (!c) return DB_ERR_ARG;
  if (!c->p.use_les) return fail(c, DB_ERR_STATE, "db_les_eval needs a context created with use_les");
  if (model != 5 && model != 6) return fail(c, DB_ERR_ARG, "model must be 5 (AMD) or 6 (learned closure)");
  if (model == 6 && !c->sgs) return fail(c, DB_ERR_STATE, "model 6 needs a network (db_set_sgs_net)");
  const Geom& g = c->g;
  State& s = c->s;
  cudaStream_t st = c->st;
  CK(launch_les_bc(g, c->ph, s, st));
  CK(launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3, s.cth, s.cu1, s.cu2, s.cu3, s.cth),
                  fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[4], s.xh[5], s.xh[6], s.xh[7]), 8, st, 0xF0u,
                  s.ghost));
  FieldSet in = fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[0], s.xh[1], s.xh[2], s.xh[3]);
  FieldSet out = fset(s.u1, s.u2, s.u3, s.th, s.gx[0], s.gx[1], s.gx[2], s.gx[3]);
  for (int i = 0; i < 4; ++i) { in.p[8 + i] = s.xh[4 + i]; out.p[8 + i] = s.gz[i]; }
  CK(launch_inv_x(g, in, out, 12, st, 0xF0u));
  if (feat) CK(launch_les_amd(g, c->ph, s, st, 1));
  if (model == 6) {
    if (sgs_forward_les_async(c->sgs, les_feat_src(c), g.prec != 0, s.sgs_out, (long long)g.np * g.pp, st))
      return fail(c, DB_ERR_CUDA, "closure inference failed");
  }
  CK(launch_les_amd(g, c->ph, s, st, model == 6 ? 2 : 0));
  c->launches += (model == 6 ? 6 : 5) + (feat ? 1 : 0);
  const size_t np_ = (size_t)g.np * g.pp;
  if (feat) {
    CK(cudaMemcpyAsync(feat, s.sgs_feat, np_ * 16 * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  const int nx2 = c->p.nx + 2, nz2 = c->p.nz + 2;
  if (nu_t) {
    memset(nu_t, 0, sizeof(double) * np_ / ((size_t)g.nx * g.nz) * nz2 * nx2);
    int rc = phys_download(c, s.nu_t, nu_t);
    if (rc) return rc;
  }
  if (kappa_t) {
    memset(kappa_t, 0, sizeof(double) * np_ / ((size_t)g.nx * g.nz) * nz2 * nx2);
    int rc = phys_download(c, s.kappa_t, kappa_t);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(st));
  return DB_OK;
}

namespace db {
struct SgsData {
  int fx, fy, fz;
  int nxc, nzc, nyc;
  int kmin, kmax;
  double dxc3, dzc3;
  const double* dyc2;
  float* feat;
  float* target;
};
cudaError_t launch_sgs_targets(const Geom& g, const State& s, const SgsData& d, cudaStream_t st);
}  // namespace db

extern "C" int db_sgs_targets(db_ctx* c, int fx, int fy, int fz, const double* gy_coarse, float* d_feat,
                              float* d_target, long long* npts) {
  if (!c || !gy_coarse || !npts) return DB_ERR_ARG;
  const Geom& g = c->g;
  if (!c->s.gx[0]) {   // a DNS context: gradient fields on first use
    const size_t bytes = (size_t)g.np * g.pp * phys_elem(c);
    for (int i = 0; i < 4; ++i) {
      int rc;
      if ((rc = balloc(c, (void**)&c->s.gx[i], bytes)) || (rc = balloc(c, (void**)&c->s.gz[i], bytes))) return rc;
    }
  }
  if (fx < 1 || fz < 1 || fy < 2 || (fy & 1) || g.nx % fx || g.nz % fz || (g.ny - 1) % fy)
    return fail(c, DB_ERR_ARG, "filter factors must divide nx, nz and ny - 1 (fy even)");
  const int nxc = g.nx / fx, nzc = g.nz / fz, nyc = (g.ny - 1) / fy + 1;
  if (nyc < 5) return fail(c, DB_ERR_SIZE, "coarse grid needs at least 5 wall-normal points");
  const long long n = (long long)nxc * nzc * (nyc - 3);
  *npts = n;
  if (!d_feat || !d_target) return DB_OK;   // size query
  // coarse metrics (same construction as db_init)
  std::vector<double> cgy(nyc + 2, 0.0), cgyf(nyc + 2, 0.0), c2dy(nyc + 2, 0.0);
  for (int j = 1; j <= nyc + 1; ++j) cgy[j] = gy_coarse[j - 1];
  for (int j = 1; j <= nyc; ++j) cgyf[j] = 0.5 * (cgy[j] + cgy[j + 1]);
  cgyf[0] = 2.0 * cgyf[1] - cgyf[2];
  cgyf[nyc + 1] = 2.0 * cgyf[nyc] - cgyf[nyc - 1];
  for (int j = 1; j <= nyc + 1; ++j) c2dy[j] = 2.0 * (cgyf[j] - cgyf[j - 1]);
  double* d_dy = nullptr;
  CK(cudaMalloc(&d_dy, c2dy.size() * sizeof(double)));
  CK(cudaMemcpy(d_dy, c2dy.data(), c2dy.size() * sizeof(double), cudaMemcpyHostToDevice));
  State& s = c->s;
  cudaStream_t st = c->st;
  // the state and its x and z derivatives in physical space (no ghost overlay)
  CK(launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3, s.cth, s.cu1, s.cu2, s.cu3, s.cth),
                  fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[4], s.xh[5], s.xh[6], s.xh[7]), 8, st, 0xF0u));
  FieldSet in = fset(s.xh[0], s.xh[1], s.xh[2], s.xh[3], s.xh[0], s.xh[1], s.xh[2], s.xh[3]);
  FieldSet out = fset(s.u1, s.u2, s.u3, s.th, s.gx[0], s.gx[1], s.gx[2], s.gx[3]);
  for (int i = 0; i < 4; ++i) { in.p[8 + i] = s.xh[4 + i]; out.p[8 + i] = s.gz[i]; }
  CK(launch_inv_x(g, in, out, 12, st, 0xF0u));
  SgsData d{fx, fy, fz, nxc, nzc, nyc, 3, nyc - 1, 3.0 * c->p.lx / nxc, 3.0 * c->p.lz / nzc, d_dy, d_feat, d_target};
  cudaError_t e = launch_sgs_targets(g, s, d, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaFree(d_dy);
  c->launches += 3;
  CK(e);
  CK(e2);
  return DB_OK;
}

static int need_net(db_ctx* c) {
  if (c->p.use_les && c->p.les_model_type == 6 && !c->sgs)
    return fail(c, DB_ERR_STATE, "les_model_type 6 needs a network (db_set_sgs_net)");
  return DB_OK;
}

extern "C" int db_set_wait_limit(db_ctx* c, uint32_t polls) {
  if (!c) return DB_ERR_ARG;
  c->g.wait_first = polls;
  drop_graphs(c);   // captured steps hold the old Geom
  return DB_OK;
}

extern "C" int db_kernel_launches(db_ctx* c, long long* count) {
  if (!c || !count) return DB_ERR_ARG;
  *count = c->launches;
  return DB_OK;
}

extern "C" int db_rem_div(db_ctx* c) {
  if (!c) return DB_ERR_ARG;
  CK(launch_rem_div(c->g, c->s, 0, 0, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

extern "C" int db_apply_bc_vel_post(db_ctx* c) {
  if (!c) return DB_ERR_ARG;
  CK(launch_bc_vel_post(c->g, c->ph, c->s, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DB_OK;
}

extern "C" int db_courant(db_ctx* c, double* delta_t_out) {
  if (!c) return DB_ERR_ARG;
  const Geom& g = c->g;
  State& s = c->s;
  CK(launch_inv_z(g, fset(s.cu1, s.cu2, s.cu3), fset(s.xh[0], s.xh[1], s.xh[2]), 3, c->st));
  CK(launch_inv_x(g, fset(s.xh[0], s.xh[1], s.xh[2]), fset(s.u1, s.u2, s.u3), 3, c->st));
  CflCtl ctl{c->p.cfl, c->p.time_limit, 1, 1, 1};
  CK(launch_courant(g, c->ph, s, ctl, c->st));
  CK(launch_apply_dt(s.sc, c->st));
  db_status stt;
  int rc = db_get_status(c, &stt);
  if (rc) return rc;
  if (delta_t_out) *delta_t_out = stt.delta_t;
  return DB_OK;
}

extern "C" int db_stats(db_ctx* c, double* out) {
  if (!c || !out) return DB_ERR_ARG;
  const int np = c->g.np;
  // the device rows: ume vme wme thme, the four variances, uv wv uw thv,
  // the gradient sum of epsilon, |grad th|^2 (k_stats.cu)
  constexpr int NDEV = 14;
  static_assert(NDEV == DB_NSTAT, "device rows and output rows");
  if (!c->stats && balloc(c, (void**)&c->stats, (size_t)NDEV * np * sizeof(double)))
    return fail(c, DB_ERR_CUDA, "db_stats: out of device memory");
  const int homx = !(c->p.ic_type >= 5 && c->p.ic_type <= 8);   // for/parameters.f90:282-286
  CK(launch_stats(c->g, c->s, homx, c->stats, c->st));
  CK(cudaMemcpyAsync(out, c->stats, (size_t)NDEV * np * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const double bg = c->ph.dthdx * c->ph.dthdx + c->ph.dthdz * c->ph.dthdz;
  for (int j = 0; j < np; ++j) {
    for (int r = DB_ST_URMS; r <= DB_ST_THRMS; ++r) out[r * np + j] = sqrt(fmax(out[r * np + j], 0.0));
    out[DB_ST_EPSILON * np + j] *= c->ph.nu;
    if (j >= 1 && j <= c->g.ny) out[DB_ST_CHI * np + j] += bg;
  }
  return DB_OK;
}

// FP64 scratch of the diagnostics (first use): four physical fields and one
// x-half field
static int budget_alloc(db_ctx* c) {
  const Geom& g = c->g;
  const size_t Pn = (size_t)g.np * g.pp, H = (size_t)g.np * g.hp;
  for (int f = 0; f < 4; ++f)
    if (!c->bud_phys[f] && balloc(c, (void**)&c->bud_phys[f], Pn * sizeof(double)))
      return fail(c, DB_ERR_CUDA, "diagnostics scratch: out of device memory");
  if (!c->bud_xh && balloc(c, (void**)&c->bud_xh, H * sizeof(double2)))
    return fail(c, DB_ERR_CUDA, "diagnostics scratch: out of device memory");
  return DB_OK;
}

// FP64 transforms with the built-in launch shapes, whatever the context's
// work type and tuning
static Geom fp64_geom(const Geom& g) {
  Geom g64 = g;
  g64.prec = 0;
  g64.tune_xcps = g64.tune_xgrid = g64.tune_zns = 0;
  return g64;
}

// the state's u1, u2, u3, th in FP64 physical space (the budget scratch),
// whatever the work type of the context
static int budget_fields(db_ctx* c) {
  int rc = budget_alloc(c);
  if (rc) return rc;
  const Geom g64 = fp64_geom(c->g);
  double2* src[4] = {c->s.cu1, c->s.cu2, c->s.cu3, c->s.cth};
  for (int f = 0; f < 4; ++f) {
    CK(launch_inv_z(g64, fset(src[f]), fset(c->bud_xh), 1, c->st));
    CK(launch_inv_x(g64, fset(c->bud_xh), fset(c->bud_phys[f]), 1, c->st));
  }
  return DB_OK;
}

static int homogeneous_x(const db_ctx* c) { return !(c->p.ic_type >= 5 && c->p.ic_type <= 8); }   // parameters.f90:282-286

extern "C" int db_budget(db_ctx* c, double* out) {
  if (!c || !out) return DB_ERR_ARG;
  const int np = c->g.np;
  if (!c->bud_mxy && balloc(c, (void**)&c->bud_mxy, (size_t)3 * np * c->g.nx * sizeof(double)))
    return fail(c, DB_ERR_CUDA, "db_budget: out of device memory");
  if (!c->bud_out && balloc(c, (void**)&c->bud_out, (size_t)DB_NBUD * np * sizeof(double)))
    return fail(c, DB_ERR_CUDA, "db_budget: out of device memory");
  int rc = budget_fields(c);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->bud_out, 0, (size_t)DB_NBUD * np * sizeof(double), c->st));
  CK(launch_budget(c->g, c->ph, c->s, fset(c->bud_phys[0], c->bud_phys[1], c->bud_phys[2], c->bud_phys[3]),
                   homogeneous_x(c), c->bud_mxy, c->bud_out, c->st));
  CK(cudaMemcpyAsync(out, c->bud_out, (size_t)DB_NBUD * np * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->launches += 3 + 8;
  return DB_OK;
}

// save_stats_LES_OOL's means and compute_TKE_diss_les (k_budget.cu)
extern "C" int db_les_stats(db_ctx* c, double* out) {
  if (!c || !out) return DB_ERR_ARG;
  if (!c->p.use_les || !c->s.nu_t) return fail(c, DB_ERR_ARG, "db_les_stats: not an LES context");
  const int np = c->g.np;
  if (!c->bud_out && balloc(c, (void**)&c->bud_out, (size_t)DB_NBUD * np * sizeof(double)))
    return fail(c, DB_ERR_CUDA, "db_les_stats: out of device memory");
  int rc = budget_fields(c);
  if (rc) return rc;
  CK(launch_les_stats(c->g, c->s, fset(c->bud_phys[0], c->bud_phys[1], c->bud_phys[2]), c->bud_out, c->st));
  CK(cudaMemcpyAsync(out, c->bud_out, (size_t)DB_NLES * np * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->launches += 1 + 8;
  return DB_OK;
}

extern "C" int db_bpe(db_ctx* c, int nbin, double* pdf, double* th_bin, double* bpe) {
  if (!c || nbin < 1 || nbin > (1 << 16)) return DB_ERR_ARG;
  if (c->bud_nbin < nbin) {
    if (balloc(c, (void**)&c->bud_pdf, (size_t)nbin * sizeof(double)))
      return fail(c, DB_ERR_CUDA, "db_bpe: out of device memory");
    c->bud_nbin = nbin;
  }
  int rc = budget_fields(c);
  if (rc) return rc;
  const int homx = homogeneous_x(c);
  CK(cudaMemsetAsync(c->bud_pdf, 0, (size_t)nbin * sizeof(double), c->st));
  CK(launch_bpe_pdf(c->g, c->ph, c->bud_phys[3], homx, nbin, c->bud_pdf, c->st));
  std::vector<double> P((size_t)nbin), B((size_t)nbin + 1), Y((size_t)nbin + 1);
  CK(cudaMemcpyAsync(P.data(), c->bud_pdf, (size_t)nbin * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->launches += 1 + 8;
  // bins, normalised PDF, sorted heights Y_r and the BPE (diagnostics.f90:1762-1835)
  const Phys& ph = c->ph;
  if (homx) {
    const double thmin = -ph.dthdx * 0.5 * ph.lx * 1.1, thmax = ph.dthdx * 0.5 * ph.lx * 1.1;
    const double dth = (thmax - thmin) / nbin + 1.e-14;
    for (int i = 0; i <= nbin; ++i) B[i] = thmin + i * dth;
  } else {
    for (int i = 0; i <= nbin; ++i) B[i] = -(ph.ro_inv + 1.e-14) * cos(i * c->pi_ref / nbin);
  }
  double sum = 0.0;
  for (double v : P) sum += v;
  if (sum > 0.0)
    for (double& v : P) v /= sum;
  Y[0] = 0.0;
  for (int i = 1; i <= nbin; ++i) Y[i] = Y[i - 1] + P[i - 1];
  for (double& v : Y) v *= c->p.ly;
  double e = 0.0;
  for (int i = 0; i < nbin; ++i)
    e -= (0.5 * (B[i + 1] + B[i]) * 0.5 * (Y[i + 1] + Y[i])) * (Y[i + 1] - Y[i]) / c->p.ly;
  if (pdf) std::copy(P.begin(), P.end(), pdf);
  if (th_bin) std::copy(B.begin(), B.end(), th_bin);
  if (bpe) *bpe = e;
  return DB_OK;
}

// Bin_Ystar_and_Write (for/diagnostics.f90:1859-1950): a physical field
// binned by the buoyancy with its background gradient (the bins of
// compute_BPE), dyf-weighted, divided by the bins' weights
extern "C" int db_bin_ystar(db_ctx* c, int kind, const double* field, int nbin, double* binned, double* weight) {
  if (!c || nbin < 1 || nbin > (1 << 13) || !binned) return DB_ERR_ARG;
  if (kind != DB_ZS_FIELD && kind != DB_ZS_KE) return fail(c, DB_ERR_ARG, "db_bin_ystar: unknown kind");
  if (kind == DB_ZS_FIELD && !field) return fail(c, DB_ERR_ARG, "db_bin_ystar: no field");
  const Geom& g = c->g;
  if (c->bud_nbin < 2 * nbin) {
    if (balloc(c, (void**)&c->bud_pdf, (size_t)2 * nbin * sizeof(double)))
      return fail(c, DB_ERR_CUDA, "db_bin_ystar: out of device memory");
    c->bud_nbin = 2 * nbin;
  }
  int rc = budget_fields(c);
  if (rc) return rc;
  const double* f0 = c->bud_phys[0];
  if (kind == DB_ZS_FIELD) {
    if (!c->zs_field && balloc(c, (void**)&c->zs_field, (size_t)g.np * g.pp * sizeof(double)))
      return fail(c, DB_ERR_CUDA, "db_bin_ystar: out of device memory");
    // reference physical layout real(0:Nx+1, 0:Nz+1, 0:Nyp+1): the Nx x Nz
    // points of each plane
    for (int j = 0; j < g.np; ++j)
      CK(cudaMemcpy2DAsync(c->zs_field + (size_t)j * g.pp, (size_t)g.nx * sizeof(double),
                           field + (size_t)j * (g.nz + 2) * (g.nx + 2), (size_t)(g.nx + 2) * sizeof(double),
                           (size_t)g.nx * sizeof(double), (size_t)g.nz, cudaMemcpyHostToDevice, c->st));
    f0 = c->zs_field;
  }
  CK(cudaMemsetAsync(c->bud_pdf, 0, (size_t)2 * nbin * sizeof(double), c->st));
  CK(launch_bpe_pdf(g, c->ph, c->bud_phys[3], homogeneous_x(c), nbin, c->bud_pdf, c->st, c->bud_pdf + nbin, kind,
                    f0, c->bud_phys[1], c->bud_phys[2]));
  std::vector<double> h((size_t)2 * nbin);
  CK(cudaMemcpyAsync(h.data(), c->bud_pdf, (size_t)2 * nbin * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->launches += 1 + 8;
  for (int b = 0; b < nbin; ++b) {
    binned[b] = h[(size_t)nbin + b] / h[b];   // 0/0 in an empty bin, as the reference divides
    if (weight) weight[b] = h[b];
  }
  return DB_OK;
}

// poisson_p_chan (for/solver.f90:1382-1590), k_pressure.cu
extern "C" int db_poisson_p(db_ctx* c) {
  if (!c) return DB_ERR_ARG;
  int rc = budget_alloc(c);
  if (rc) return rc;
  const Geom g64 = fp64_geom(c->g);
  const State& s = c->s;
  cudaStream_t st = c->st;
  double2 *w1 = s.crs[0], *w2 = s.crs[1], *R = s.crs[2];   // free between substeps
  double *P1 = c->bud_phys[0], *P2 = c->bud_phys[1], *Q = c->bud_phys[2];
  CK(cudaMemsetAsync(Q, 0, (size_t)c->g.np * c->g.pp * sizeof(double), st));
  for (int term = 0; term < 6; ++term) {
    const bool pair = term >= 3;
    CK(launch_pp_terms(c->g, s, term, w1, pair ? w2 : nullptr, st));
    CK(launch_inv_z(g64, fset(w1), fset(c->bud_xh), 1, st));
    CK(launch_inv_x(g64, fset(c->bud_xh), fset(P1), 1, st));
    if (pair) {
      CK(launch_inv_z(g64, fset(w2), fset(c->bud_xh), 1, st));
      CK(launch_inv_x(g64, fset(c->bud_xh), fset(P2), 1, st));
    }
    CK(launch_pp_accum(c->g, P1, P2, pair ? 0 : 1, Q, st));
  }
  CK(launch_fwd_x(g64, fset(Q), fset(c->bud_xh), 1, st));
  CK(launch_fwd_z(g64, fset(c->bud_xh), fset(R), 1, st));
  CK(launch_pp_solve(c->g, s, R, s.phi_g, reinterpret_cast<double*>(s.crs[3]), st));
  CK(cudaStreamSynchronize(st));
  c->launches += 6 * 3 + 3 * 2 + 3;
  return DB_OK;
}

extern "C" int db_divergence(db_ctx* c, double* max_div_out) {
  if (!c) return DB_ERR_ARG;
  CK(cudaMemsetAsync(&c->s.sc->max_div, 0, sizeof(double), c->st));
  CK(launch_divergence(c->g, c->s, c->st));
  db_status stt;
  int rc = db_get_status(c, &stt);
  if (rc) return rc;
  if (max_div_out) *max_div_out = stt.max_div;
  return DB_OK;
}
