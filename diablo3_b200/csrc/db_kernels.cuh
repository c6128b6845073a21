// db_kernels.cuh -- declarations shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include "db_common.cuh"
#include "cplx_dft.cuh"

namespace db {

// FFT twiddle tables in the work precision R
template <typename R> __device__ __forceinline__ const typename CplxOf<R>::type* tw_x(const Geom& g);
template <> __device__ __forceinline__ const double2* tw_x<double>(const Geom& g) { return g.twx; }
template <> __device__ __forceinline__ const float2* tw_x<float>(const Geom& g) { return g.twxf; }
template <typename R> __device__ __forceinline__ const typename CplxOf<R>::type* tw_z(const Geom& g);
template <> __device__ __forceinline__ const double2* tw_z<double>(const Geom& g) { return g.twz; }
template <> __device__ __forceinline__ const float2* tw_z<float>(const Geom& g) { return g.twzf; }

constexpr int KT = 4;           // kx columns per z-pass CTA (kxs is a multiple of 4)

// minimum resident CTAs per SM requested from the compiler (register caps)
#ifndef DB_LB_FFT
#define DB_LB_FFT 3
#endif
// k_rhs_cn: minimum resident 32-thread CTAs per SM (13 keeps every mode's
// thread of a 512x512 plane resident at once: 128 registers)
#ifndef DB_RHSCN_LB
#define DB_RHSCN_LB 13
#endif
#ifndef DB_LB_ZPASS
#define DB_LB_ZPASS 2
#endif
#ifndef DB_ZPASS_LAZY
#define DB_ZPASS_LAZY 1
#endif
#ifndef DB_LB_PROD
#define DB_LB_PROD 4
#endif
constexpr int MAXF = 12;

struct FieldSet {
  void* p[MAXF];
};

inline FieldSet fset(void* a = nullptr, void* b = nullptr, void* c = nullptr, void* d = nullptr,
                     void* e = nullptr, void* f = nullptr, void* g = nullptr, void* h = nullptr) {
  FieldSet s{};
  s.p[0] = a; s.p[1] = b; s.p[2] = c; s.p[3] = d;
  s.p[4] = e; s.p[5] = f; s.p[6] = g; s.p[7] = h;
  return s;
}

// k_fft.cu
cudaError_t launch_fwd_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st);
// dmask: bit f set -> field f is differentiated (x: i kx, z: i kz) on the way
cudaError_t launch_inv_x(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, unsigned dmask = 0);
// accumulate: out += transform, with rows 0, 1, Nyp, Nyp+1 based on ghost
// (when given) instead of out
// NL_e = (Z(N_e) + i kz Z(M_e)) / Nz of the four equations from the 8 x-half
// product fields (in.p[2e], in.p[2e+1]) into out.p[e], FP64 packed spectral
cudaError_t launch_fwd_z_nl(const Geom& g, FieldSet in, FieldSet out, cudaStream_t st);
cudaError_t launch_fwd_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, int accumulate = 0,
                         const double2* ghost = nullptr);
// ghost (optional): rows 0, 1, Nyp, Nyp+1 of field f are read from
// ghost + (4 (f % 4) + q) sp instead (q = 0..3 for those rows);
// mean (optional): fields 0..3 leave their plane mean ((0,0) mode) out of the
// transform and store it in mean[f np + j] (FP64)
cudaError_t launch_inv_z(const Geom& g, FieldSet in, FieldSet out, int nf, cudaStream_t st, unsigned dmask = 0,
                         const double2* ghost = nullptr, double* mean = nullptr);

// Tridiagonal row description of one implicit equation (one per row j of
// 0..Nyp+1): coefficients l, d, u; is_bc marks rows whose right-hand side
// is the constant bc (from apply_BC_*), others take r + CN-explicit term.
struct TriRow {
  double l, d, u, bc;
  double ap;      // forward-eliminated multiplier a'_j (Thomas)
  double ibp;     // 1 / b'_j
  double cn_lo, cn_hi;  // explicit CN: term = cn_hi*(u_{j+1}-u_j) - cn_lo*(u_j-u_{j-1})
  // eddy-viscosity metric factors of the row (LES): the lower / upper
  // coupling is nu_lo * ef_lo, nu_hi * ef_hi (per-column nu), with
  // ef = 1/(dy dyf) at the neighbouring GY / GYF spacing
  double ef_lo, ef_hi;
  int is_bc, interior;
};

// Per-row constants of the AMD model (k_les_amd), host-computed once:
// reciprocals of the spacings, the filter coefficients -2 C^2 Delta^2 at GY
// and GYF rows, the filter-width ratios at GY rows and the GYF -> GY
// interpolation weights (A(j) dyf(j-1) + A(j-1) dyf(j)) / (2 dy(j)).
struct LesRow {
  double idy, idyf;        // 1/dy(j), 1/dyf(j)
  double dgy, dgyf;        // filter coefficient at GY row j, GYF row j
  double ryx, rxy;         // (2 dy(j)) / (3 dx), (3 dx) / (2 dy(j))
  double rzy, ryz;         // (3 dz) / (2 dy(j)), (2 dy(j)) / (3 dz)
  double wa, wb;           // dyf(j-1) / (2 dy(j)), dyf(j) / (2 dy(j))
  double dys_f;            // 2 dyf(j)  (GYF-row y filter width)
  double dys_y;            // 2 dy(j)   (GY-row y filter width)
};

__device__ __forceinline__ bool in_rng(int j, int a, int b) { return j >= a && j <= b; }

// per-plane metric factors of the nonlinear products: 1 / (2 dyf_j),
// 1 / dy_j, dyf_j / (2 dy_j), dyf_{j-1} / (2 dy_j) (the y-differences and GY
// interpolations multiply by these instead of dividing per point)
template <typename R>
struct ProdY {
  R i2dyf, idy, wj, wjm;
  __device__ ProdY(const Geom& g, int j) {
    const double dyj = g.dy[j], dyfj = g.dyf[j], dyfjm = (j >= 1) ? g.dyf[j - 1] : 0.0;
    i2dyf = (R)(1.0 / (2.0 * dyfj));
    idy = (R)(1.0 / dyj);
    wj = (R)(dyfj / (2.0 * dyj));
    wjm = (R)(dyfjm / (2.0 * dyj));
  }
};

// Pointers of the full device state for the substep kernels.  Physical and
// x-half fields are typed double / double2 here; with Geom::prec = 1 they
// hold float / float2 and the kernels cast them to their work type.
struct State {
  double2 *cu1, *cu2, *cu3, *cp, *cth;       // spectral
  double2 *cf1, *cf2, *cf3, *cfth;           // spectral RK history
  double2* xh[8];                            // x-half scratch
  double *u1, *u2, *u3, *th;                 // physical
  double *r1, *r2, *r3, *rth;                // physical RHS
  double2* phi_g;                            // rem_div forward-sweep scratch (spectral)
  double2* nls[8];                           // z-pass scratch of the FP64 path: Z(N_e), Z(M_e), then cr_e (spectral)
  double2* crs[4];                           // cr of u1, u3, u2, th (spectral FP64) for the spectral CN solve (no LES)
  double2* pfac;                             // rem_div factors: a' then 1/b', each np x sp doubles
  TriRow* tri;                               // 4 equations x np rows (th, u2, u1, u3)
  DevScalars* sc;
  // LES (les_model_type 5), physical [j][z][x]; null without use_les
  double* gx[4];                             // d/dx of u1, u2, u3, th
  double* gz[4];                             // d/dz of u1, u2, u3, th
  double* les[11];                           // LES: the products' 11 real sequences + SGS forcing (k_les.cu)
  double *nu_t, *kappa_t;                    // eddy viscosity / diffusivity at GY rows
  double2* ghost;                            // [4 fields][rows 0, 1, Nyp, Nyp+1][sp] (k_les_bc)
  double* tscr;                              // FP64 Thomas scratch, two fields per equation (LES)
  const LesRow* lrow;                        // np rows (LES)
  // learned closure (les_model_type 6): features [point][16], outputs
  // [point][2] (nu_t, kappa_t), training range lo[16], hi[16]
  float* sgs_feat;
  float* sgs_out;
  const float* sgs_range;
  // plane means of u1, u2, u3, th ([f][j], FP64) when the physical fields of
  // this substep hold fluctuations about them (mixed path with LES), else null
  double* umean;                             // the table (allocated with LES)
  const double* pmean;                       // umean while the split is in effect
};

// a physical field value with its plane mean added back (pmean non-null):
// the single rounding every consumer of the split fields shares
template <typename R>
__device__ __forceinline__ R with_mean(R v, const double* pmean, int f, int np, int j) {
  return pmean ? v + (R)pmean[(long long)f * np + j] : v;
}

// (a - b) * id for the values a, b of field f at rows ja, jb: with split
// fields the difference of the fluctuations plus that of the FP64 means, so
// a large mean (the stratification in th) adds no rounding noise to a
// y-derivative; one explicit fma, so every call site rounds alike
template <typename R>
__device__ __forceinline__ R ydiff(R a, R b, const double* pmean, int f, int np, int ja, int jb, double id) {
  const R dm = pmean ? (R)((pmean[(long long)f * np + ja] - pmean[(long long)f * np + jb]) * id) : (R)0;
  return fma(a - b, (R)id, dm);
}

// Member-batched launches (ensembles of equal-sized channels without LES):
// one launch covers every member, the member index folded into a grid
// dimension the kernel does not use otherwise; member m's state, physics
// and the field sets of the batched transforms come from a device table,
// the geometry is member 0's kernel parameter (the same for every member;
// of the table's copy only the flags word is used).  Kernels instantiated
// with B = false take their arguments as before and ignore the table.
enum { FS_CU4 = 0, FS_XH4, FS_U4, FS_XH8, FS_XH8Z, FS_NL, FS_NSLOT };
struct MemberArgs {
  State s;
  Geom g;
  Phys ph;
  // FS_CU4 cu1, cu2, cu3, cth; FS_XH4 xh[0..3]; FS_U4 u1, u2, u3, th;
  // FS_XH8 xh[0..7]; FS_XH8Z xh[0, 2, 4, 6, 1, 3, 5, 7] (the FP64 z-pass
  // input order); FS_NL crs[0..3], nls[4..7]
  FieldSet fs[FS_NSLOT];
};
struct Batch {
  const MemberArgs* tab;   // device table of n members (null: one context)
  int n;
  int nf;                  // fields per member of a batched transform
  int fin, fout;           // its field-set slots
};
// the table entry of one context
MemberArgs member_args(const Geom& g, const Phys& ph, const State& s);
// one substep's kernels for every member (spectral path: no LES, fixed dt),
// with g member 0's geometry (launch shapes); tri_coef on st_side, joined
// through the two events before the solves
cudaError_t launch_substep_batch(const Geom& g, const Batch& b, int rk, cudaStream_t st, cudaStream_t st_side,
                                 cudaEvent_t ev_fork, cudaEvent_t ev_join);
// time_step += 1 (end = 0) or time += delta_t (end = 1) of every member
cudaError_t launch_steps_batch(const Batch& b, int end, cudaStream_t st);
// batched transforms (k_fft.cu): nf fields of every member from slot fin
// to slot fout
cudaError_t launch_inv_z_batch(const Geom& g, const Batch& b, cudaStream_t st);
cudaError_t launch_inv_x_batch(const Geom& g, const Batch& b, cudaStream_t st);
cudaError_t launch_fwd_z_batch(const Geom& g, const Batch& b, cudaStream_t st);
cudaError_t launch_fwd_z_nl_batch(const Geom& g, const Batch& b, cudaStream_t st);

// k_substep.cu; les: add the SGS forcing fields s.les to the products
int sm_count();   // SMs of the current device (cached)
cudaError_t launch_products(const Geom& g, const State& s, cudaStream_t st, bool les = false);
// ghost: the LES overlay, when the inverse transforms of this substep used it
cudaError_t launch_zpass_rhs(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st,
                             const double2* ghost = nullptr);
cudaError_t launch_tri_coef(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st);
// the substep without LES: the nonlinear terms NL_e of the 4 equations into
// spectral scratch (s.crs), then the spectral RHS joined with the CN solves
// in spectral space (k_rhs_cn, k_cn_back), the state in place
cudaError_t launch_zpass_spec(const Geom& g, const State& s, cudaStream_t st);
cudaError_t launch_rhs_cn(const Geom& g, const Phys& ph, const State& s, int rk, cudaStream_t st);

struct CflCtl {
  double cfl, time_limit;
  int variable_dt, update_dt;
  int force;               // 1: evaluate regardless of variable_dt/time_step
};
cudaError_t launch_courant(const Geom& g, const Phys& ph, const State& s, CflCtl ctl, cudaStream_t st);
// courant from the x-half u1, u2, u3 (in): their inverse x-pass reduces the
// CFL terms instead of storing the physical fields, then k_courant_final
cudaError_t launch_inv_x_cfl(const Geom& g, const Phys& ph, const State& s, CflCtl ctl, FieldSet in, cudaStream_t st);
cudaError_t launch_courant_final(const Phys& ph, const State& s, CflCtl ctl, cudaStream_t st);
cudaError_t launch_rem_div(const Geom& g, const State& s, int rk, int update_cp, cudaStream_t st);
cudaError_t launch_pfac(const Geom& g, const State& s, cudaStream_t st);
cudaError_t launch_apply_dt(DevScalars* sc, cudaStream_t st);
cudaError_t launch_step_begin(DevScalars* sc, cudaStream_t st);
cudaError_t launch_step_end(DevScalars* sc, cudaStream_t st);
cudaError_t launch_divergence(const Geom& g, const State& s, cudaStream_t st);
cudaError_t launch_stats(const Geom& g, const State& s, int homx, double* out, cudaStream_t st);
// spectral field: compact device layout <-> reference host layout, on the device
cudaError_t launch_spec_to_ref(const Geom& g, int nx, int nz, const double2* src, double2* ref, cudaStream_t st);
cudaError_t launch_ref_to_spec(const Geom& g, int nx, int nz, const double2* ref, double2* dst, cudaStream_t st);
// one physical field between the reference layout (device doubles) and the
// compact layout at the context's precision
cudaError_t launch_phys_from_ref(const Geom& g, int nx, int nz, const double* ref, void* dst, cudaStream_t st);
cudaError_t launch_phys_to_ref(const Geom& g, int nx, int nz, const void* src, double* ref, cudaStream_t st);
cudaError_t launch_bc_vel_post(const Geom& g, const Phys& ph, const State& s, cudaStream_t st);

// k_les.cu
cudaError_t launch_les_bc(const Geom& g, const Phys& ph, const State& s, cudaStream_t st);
// mode 0: AMD; 1: closure features only; 2: closure nu_t, kappa_t with AMD fallback
cudaError_t launch_les_amd(const Geom& g, const Phys& ph, const State& s, cudaStream_t st, int mode = 0);
cudaError_t launch_thomas_les(const Geom& g, const State& s, int rk, cudaStream_t st, bool keep_u);
// k_budget.cu: energy-budget rows (homx: x-z means, else z-means per x)
// from the FP64 physical u1, u2, u3 (phys.p[0..2]) and the spectral state;
// mxy scratch [3][np][Nx], out [DB_NBUD][np]
cudaError_t launch_budget(const Geom& g, const Phys& ph, const State& s, FieldSet phys, int homx, double* mxy,
                          double* out, cudaStream_t st);
// save_stats_LES_OOL's plane means of nu_t, kappa_t and compute_TKE_diss_les
// (out[3][np]) from the FP64 physical u1, u2, u3 (phys)
cudaError_t launch_les_stats(const Geom& g, const State& s, FieldSet phys, double* out, cudaStream_t st);
// PDF of th + dTHdX (x - Lx/2) over planes jstart_th..jend_th (weights dyf)
cudaError_t launch_bpe_pdf(const Geom& g, const Phys& ph, const double* th, int homx, int nbin, double* pdf,
                           cudaStream_t st, double* fbin = nullptr, int kind = 0, const double* f0 = nullptr,
                           const double* f1 = nullptr, const double* f2 = nullptr);
// k_pressure.cu: poisson_p_chan's term factors, physical products and the
// Poisson solve of cp
cudaError_t launch_pp_terms(const Geom& g, const State& s, int term, double2* w1, double2* w2, cudaStream_t st);
cudaError_t launch_pp_accum(const Geom& g, const double* p1, const double* p2, int square, double* q,
                            cudaStream_t st);
cudaError_t launch_pp_solve(const Geom& g, const State& s, const double2* rhs, double2* gsc, double* bsc,
                            cudaStream_t st);
// mixed path: the LES solve's FP64 increments (u1, u2, u3, th) and the
// FP64 x-half scratch beside them (k_les.cu)
void thomas_les_inc(const Geom& g, const State& s, double* inc[4], double2* xh64[4]);

}  // namespace db
