/* SPDX-License-Identifier: GPL-3.0-or-later
 *
 * cw_dycore.h -- C ABI of the B200-native WRF-ARW RK3 split-explicit dynamical core.
 *
 * This is the drop-in boundary for CPPWRF's dynamics step. Every entry point below replaces one
 * reference interface; the citation after each declaration names it (file:line in CPPWRF).
 * Conventions (all entry points):
 *   - plain C types, no C++ or torch types; every function returns int: 0 = ok, < 0 = error
 *     (the message is kept per handle, cw_last_error), > 0 = a WRF fatal code raised on the device;
 *   - no exceptions cross the ABI; a handle is used by one host thread at a time (as RK3 is,
 *     src/dyn/rk3.hpp:34, one host thread per domain, src/core/backend.cpp:73-81);
 *   - field memory uses CPPWRF's Layout (src/core/halo.cpp:12-48): structure of arrays, i fastest,
 *     k slowest, halo 3 in x (and y when ny > 1), row pitch a multiple of 32 elements, element
 *     (0,0,0) at offset 8 + hy*pitch; horizontally uniform base fields are stored 1D (one value
 *     per level, src/core/field.hpp:145-191). cw_field_layout reports it for every field.
 */
#ifndef CW_DYCORE_H
#define CW_DYCORE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Lateral boundary kinds, cppwrf::BC (src/core/grid.hpp:19). */
enum cw_bc { CW_BC_PERIODIC = 0, CW_BC_SYMMETRIC = 1, CW_BC_SPECIFIED = 2, CW_BC_OPEN = 3 };

/* Arithmetic of a handle: CW_FP64 is the plain form, bit-identical to the reference CPU FP64 build;
 * CW_MIXED keeps the bulk stencils in FP32 and the column solves / sums in FP64. */
enum cw_precision { CW_FP64 = 0, CW_MIXED = 1 };

/* cppwrf::Grid (src/core/grid.hpp:21-55): mass points nx, ny, nz (ny = 1: 2-D x-z). */
typedef struct cw_grid {
  int nx, ny, nz;
  double dx, dy, dt, ztop, p_top;
  int bc_x, bc_y; /* enum cw_bc */
} cw_grid;

/* Namelist options of the dynamics step, as cases::Model::build maps them (src/cases/model.cpp:255-345). */
typedef struct cw_options {
  /* LargeStepParams (src/dyn/large_step.hpp:14-22) */
  double khdif, kvdif, pr_inv;
  int top_lid, h_adv_order, v_adv_order, w_damping;
  double w_crit_cfl;
  /* AcousticParams (src/dyn/rk3.hpp:19-25) */
  double epssm, smdiv, emdiv;
  int damp_opt, hypsometric_opt;
  double zdamp, dampcoef;
  int time_step_sound; /* 0: RK3::auto_sound_steps (src/dyn/rk3.cpp:69-72) */
  /* ScalarParams (src/dyn/scalars.hpp:14-19) */
  int moist_adv_opt, scalar_adv_opt, tke_adv_opt;
  /* DiffusionConfig (src/dyn/diffusion_driver.hpp:24-51): diff_opt 0, or 1 with km_opt 1 (constant K) or 4 (2-D
     Smagorinsky, c_s 0.25) */
  int diff_opt, km_opt;
  /* State / BaseState shape: flat = horizontally uniform base state (1-D storage, BaseState::flat) */
  int flat;
  int n_moist;   /* moist species (they come first among the scalars, State::add_scalar) */
  int n_scalars; /* moist species + passive tracers */
  int lbc;       /* 1: a LateralBC is attached (RK3::set_lateral_bc, width 5 / spec 1 / relax 4) */
  int precision; /* enum cw_precision */
  /* PhysicsParams (src/dyn/physics_coupling.hpp:23-35): 0 none, 1 Kessler (species 0, 1, 2 are qv, qc, qr),
   * run after the RK3 loop as solve_em does (src/dyn/rk3.cpp:146-158) */
  int mp_physics;
  double mp_tend_lim; /* K/s, limit on the microphysics heating rate */
  /* DiffusionConfig (src/dyn/diffusion_driver.hpp:42-43): sixth-order horizontal filter at the first RK stage,
   * 0 off, 1 linear, 2 flux-limited (monotonic); its factor */
  int diff_6th_opt;
  double diff_6th_factor;
  /* BaseState::coriolis (src/dyn/state.hpp:107, set with nonzero f0 / e0, src/cases/model.cpp:108-113): the Coriolis
   * terms of the u, v, w tendencies from the fields CW_F, CW_E, CW_SINA, CW_COSA */
  int coriolis;
  /* BaseState::mapped (src/dyn/state.hpp:97, :67-73): the map factors and CW_F, CW_E, CW_SINA, CW_COSA vary in the
   * horizontal (2-D storage instead of one value; a real-data projection); adds the curvature terms of u and v from
   * the map factors' gradients, and the Coriolis terms */
  int mapped;
} cw_options;

/* Fills o with the reference defaults (the values Model::build takes when a key is absent). */
int cw_default_options(cw_options* o);

/* Vertical coordinate: BaseState's 1-D arrays and scalars (src/dyn/state.hpp:108-115), sizes
 * nz (mass levels) or nz + 1 (w levels) as noted. The caller computes them (BaseState::set_levels,
 * src/dyn/state.cpp:86-116, or cw_levels_from_eta below). */
typedef struct cw_vertical {
  const double *znu, *dnw, *rdnw, *c1h, *c2h, *c3h, *c4h;          /* nz */
  const double *znw, *dn, *rdn, *fnm, *fnp, *c1f, *c2f, *c3f, *c4f; /* nz + 1 */
  const double *u_base, *v_base, *t_base, *qv_base_1d, *z_base;    /* nz (may be NULL: zero) */
  double cf1, cf2, cf3, cfn, cfn1, rdx, rdy, p_top, t0;
} cw_vertical;

/* Field identifiers: State (src/dyn/state.hpp:30-78), Tendencies (:80-90), BaseState (:92-119).
 * Scalars take an index n (0 .. n_scalars-1). */
enum cw_field {
  CW_U_1 = 0, CW_U_2, CW_V_1, CW_V_2, CW_W_1, CW_W_2, CW_T_1, CW_T_2, CW_PH_1, CW_PH_2, CW_MU_1, CW_MU_2,
  CW_P, CW_AL, CW_ALT, CW_PHP, CW_WW, CW_MUT, CW_MUU, CW_MUV, CW_MUTS, CW_MUUS, CW_MUVS, CW_RU, CW_RV, CW_RW,
  CW_RU_M, CW_RV_M, CW_WW_M, CW_CQU, CW_CQV, CW_CQW, CW_H_DIABATIC,
  CW_RU_TEND, CW_RV_TEND, CW_RW_TEND, CW_T_TEND, CW_PH_TEND, CW_MU_TEND,
  CW_RU_TENDF, CW_RV_TENDF, CW_RW_TENDF, CW_T_TENDF, CW_PH_TENDF,
  CW_MUB, CW_PB, CW_ALB, CW_T_INIT, CW_QV_BASE, CW_PHB, CW_HT,
  CW_MSFTX, CW_MSFTY, CW_MSFUX, CW_MSFUY, CW_MSFVX, CW_MSFVY, CW_MSFVX_INV, CW_F, CW_E, CW_SINA, CW_COSA,
  CW_RAINNC, CW_RAINNCV, /* PhysicsCoupling::rainnc, rainncv (physics_coupling.hpp:54): grid-scale rain [mm] */
  CW_Q_1, CW_Q_2, CW_Q_TENDF, /* with index n */
  CW_NFIELDS
};

/* A field's storage, cppwrf::Layout (src/core/field.hpp:46-64). Element (i,j,k) is at
 * offset + i*si + j*sj + k*sk of an allocation of total elements. stagger: 'M','U','V','W'. */
typedef struct cw_layout {
  int nx, ny, nz, rank, uniform;
  char stagger;
  int64_t si, sj, sk, offset, total;
  int wi0, wi1, wj0, wj1;
} cw_layout;

/* Lateral boundary slabs, LateralBC::Var / Side (src/dyn/lateral_bc.hpp:30-31). */
enum cw_lbc_var { CW_LBC_U = 0, CW_LBC_V, CW_LBC_T, CW_LBC_PH, CW_LBC_MU };
enum cw_lbc_side { CW_XS = 0, CW_XE, CW_YS, CW_YE };

typedef struct cw_handle cw_handle;

/* Layout of a field of a grid without a handle: Layout::make (src/core/halo.cpp:12-48). */
int cw_layout_of(const cw_grid* g, const cw_options* o, int field, cw_layout* out);

/* RK3 ctor (src/dyn/rk3.hpp:36-37, rk3.cpp:48-56) together with the State, Tendencies and BaseState
 * allocation of cases::Model (src/cases/model.hpp:28-50): device-resident, zero-filled. */
int cw_create(const cw_grid* g, const cw_options* o, cw_handle** out);
/* ~RK3 and the Model's fields. */
int cw_destroy(cw_handle* h);
/* BaseState::set_levels + upload_levels (src/dyn/state.cpp:86-124): the 1-D vertical arrays. */
int cw_set_vertical(cw_handle* h, const cw_vertical* v);
/* FieldT::fill_host / download (src/core/field.hpp:119-129): copies a field's whole allocation
 * (halo included, Layout order) from / to host memory; count = layout.total. */
int cw_upload(cw_handle* h, int field, int n, const double* host, size_t count);
int cw_download(cw_handle* h, int field, int n, double* host, size_t count);
/* The same for several fields in one call (FieldT::fill_host / download of each of nf fields, src/core/field.hpp:
 * 119-129): fields[i], ns[i] (species index for CW_Q_*), host[i], counts[i]. The copies are queued on the handle's
 * stream with one synchronisation: cw_upload_fields returns before they finish, in order with the next cw_step, so
 * its host buffers must not change before the next synchronising call (cw_download_fields, cw_download, cw_sync);
 * cw_download_fields returns when every field has arrived. Pinned host memory makes the copies asynchronous. */
int cw_upload_fields(cw_handle* h, int member, int nf, const int* fields, const int* ns, const double* const* host,
                     const size_t* counts);
int cw_download_fields(cw_handle* h, int member, int nf, const int* fields, const int* ns, double* const* host,
                       const size_t* counts);
/* The same for the points of each field's window only (its domain and halo, the points a step reads and writes;
 * FieldT's allocation also holds row padding, which no computation reads): one strided copy per field, about a
 * fifth fewer bytes than the whole allocations. The host arrays keep the layout; their padding is neither read nor
 * written (the device's padding holds zeros after an upload in the mixed form, and is left as it was in FP64). */
int cw_upload_windows(cw_handle* h, int member, int nf, const int* fields, const int* ns, const double* const* host,
                      const size_t* counts);
int cw_download_windows(cw_handle* h, int member, int nf, const int* fields, const int* ns, double* const* host,
                        const size_t* counts);
/* The field's layout (FieldT::layout, src/core/field.hpp:107). */
int cw_field_layout(cw_handle* h, int field, int n, cw_layout* out);
/* The device address of element (0,0,0) of a field (FieldT::data, src/core/field.hpp:108). */
int cw_field_device_ptr(cw_handle* h, int field, int n, void** out);
/* LateralBC::set / set_scalar (src/dyn/lateral_bc.hpp:42-44): values and tendencies of one
 * variable and side, (pos, k, b) with pos fastest, b = 0 the outermost row. */
int cw_set_lbc(cw_handle* h, int var, int side, const double* values, const double* tends, size_t count);
int cw_set_lbc_scalar(cw_handle* h, int n, int side, const double* values, const double* tends, size_t count);
/* LateralBC::dtbc (src/dyn/lateral_bc.hpp:57): seconds since the start of the boundary interval. */
int cw_set_lbc_time(cw_handle* h, double dtbc);
/* RK3::step (src/dyn/rk3.hpp:52, rk3.cpp:86-170), nsteps times in a row on the handle's stream. */
int cw_step(cw_handle* h, int nsteps);
/* RK3::set_dt (src/dyn/rk3.hpp:45, rk3.cpp:79-84). */
int cw_set_dt(cw_handle* h, double dt, int n_sound);
/* RK3::n_sound (src/dyn/rk3.hpp:43). */
int cw_n_sound(cw_handle* h, int* out);
/* The stream the handle launches on (cuda_stream_raw, src/core/backend.cpp:73-81); NULL = its own. */
int cw_set_stream(cw_handle* h, void* cuda_stream);
/* dev_sync + fatal_check (src/core/backend.hpp:745-769): waits for the handle's work and reports a
 * device-side error status: a CUDA error, or the handle's status word (a kernel whose bounded wait for its
 * tensor-memory copies ran out, about a second, left its part of the step undone; the word is cleared). */
int cw_sync(cw_handle* h);
/* Self-test of the kernels' bounded waits (no reference counterpart): one block waits on a shared-memory barrier
 * that nothing completes, gives up after `cycles` SM clock cycles (<= 0: the kernels' own limit, about a second) and
 * sets the status word, so that the next cw_sync fails with its message and clears it; the handle stays usable. */
int cw_selftest_wait(cw_handle* h, long long cycles);
/* The last error message of h (or of the last failed cw_create when h is NULL). */
const char* cw_last_error(cw_handle* h);
/* Kernel launches of the last cw_step call (the count this library issued). */
int cw_launch_count(cw_handle* h, long long* out);

/* Per-kernel device time of nsteps steps run without the graph, with CUDA events around every launch
 * (the reference's CPPWRF_KTIME table, src/core/backend.cpp:26-65); the steps advance the state.
 * cw_profile_entry returns kernel idx (0 .. *nkernels-1): its name, total milliseconds and launches. */
int cw_profile(cw_handle* h, int nsteps, int* nkernels);
int cw_profile_entry(cw_handle* h, int idx, char* name, int len, double* ms, long long* launches);
/* cudaSetDevice for the calling host thread before cw_create (one process per GPU, or a thread per GPU). */
int cw_use_device(int device);
/* CUDA-graph replay of the step (StepScope, src/core/backend.hpp:381-399): on by default. */
int cw_set_graph(cw_handle* h, int on);

/* ---- batches: several domains of uneven sizes in one handle, advanced together by the same launches
 * (no reference counterpart: CPPWRF advances domains one after the other, src/cases/nest_driver.cpp:871).
 * Members share the precision and the acoustic step count; member i's fields are addressed by the
 * cw_member_* variants of the single-domain calls above (cw_upload is cw_member_upload of member 0). */
int cw_batch_create(int n, const cw_grid* g, const cw_options* o, cw_handle** out);
int cw_members(cw_handle* h, int* out);
/* Members joining and leaving a batch (continuous batching of the served form; no reference counterpart).
 * n = 0 in cw_batch_create makes an empty batch whose precision is o[0].precision. cw_batch_add allocates
 * a new member (its fields zeroed, map factors 1) as the last index; cw_batch_remove frees one member and
 * moves the members after it down by one index. Both rebuild the handle's tables; the next cw_step captures
 * the step again. cw_step on an empty batch does nothing. */
/* Non-finite detection (CPPWRF's run.check_nonfinite_every_step, tests/robustness/run_test.sh:51-64): scans the
 * interior of member's prognostic state (U_2 V_2 W_2 T_2 PH_2 MU_2 P AL, then Q_2 of each species) and returns 0
 * when every value is finite (field = -1), 1 with the first non-finite value's field id, species n and point
 * (i, j, k) in that order of fields and then k, j, i, < 0 on error. It synchronizes the handle's stream. */
int cw_check_finite(cw_handle* h, int member, int* field, int* n, int* i, int* j, int* k);
/* Self-check of the device arithmetic the flux statement functions rely on (no counterpart in the reference: its
 * CPU build divides): the division by the constants 60 and 12 without a divide instruction (cw_div_const) against the
 * IEEE division __ddiv_rn on n operands per constant drawn from seed (random bit patterns over every exponent,
 * quotients next to a rounding midpoint, exact quotients and their neighbours), on the current device. */
int cw_check_div_const(unsigned long long n, unsigned long long seed, unsigned long long* checked,
                       unsigned long long* mismatches);
/* Block-shape autotuning (no reference counterpart). With on = 1 the next six cw_step steps run every tunable kernel
 * in one of its shapes -- a point kernel's block of 0: 128 x 1, 1: 64 x 2, 2: 32 x 4 points along i x j, a column
 * kernel's 0: 8, 1: 16, 2: 4 warps per column block -- two steps per shape (orders 0 1 2, then 2 1 0), timed per
 * launch; afterwards each kernel keeps its fastest shape and the step is captured again. The tuning steps are ordinary steps: every shape computes the same values. Calling it
 * again re-tunes. cw_autotune_choice gives a kernel's chosen shape (-1 before the tuning has finished). */
int cw_set_autotune(cw_handle* h, int on);
/* LargeStep::cfl_max (src/dyn/large_step.cpp:865-877), the maxima behind RK3::on_cfl (rk3.hpp) that the reference's
 * adaptive time step (src/cases/adapt_timestep.cpp) and w_damp read: with on = 1 every step records, after each RK
 * stage's tendencies, the largest vertical and horizontal Courant numbers of levels 1 .. nz-1 (a small reduction
 * launch per stage; the step is captured again). cw_cfl_max gives a member's values of the last step, stages 1..3. */
int cw_set_cfl_diagnostics(cw_handle* h, int on);
int cw_cfl_max(cw_handle* h, int member, double vert[3], double horiz[3]);
int cw_autotune_choice(cw_handle* h, const char* kernel, int* shape);
int cw_batch_add(cw_handle* h, const cw_grid* g, const cw_options* o, int* member);
int cw_batch_remove(cw_handle* h, int member);
/* Moves the one domain of handle `single` (made with cw_create and filled, e.g. on another thread while the
 * batch steps) into the batch as its last member, without copying its fields; `single` is left empty (destroy
 * it). Same precision and acoustic step count as the batch's members. */
int cw_batch_adopt(cw_handle* h, cw_handle* single, int* member);
/* The reverse of cw_batch_adopt: moves member `member` out of the batch into a new single-domain handle (*out,
 * with its own stream) without copying its fields, so that it can be read back on another thread while the batch
 * steps on; the members after it move down by one. Destroy *out with cw_destroy. (No counterpart in the
 * reference, which runs one domain per RK3 object.) */
int cw_batch_release(cw_handle* h, int member, cw_handle** out);
/* Device bytes one domain takes in a handle (fields, work fields, scalars, slabs, vertical arrays): the
 * footprint the served form admits by. Needs no device. */
int cw_footprint(const cw_grid* g, const cw_options* o, size_t* bytes);
/* The grid and options a member was made with. */
int cw_member_config(cw_handle* h, int member, cw_grid* g, cw_options* o);
int cw_member_set_vertical(cw_handle* h, int member, const cw_vertical* v);
int cw_member_upload(cw_handle* h, int member, int field, int n, const double* host, size_t count);
int cw_member_download(cw_handle* h, int member, int field, int n, double* host, size_t count);
int cw_member_field_layout(cw_handle* h, int member, int field, int n, cw_layout* out);
int cw_member_set_lbc(cw_handle* h, int member, int var, int side, const double* values, const double* tends,
                      size_t count);
int cw_member_set_lbc_scalar(cw_handle* h, int member, int n, int side, const double* values, const double* tends,
                             size_t count);
int cw_member_set_lbc_time(cw_handle* h, int member, double dtbc);

/* ---- host-side inputs ----
 * A cw_case holds one domain's complete input in host memory, in the same layouts as the handle's
 * fields: State, BaseState, the vertical arrays and the boundary slabs. The generators fill it from a
 * seed; cw_upload_case copies it into a handle (the Model set-up, src/cases/model.cpp:71-179). It
 * needs no GPU. */
typedef struct cw_case cw_case;
int cw_case_create(const cw_grid* g, const cw_options* o, cw_case** out);
int cw_case_destroy(cw_case* c);
/* a deep copy of a case; the grid and options a case was made for */
int cw_case_clone(const cw_case* c, cw_case** out);
int cw_case_config(const cw_case* c, cw_grid* g, cw_options* o);
/* host array of a field (the whole allocation) and its layout */
int cw_case_field(cw_case* c, int field, int n, double** data, cw_layout* layout);
int cw_case_vertical(cw_case* c, cw_vertical* out);
/* boundary slabs of a variable (is_scalar = 0, var = enum cw_lbc_var) or scalar n (is_scalar = 1) */
int cw_case_lbc(cw_case* c, int is_scalar, int var, int side, double** values, double** tends, size_t* count);
int cw_case_lbc_time(cw_case* c, double* dtbc);
int cw_upload_case(cw_handle* h, cw_case* c);
int cw_member_upload_case(cw_handle* h, int member, cw_case* c);

/* Idealized cases of CPPWRF (cases::make_case, src/cases/cases.cpp:90-192, and cases::initialize,
 * :224-287, with make_eta_levels "uniform_z", :194-201, and the base profiles of model.cpp:149-177).
 * kind: CW_IDEAL_REST_STATE (theta0 exp(N^2 z / g), uniform u0), CW_IDEAL_STRAKA (cold bubble),
 * CW_IDEAL_WARM_BUBBLE (Bryan-Fritsch thermal), CW_IDEAL_IGW (Skamarock-Klemp gravity wave).
 * Parameters left at CW_DEFAULT take the reference's defaults for the kind. */
enum cw_ideal_kind { CW_IDEAL_REST_STATE = 0, CW_IDEAL_STRAKA = 1, CW_IDEAL_WARM_BUBBLE = 2, CW_IDEAL_IGW = 3,
                     CW_IDEAL_SQUALL2D = 4 };
#define CW_DEFAULT (-1.0e300)
typedef struct cw_ideal_params {
  int kind;
  double theta0, n_bv, u0, xc, zc, xr, zr, amplitude, radius, a, p_surf;
} cw_ideal_params;
int cw_default_ideal_params(cw_ideal_params* p, int kind);
int cw_gen_ideal(cw_case* c, const cw_ideal_params* p);

/* Limited-area case: terrain, hybrid sigma-pressure coordinate, moist species, specified boundaries
 * relaxed toward the initial state; all randomness from seed. */
typedef struct cw_lam_params {
  uint64_t seed;
  double t_surf, lapse, t_strat, p_surf, hill_height, hill_halfwidth, orog_max, u_mean, u_pert, rh_mean, rh_pert,
      q_patch_max, theta_pert, wind_pert, etac;
  int hybrid_opt;
} cw_lam_params;
int cw_default_lam_params(cw_lam_params* p);
int cw_gen_lam(cw_case* c, const cw_lam_params* p);

/* ---- one domain decomposed into px x py patches (tile::Options, src/core/tiles.hpp:22-120; docs/MPI.md §3) ----
 * Patch t = tx + px ty owns the mass points [tx nx / px, (tx + 1) nx / px) x [ty ny / py, (ty + 1) ny / py) and the
 * faces between them; the east / north edge patches also own the faces nx / ny and the lateral halos beyond the
 * domain's edges (tile::set_domain, tiles.hpp:70-74). Each patch is a member of the handle whose fields are allocated
 * for its patch and a halo of 3 and indexed with the domain's indices (Grid::dom, pi0 .. pj1); every launch covers
 * every patch and is clipped to the points each owns, and at every halo fill point each patch first receives the
 * points of its allocation that other patches own (the exchange), then fills the domain's halo where it touches the
 * domain's edge, as core/halo.cpp:120-140 does. The result equals the undecomposed domain's bit for bit. Here the
 * patches share the handle's device and stream. Refused: a periodic direction split over several patches, a split
 * along y of a 2-D domain, patches under 6 x 6 points. */
int cw_decomp_patch(const cw_grid* g, int px, int py, int t, int box[4]); /* i0, i1, j0, j1 of patch t (no device) */
int cw_decomp_create(const cw_grid* g, const cw_options* o, int px, int py, cw_handle** out);
/* A field as one whole-domain array (the layout of cw_layout_of): uploaded into every patch's allocation, or
 * gathered from the points each patch owns (tile::download, tiles.hpp:84-97). */
int cw_decomp_upload(cw_handle* h, int field, int n, const double* host, size_t count);
int cw_decomp_download(cw_handle* h, int field, int n, double* host, size_t count);
/* cw_upload_case into every patch (vertical arrays, each patch's window of the fields, the boundary slabs). */
int cw_decomp_upload_case(cw_handle* h, cw_case* c);

/* ---- the patches of one domain over several processes, one GPU each (tiles_mpi.cpp:35-64: the ranks of
 * docs/MPI.md §3 with NCCL in place of MPI) ----
 * Patch t belongs to rank t % nranks (one patch per rank when nranks = px py, the reference's layout). Each rank's
 * handle holds its patches; at every fill point each rank packs the points that other ranks' patches receive into
 * one send buffer on its GPU (one segment per receiving rank), the segments cross as NCCL point-to-point transfers
 * grouped on the handle's stream (captured into the step's CUDA graph with the kernels), and each rank unpacks its
 * receive buffer into its patches' halos, then exchanges between its own patches and fills the domain's halo, as
 * cw_decomp_create does on one device. The boxes of a pair of ranks are listed in one order by both (receiving
 * patch, owning patch, field) and no device reads another's memory. Every rank makes the same calls in the same
 * order: cw_decomp_create_ranked (collective: NCCL's communicator), cw_step, cw_destroy.
 * cw_decomp_upload / _upload_case take the whole-domain arrays on every rank (each keeps its patches' windows);
 * cw_decomp_download gives the points this rank's patches own (the others 0: the ranks' arrays sum to the domain).
 * nccl_id: 128 bytes from cw_nccl_unique_id on one rank, passed to all (e.g. by torch.distributed). nccl_id = NULL
 * is the loopback form: this process holds every patch and the exchanges between patches of different ranks go
 * through the packed buffers with a device copy in place of the transfer (the whole path on one GPU but NCCL). */
int cw_nccl_unique_id(unsigned char id[128]);
int cw_decomp_create_ranked(const cw_grid* g, const cw_options* o, int px, int py, int rank, int nranks,
                            const unsigned char* nccl_id, cw_handle** out);
/* The fill point indices of cw_decomp_plan (the halo refreshes of one RK3 step, src/dyn/rk3.cpp:86-170). */
enum { CW_FILL_MU1, CW_FILL_PREP0, CW_FILL_PREP1, CW_FILL_SS0, CW_FILL_UV, CW_FILL_AC, CW_FILL_POST, CW_FILL_FIN,
       CW_FILL_Q1PD, CW_FILL_SCPD, CW_FILL_Q2, CW_FILL_END_P, CW_FILL_WS0, CW_FILL_WS1, CW_FILL_MP, CW_FILL_MP_P,
       CW_FILL_XK };
/* The boxes that cross between rank `rank` and the others at the fill point made of the nsets fill points `sets`,
 * as that rank packs and unpacks them (no device): n boxes, 11 values each into out (up to cap boxes): role (0: this
 * rank packs it, 1: unpacks it), peer rank, receiving patch, owning patch, field (its id; 1000 + a work field,
 * 2000 + n: q_2 of species n, 3000 + n: q_1, 4000 + n: the PD scale), i0, i1, j0, j1, levels, element offset in the
 * send (role 0) or receive (role 1) region. The segment of a peer is its boxes' points in list order, each box's
 * points i fastest, then j, then k. For a transport of the caller's own, and for tests. */
int cw_decomp_plan(const cw_grid* g, const cw_options* o, int px, int py, int rank, int nranks, int nsets,
                   const int* sets, long long* out, int cap, int* n);
/* cw_download without any allocation (no counterpart in the reference; CPPWRF's FieldT::download always
 * stages through host memory).
 *
 * For callers that must read a field back at a moment when they cannot allocate: a checkpoint or state
 * dump taken after a host or device allocation has failed, or a serving loop whose device-memory budget is
 * fully committed to resident domains. cw_download stages an FP32 field (CW_MIXED handles) through a host
 * vector; this call widens it to double on the device, in a scratch array that is part of the library's
 * device image (CW_NOALLOC_SCRATCH_DOUBLES doubles = 8 MiB per device, not allocated at run time), and
 * copies that to `host`. FP64 fields are copied directly and have no size limit.
 *
 * Same arguments and result as cw_download (member 0 of the handle, the whole allocation of the field,
 * count = its layout's total). Call it with the handle's device current (another current device returns
 * CW_NOALLOC_EBADARG). The first call on each device looks up the scratch's device address
 * (cudaGetSymbolAddress), which may load the library's device code on that device: make one call early,
 * before the period in which nothing may be set up. The looked-up address is kept for the life of the
 * process and does not survive cudaDeviceReset (which unloads the library's device code): after a reset,
 * handles are gone anyway, and this call must not be used again in that process. No part of the scratch
 * has to start at zero: each call writes the count elements it then copies. An error left pending by an
 * earlier asynchronous launch is reported as CW_NOALLOC_ECUDA and left in place for its owner.
 *
 * The scratch is shared by every handle on a device: two calls that overlap in time (from two threads, or
 * on two streams before the first has returned) race on it, so callers serialize them. The call returns
 * after the copy has completed (it synchronizes the handle's stream). Errors are returned, not stored in
 * cw_last_error (storing a message could allocate):
 *   CW_NOALLOC_EBADARG  null handle or buffer, unknown field, species out of range, count != layout total,
 *                       or a current device other than the handle's
 *   CW_NOALLOC_ETOOBIG  an FP32 field of more than CW_NOALLOC_SCRATCH_DOUBLES elements (nothing is copied)
 *   CW_NOALLOC_ECUDA    a CUDA call failed */
#define CW_NOALLOC_SCRATCH_DOUBLES 1048576
#define CW_NOALLOC_EBADARG (-1)
#define CW_NOALLOC_ETOOBIG (-2)
#define CW_NOALLOC_ECUDA (-3)
int cw_download_noalloc(cw_handle* h, int field, int n, double* host, size_t count);

#ifdef __cplusplus
}
#endif

#endif /* CW_DYCORE_H */
