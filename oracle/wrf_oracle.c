/* SPDX-License-Identifier: GPL-3.0-or-later
 *
 * TEST INFRASTRUCTURE ONLY (see wrf_oracle.h): a sequential C restatement of CPPWRF's RK3 dynamics
 * step, used as the parity checker of the CUDA path and as the timed CPU baseline. Every function
 * names the reference code it restates (paths relative to the CPPWRF source tree). Each point
 * formula keeps the reference's statement and summation order (IEEE double, no FMA contraction:
 * compile with -ffp-contract=off), so a difference in a single bit is a real difference.
 *
 * Scope: the options of the dynamics step that the benchmark cases use -- 2-D (ny = 1) and 3-D,
 * periodic / symmetric / specified / open lateral boundaries, flat or terrain base state, any hybrid
 * coefficients, moist species (calc_cq, positive-definite scalar advection at rk 3), passive
 * tracers, constant-K diffusion (diff_opt 1, km_opt 1), specified lateral boundaries (width 5),
 * top_lid, w_damping, h/v_adv_order 5/6, 3/4, damp_opt 2 and 3 (sin by the pow mode: glibc's or cw_sin), the
 * sixth-order filter, hypsometric_opt 1 and 2 (log by the pow mode), damp_opt 1 (cos by the pow mode), Kessler
 * microphysics, the Coriolis terms, horizontally varying map factors with their curvature terms (BaseState::mapped).
 */
#include "wrf_oracle.h"

#include <immintrin.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../cppwrf_b200/csrc/cw_pow.h"

/* glibc's libmvec 2-lane pow, the reference CPU build's vm::pow (src/core/backend.hpp:118, :171) */
extern __m128d _ZGVbN2vv_pow(__m128d, __m128d);
extern __m128d _ZGVbN2v_exp(__m128d);
extern __m128d _ZGVbN2v_log(__m128d);
extern __m128d _ZGVbN2v_cos(__m128d);

/* ------------------------------------------------------------------ constants
 * src/core/constants.hpp:4-18 (WRF module_model_constants) */
#define G_ 9.81
#define R_D 287.0
#define CP (7.0 * R_D / 2.0)
#define CV (CP - R_D)
#define CPOVCV (CP / (CP - R_D))
#define P1000MB 100000.0
#define T0 300.0
#define H 0.5
#define Q 0.25
#define RERADIUS (1. / 6370.0e03)
#define CB 25.0 /* phase speed of the open (radiative) lateral boundaries, cst::cb */

/* ------------------------------------------------------------------ storage */
typedef struct {
  double* a; /* allocation */
  double* p; /* element (0,0,0) */
  long si, sj, sk;
  cw_layout L;
} fld;

#define AT(f, i, j, k) ((f)->p[(long)(i) * (f)->si + (long)(j) * (f)->sj + (long)(k) * (f)->sk])

enum { ST_M = 'M', ST_U = 'U', ST_V = 'V', ST_W = 'W' };

typedef struct {
  double* d; /* values (4 sides) then tendencies (4 sides) */
  size_t off[8];
  int npos[4], nk;
  int have;
} slabset;

struct or_dom {
  cw_grid g;
  cw_options o;
  int n_sound;
  int pow_mode;
  fld f[CW_NFIELDS];
  fld *q1, *q2, *qtf; /* n_scalars each */
  /* SmallStep's fields (src/dyn/small_step.hpp:45-49) */
  fld u_save, v_save, w_save, t_save, ph_save, ww1, c2a, pm1, t_2save, a, alpha, gamma, mu_save, mudf, muave, w_rhs,
      t2a, dvdxi;
  /* DiffusionDriver's eddy viscosities (src/dyn/diffusion_driver.hpp:76) */
  fld xkmh, xkmv, xkhh, xkhv;
  /* ScalarTransport::Work per species (src/dyn/scalars.hpp:47-51) */
  fld *q_new, *scale, *dhx, *lox, *dhy, *loy, *dhz, *loz;
  /* BaseState 1-D arrays (src/dyn/state.hpp:110-115) */
  double *znu, *znw, *dnw, *dn, *rdnw, *rdn, *fnm, *fnp, *c1h, *c2h, *c3h, *c4h, *c1f, *c2f, *c3f, *c4f, *u_base,
      *v_base, *t_base, *qv_base_1d, *z_base;
  double cf1, cf2, cf3, cfn, cfn1, rdx, rdy, p_top;
  /* LateralBC (src/dyn/lateral_bc.hpp:28-91) */
  slabset lbc[5];
  slabset* lbcq; /* per scalar */
  double dtbc, fcx[5], gcx[5];
  double cfl[6]; /* LargeStep::cfl_max of each RK stage of the last step: (vertical, horizontal) */
  char err[256];
};

static void set_err(or_dom* d, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(d->err, sizeof d->err, fmt, ap);
  va_end(ap);
}

/* ------------------------------------------------------------------ grid (src/core/grid.hpp:35-54) */
static int two_d(const cw_grid* g) { return g->ny == 1; }
static int hy_of(const cw_grid* g) { return two_d(g) ? 0 : 3; }
static int nxs(const cw_grid* g, char s) { return s == ST_U ? g->nx + 1 : g->nx; }
static int nys(const cw_grid* g, char s) { return (s == ST_V && !two_d(g)) ? g->ny + 1 : g->ny; }
static int nzs(const cw_grid* g, char s) { return s == ST_W ? g->nz + 1 : g->nz; }
static int flat_x(const cw_grid* g) { return g->bc_x == CW_BC_SPECIFIED || g->bc_x == CW_BC_OPEN; }
static int flat_y(const cw_grid* g) { return g->bc_y == CW_BC_SPECIFIED || g->bc_y == CW_BC_OPEN; }
static int specified(const cw_grid* g) { return g->bc_x == CW_BC_SPECIFIED || g->bc_y == CW_BC_SPECIFIED; }

/* Layout::make (src/core/halo.cpp:12-48), whole domain */
static cw_layout layout_make(const cw_grid* g, char s, int rank, int uniform) {
  cw_layout L;
  memset(&L, 0, sizeof L);
  L.nx = nxs(g, s);
  L.ny = nys(g, s);
  L.nz = rank == 3 ? nzs(g, s) : 1;
  L.rank = rank;
  L.uniform = uniform;
  L.stagger = s;
  if (uniform) {
    L.si = 0;
    L.sj = 0;
    L.sk = rank == 3 ? 1 : 0;
    L.offset = 0;
    L.total = L.nz;
    return L;
  }
  const int hy = hy_of(g);
  L.wi0 = -3;
  L.wi1 = L.nx + 3;
  L.wj0 = -hy;
  L.wj1 = L.ny + hy;
  const long pitch = (8 + (L.wi1 - L.wi0 - 3) + 31) / 32 * 32;
  L.si = 1;
  L.sj = two_d(g) ? 0 : pitch;
  const long plane = pitch * (L.wj1 - L.wj0);
  L.sk = rank == 3 ? plane : 0;
  L.offset = 8 - (L.wi0 + 3) - (long)L.wj0 * L.sj;
  L.total = plane * (rank == 3 ? L.nz : 1);
  return L;
}

static void fld_alloc(fld* f, const cw_grid* g, char s, int rank, int uniform) {
  f->L = layout_make(g, s, rank, uniform);
  f->a = (double*)calloc((size_t)f->L.total, sizeof(double));
  f->p = f->a + f->L.offset;
  f->si = f->L.si;
  f->sj = f->L.sj;
  f->sk = f->L.sk;
}
static void fld_free(fld* f) {
  free(f->a);
  f->a = f->p = NULL;
}
static void fld_fill(fld* f, double v) {
  for (long n = 0; n < f->L.total; ++n) f->a[n] = v;
}

/* the stagger, rank and uniform flag of each cw_field (src/dyn/state.cpp:10-24, :67-84) */
static void field_kind(const cw_options* o, int id, char* s, int* rank, int* uniform) {
  *rank = 3;
  *uniform = 0;
  switch (id) {
    case CW_U_1: case CW_U_2: case CW_RU: case CW_RU_M: case CW_CQU: case CW_RU_TEND: case CW_RU_TENDF: *s = ST_U; break;
    case CW_V_1: case CW_V_2: case CW_RV: case CW_RV_M: case CW_CQV: case CW_RV_TEND: case CW_RV_TENDF: *s = ST_V; break;
    case CW_W_1: case CW_W_2: case CW_PH_1: case CW_PH_2: case CW_WW: case CW_RW: case CW_WW_M: case CW_CQW:
    case CW_RW_TEND: case CW_PH_TEND: case CW_RW_TENDF: case CW_PH_TENDF: *s = ST_W; break;
    case CW_MU_1: case CW_MU_2: case CW_MUT: case CW_MUTS: case CW_MU_TEND: case CW_RAINNC: case CW_RAINNCV:
      *s = ST_M; *rank = 2; break;
    case CW_MUU: case CW_MUUS: *s = ST_U; *rank = 2; break;
    case CW_MUV: case CW_MUVS: *s = ST_V; *rank = 2; break;
    case CW_MUB: case CW_HT: *s = ST_M; *rank = 2; *uniform = o->flat; break;
    case CW_PB: case CW_ALB: case CW_T_INIT: case CW_QV_BASE: *s = ST_M; *uniform = o->flat; break;
    case CW_PHB: *s = ST_W; *uniform = o->flat; break;
    case CW_MSFTX: case CW_MSFTY: case CW_F: case CW_E: case CW_SINA: case CW_COSA: *s = ST_M; *rank = 2; *uniform = !o->mapped; break;
    case CW_MSFUX: case CW_MSFUY: *s = ST_U; *rank = 2; *uniform = !o->mapped; break;
    case CW_MSFVX: case CW_MSFVY: case CW_MSFVX_INV: *s = ST_V; *rank = 2; *uniform = !o->mapped; break;
    default: *s = ST_M; break; /* M 3-D: t, p, al, alt, php, h_diabatic, t_tend, t_tendf, q */
  }
}

/* ------------------------------------------------------------------ halos
 * HaloLine (src/core/halo.cpp:52-88) and fill_impl (:93-117): x pass over the rows, then y over
 * the full x extent (corners), parities as HaloField / fill_halo's defaults. */
enum { EVEN = 0, ODD = 1, ODD_FACE = 2 };

static void halo_line(double* p, long sn, int n, int face, int periodic, int odd, int flat, int odd_face, int lo, int hi,
                      int a) {
  const int nl = face ? 4 : 3;
  const int i = a < nl ? (face ? -a : -1 - a) : n + (a - nl);
  if (i < lo || i >= hi) return;
  int src;
  if (flat) {
    const int last = face ? n : n - 1;
    src = i < 0 ? 0 : (i > last ? last : i);
  } else if (periodic) {
    src = ((i % n) + n) % n;
  } else if (face) {
    src = i <= 0 ? -i : 2 * n - i;
  } else {
    src = i < 0 ? -1 - i : 2 * n - 1 - i;
  }
  double v = p[src * sn];
  if (!periodic && !flat && src == i) {
    if (odd_face) p[i * sn] = -v;
    return;
  }
  if (!periodic && !flat && odd) v = -v;
  p[i * sn] = v;
}

static void fill_halo_p(or_dom* d, fld* f, int px, int py) {
  const cw_grid* g = &d->g;
  const cw_layout* L = &f->L;
  if (L->uniform) return;
  const int ux = L->stagger == ST_U, vy = L->stagger == ST_V;
  const int nk = L->nz;
  { /* x direction over the interior rows */
    const int na = ux ? 8 : 6;
    const int j0 = L->wj0 > 0 ? L->wj0 : 0, j1 = L->wj1 < L->ny ? L->wj1 : L->ny;
    for (int k = 0; k < nk; ++k)
      for (int a = 0; a < na; ++a)
        for (int j = j0; j < j1; ++j)
          halo_line(f->p + (long)j * f->sj + (long)k * f->sk, 1, g->nx, ux, g->bc_x == CW_BC_PERIODIC, px != EVEN,
                    flat_x(g), px == ODD_FACE, L->wi0, L->wi1, a);
  }
  if (two_d(g)) return;
  { /* y direction over the full x extent */
    const int na = vy ? 8 : 6;
    for (int k = 0; k < nk; ++k)
      for (int i = L->wi0; i < L->wi1; ++i)
        for (int a = 0; a < na; ++a)
          halo_line(f->p + i + (long)k * f->sk, f->sj, g->ny, vy, g->bc_y == CW_BC_PERIODIC, py != EVEN, flat_y(g),
                    py == ODD_FACE, L->wj0, L->wj1, a);
  }
}
/* fill_halo(f, g) / HaloField(f): U odd in x, V odd in y, the rest even; 2-D fields even */
static void fill_halo(or_dom* d, fld* f) {
  if (f->L.rank == 2) fill_halo_p(d, f, EVEN, EVEN);
  else fill_halo_p(d, f, f->L.stagger == ST_U ? ODD : EVEN, f->L.stagger == ST_V ? ODD : EVEN);
}

/* ------------------------------------------------------------------ flux library
 * src/dyn/kernels_common.hpp:11-105 (WRF module_advect_em.F statement functions) */
static double sgn1(double a) { return a >= 0.0 ? 1.0 : -1.0; }
static double flux5(double qm3, double qm2, double qm1, double q0, double qp1, double qp2, double ua, double up) {
  return (37.0 * (q0 + qm1) - 8.0 * (qp1 + qm2) + (qp2 + qm3)) / 60.0 -
         up * sgn1(ua) * ((qp2 - qm3) - 5.0 * (qp1 - qm2) + 10.0 * (q0 - qm1)) / 60.0;
}
static double flux3(double qm2, double qm1, double q0, double qp1, double ua, double up) {
  return (7.0 * (q0 + qm1) - (qp1 + qm2)) / 12.0 + up * sgn1(ua) * ((qp1 - qm2) - 3.0 * (q0 - qm1)) / 12.0;
}
static double flux5_pd(double qm3, double qm2, double qm1, double q0, double qp1, double qp2, double ua, double up) {
  const double f6 = (37. / 60.) * (q0 + qm1) - (2. / 15.) * (qp1 + qm2) + (1. / 60.) * (qp2 + qm3);
  return f6 - up * sgn1(ua) * (1. / 60.) * ((qp2 - qm3) - 5. * (qp1 - qm2) + 10. * (q0 - qm1));
}
static double flux3_pd(double qm2, double qm1, double q0, double qp1, double ua, double up) {
  const double f4 = (7. / 12.) * (q0 + qm1) - (1. / 12.) * (qp1 + qm2);
  return f4 + up * sgn1(ua) * (1. / 12.) * ((qp1 - qm2) - 3. * (q0 - qm1));
}
static int ord_face(int f, int n, int on) {
  if (!on) return 5;
  if (f <= 1 || f >= n - 1) return 2;
  if (f == 2 || f == n - 2) return 3;
  return 5;
}
static int ord_mass(int f, int n, int on) {
  if (!on) return 5;
  if (f <= 1 || f >= n) return 2;
  if (f == 2 || f == n - 1) return 3;
  return 5;
}
static double flux_upwind(double qm1, double q0, double cr) {
  const double a = cr < 0.0 ? -cr : cr;
  const double lo = cr + a, hi = cr - a;
  return 0.5 * (lo < 1.0 ? lo : 1.0) * qm1 + 0.5 * (hi > -1.0 ? hi : -1.0) * q0;
}

/* kern::Spec (kernels_common.hpp:33-45): x / y = degraded orders (specified or open), ox / oy = open (the boundary
 * cells are advected with the open terms), sx / sy = specified only (the outermost row is set from boundary data) */
typedef struct {
  int x, y, nx, ny, ox, oy, sx, sy;
} spec_t;
static int open_x(const cw_grid* g) { return g->bc_x == CW_BC_OPEN; }
static int open_y(const cw_grid* g) { return g->bc_y == CW_BC_OPEN && !two_d(g); }
static spec_t spec_of(const cw_grid* g) {
  spec_t s = {flat_x(g), flat_y(g) && !two_d(g), g->nx, g->ny, open_x(g), open_y(g), 0, 0};
  s.sx = s.x && !s.ox;
  s.sy = s.y && !s.oy;
  return s;
}

/* MoistCoef (kernels_common.hpp:98-104) */
static double cqu_(or_dom* d, int i, int j, int k) { return d->o.n_moist > 0 ? AT(&d->f[CW_CQU], i, j, k) : 1.0; }
static double cqv_(or_dom* d, int i, int j, int k) { return d->o.n_moist > 0 ? AT(&d->f[CW_CQV], i, j, k) : 1.0; }
static double cqw_(or_dom* d, int i, int j, int k) { return d->o.n_moist > 0 ? AT(&d->f[CW_CQW], i, j, k) : 0.0; }
static double cq1_(or_dom* d, int i, int j, int k) { return 1.0 / (1.0 + cqw_(d, i, j, k)); }

#define F_(id) (&d->f[id])

/* ------------------------------------------------------------------ LargeStep::prep
 * src/dyn/large_step.cpp:697-733 with KMu (:49-66), KPrep3 (:68-81), KWW (:83-108), KCq (:127-148) */
static double ww_mu_u(or_dom* d, int i, int j) {
  fld *mu = F_(CW_MU_2), *mub = F_(CW_MUB);
  return H * (AT(mu, i, j, 0) + AT(mub, i, j, 0) + AT(mu, i - 1, j, 0) + AT(mub, i - 1, j, 0));
}
static double ww_mu_v(or_dom* d, int i, int j) {
  fld *mu = F_(CW_MU_2), *mub = F_(CW_MUB);
  return H * (AT(mu, i, j, 0) + AT(mub, i, j, 0) + AT(mu, i, j - 1, 0) + AT(mub, i, j - 1, 0));
}
static double ww_divv(or_dom* d, int i, int j, int k) {
  fld *u = F_(CW_U_2), *v = F_(CW_V_2), *msftx = F_(CW_MSFTX), *msfuy = F_(CW_MSFUY), *mvi = F_(CW_MSFVX_INV);
  const double mu1 = ww_mu_u(d, i + 1, j), mu0 = ww_mu_u(d, i, j), mv1 = ww_mu_v(d, i, j + 1), mv0 = ww_mu_v(d, i, j);
  const double* c1h = d->c1h;
  const double* c2h = d->c2h;
  return AT(msftx, i, j, 0) * d->dnw[k] *
         (d->rdx * ((c1h[k] * mu1 + c2h[k]) * AT(u, i + 1, j, k) / AT(msfuy, i + 1, j, 0) -
                    (c1h[k] * mu0 + c2h[k]) * AT(u, i, j, k) / AT(msfuy, i, j, 0)) +
          d->rdy * ((c1h[k] * mv1 + c2h[k]) * AT(v, i, j + 1, k) * AT(mvi, i, j + 1, 0) -
                    (c1h[k] * mv0 + c2h[k]) * AT(v, i, j, k) * AT(mvi, i, j, 0)));
}

static void large_prep(or_dom* d) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz, nyv = nys(g, ST_V);
  fill_halo(d, F_(CW_U_2));
  fill_halo(d, F_(CW_V_2));
  fill_halo(d, F_(CW_W_2));
  fill_halo(d, F_(CW_T_2));
  fill_halo(d, F_(CW_PH_2));
  fill_halo(d, F_(CW_P));
  fill_halo(d, F_(CW_AL));
  if (!specified(g)) fill_halo(d, F_(CW_MU_2));
  fld *mu = F_(CW_MU_2), *mub = F_(CW_MUB), *mut = F_(CW_MUT), *muu = F_(CW_MUU), *muv = F_(CW_MUV);
  const int spx = flat_x(g), spy = flat_y(g) && !two_d(g);
  for (int j = 0; j < nyv; ++j)
    for (int i = 0; i < nx + 1; ++i) { /* KMu */
      if (i < nx && j < ny) AT(mut, i, j, 0) = AT(mu, i, j, 0) + AT(mub, i, j, 0);
      if (j < ny) {
        if (spx && i == 0)
          AT(muu, i, j, 0) = H * (AT(mu, 0, j, 0) + AT(mu, 0, j, 0) + AT(mub, 0, j, 0) + AT(mub, 0, j, 0));
        else if (spx && i == nx)
          AT(muu, i, j, 0) =
              H * (AT(mu, nx - 1, j, 0) + AT(mu, nx - 1, j, 0) + AT(mub, nx - 1, j, 0) + AT(mub, nx - 1, j, 0));
        else
          AT(muu, i, j, 0) = H * (AT(mu, i, j, 0) + AT(mu, i - 1, j, 0) + AT(mub, i, j, 0) + AT(mub, i - 1, j, 0));
      }
      if (i < nx && j < nyv) {
        if (spy && j == 0)
          AT(muv, i, j, 0) = H * (AT(mu, i, 0, 0) + AT(mu, i, 0, 0) + AT(mub, i, 0, 0) + AT(mub, i, 0, 0));
        else if (spy && j == ny)
          AT(muv, i, j, 0) =
              H * (AT(mu, i, ny - 1, 0) + AT(mu, i, ny - 1, 0) + AT(mub, i, ny - 1, 0) + AT(mub, i, ny - 1, 0));
        else
          AT(muv, i, j, 0) = H * (AT(mu, i, j, 0) + AT(mu, i, j - 1, 0) + AT(mub, i, j, 0) + AT(mub, i, j - 1, 0));
      }
    }
  fill_halo(d, mut);
  fld *u = F_(CW_U_2), *v = F_(CW_V_2), *w = F_(CW_W_2), *al = F_(CW_AL), *ph = F_(CW_PH_2);
  fld *alb = F_(CW_ALB), *phb = F_(CW_PHB), *msfuy = F_(CW_MSFUY), *mvi = F_(CW_MSFVX_INV), *msfty = F_(CW_MSFTY);
  fld *ru = F_(CW_RU), *rv = F_(CW_RV), *rw = F_(CW_RW), *alt = F_(CW_ALT), *php = F_(CW_PHP);
  for (int k = 0; k < nz + 1; ++k)
    for (int j = 0; j < nyv; ++j)
      for (int i = 0; i < nx + 1; ++i) { /* KPrep3 */
        if (j < ny && k < nz)
          AT(ru, i, j, k) = AT(u, i, j, k) * (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k]) / AT(msfuy, i, j, 0);
        if (i < nx && j < nyv && k < nz)
          AT(rv, i, j, k) = AT(v, i, j, k) * (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k]) * AT(mvi, i, j, 0);
        if (i < nx && j < ny)
          AT(rw, i, j, k) = AT(w, i, j, k) * (d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k]) / AT(msfty, i, j, 0);
        if (i < nx && j < ny && k < nz) {
          AT(alt, i, j, k) = AT(al, i, j, k) + AT(alb, i, j, k);
          AT(php, i, j, k) = H * (AT(phb, i, j, k) + AT(phb, i, j, k + 1) + AT(ph, i, j, k) + AT(ph, i, j, k + 1));
        }
      }
  fill_halo(d, ru);
  fill_halo(d, rv);
  fill_halo(d, rw);
  fill_halo(d, alt);
  fill_halo(d, php);
  fill_halo_p(d, muu, ODD_FACE, EVEN);
  fill_halo_p(d, muv, EVEN, ODD);
  fld* ww = F_(CW_WW);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) { /* KWW */
      double dmdt = 0;
      for (int k = 0; k < nz; ++k) dmdt += ww_divv(d, i, j, k);
      double wv = 0;
      AT(ww, i, j, 0) = 0;
      for (int k = 1; k < nz; ++k) {
        wv = wv - d->dnw[k - 1] * d->c1h[k - 1] * dmdt - ww_divv(d, i, j, k - 1);
        AT(ww, i, j, k) = wv;
      }
      AT(ww, i, j, nz) = 0;
    }
  fill_halo(d, ww);
  if (d->o.n_moist > 0) { /* KCq */
    fld *cqu = F_(CW_CQU), *cqv = F_(CW_CQV), *cqw = F_(CW_CQW);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < nyv; ++j)
        for (int i = 0; i < nx + 1; ++i) {
          if (j < ny) {
            double t = 0;
            for (int s = 0; s < d->o.n_moist; ++s) t = t + AT(&d->q2[s], i, j, k) + AT(&d->q2[s], i - 1, j, k);
            AT(cqu, i, j, k) = 1.0 / (1.0 + 0.5 * t);
          }
          if (i < nx && j < nyv) {
            double t = 0;
            for (int s = 0; s < d->o.n_moist; ++s) t = t + AT(&d->q2[s], i, j, k) + AT(&d->q2[s], i, j - 1, k);
            AT(cqv, i, j, k) = 1.0 / (1.0 + 0.5 * t);
          }
          if (i < nx && j < ny && k >= 1) {
            double t = 0;
            for (int s = 0; s < d->o.n_moist; ++s) t = t + AT(&d->q2[s], i, j, k) + AT(&d->q2[s], i, j, k - 1);
            AT(cqw, i, j, k) = 0.5 * t;
          }
        }
  }
}

/* ------------------------------------------------------------------ rk_tendency kernels
 * KTendU (large_step.cpp:152-264), KTendV (:267-376), KTendW (:379-499), KTendT (:502-565),
 * KTendPh (:570-668); LargeStep::tendencies (:798-861). */
typedef struct {
  or_dom* d;
  spec_t sp;
  double hup, vup;
  int nz, do_y, top_lid;
} tctx;

/* MapC::vxgm (:121-124): the curvature factor at mass point (i, j, k) from the uncoupled u, v and the map factors */
static double vxgm(or_dom* d, int i, int j, int k) {
  fld *u = F_(CW_U_2), *v = F_(CW_V_2), *msfvx = F_(CW_MSFVX), *msfuy = F_(CW_MSFUY);
  return H * (AT(u, i, j, k) + AT(u, i + 1, j, k)) * (AT(msfvx, i, j + 1, 0) - AT(msfvx, i, j, 0)) * d->rdy -
         H * (AT(v, i, j, k) + AT(v, i, j + 1, k)) * (AT(msfuy, i + 1, j, 0) - AT(msfuy, i, j, 0)) * d->rdx;
}

/* --- U --- */
static double tu_fx(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *u = F_(CW_U_2), *ru = F_(CW_RU);
  const int o = ord_mass(i, c->sp.nx, c->sp.x);
  if (o == 2) {
    if (i <= 1) {
      const double ub = (c->sp.sx && AT(u, i, j, k) < 0.0) ? AT(u, i, j, k) : AT(u, i - 1, j, k);
      return Q * (AT(ru, i, j, k) + AT(ru, i - 1, j, k)) * (AT(u, i, j, k) + ub);
    }
    const double ub = (c->sp.sx && AT(u, i - 1, j, k) > 0.0) ? AT(u, i - 1, j, k) : AT(u, i, j, k);
    return Q * (AT(ru, i, j, k) + AT(ru, i - 1, j, k)) * (AT(u, i - 1, j, k) + ub);
  }
  const double vel = H * (AT(ru, i, j, k) + AT(ru, i - 1, j, k));
  if (o == 3) return vel * flux3(AT(u, i - 2, j, k), AT(u, i - 1, j, k), AT(u, i, j, k), AT(u, i + 1, j, k), vel, c->hup);
  return vel * flux5(AT(u, i - 3, j, k), AT(u, i - 2, j, k), AT(u, i - 1, j, k), AT(u, i, j, k), AT(u, i + 1, j, k),
                     AT(u, i + 2, j, k), vel, c->hup);
}
static double tu_fy(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *u = F_(CW_U_2), *rv = F_(CW_RV);
  const int o = ord_face(j, c->sp.ny, c->sp.y);
  if (o == 2) return Q * (AT(rv, i, j, k) + AT(rv, i - 1, j, k)) * (AT(u, i, j, k) + AT(u, i, j - 1, k));
  const double vel = H * (AT(rv, i, j, k) + AT(rv, i - 1, j, k));
  if (o == 3) return vel * flux3(AT(u, i, j - 2, k), AT(u, i, j - 1, k), AT(u, i, j, k), AT(u, i, j + 1, k), vel, c->hup);
  return vel * flux5(AT(u, i, j - 3, k), AT(u, i, j - 2, k), AT(u, i, j - 1, k), AT(u, i, j, k), AT(u, i, j + 1, k),
                     AT(u, i, j + 2, k), vel, c->hup);
}
static double tu_fz(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *u = F_(CW_U_2), *ww = F_(CW_WW);
  if (k == 0 || k == c->nz) return 0;
  const double vel = H * (AT(ww, i - 1, j, k) + AT(ww, i, j, k));
  if (k == 1 || k == c->nz - 1) return vel * (d->fnm[k] * AT(u, i, j, k) + d->fnp[k] * AT(u, i, j, k - 1));
  return vel * flux3(AT(u, i, j, k - 2), AT(u, i, j, k - 1), AT(u, i, j, k), AT(u, i, j, k + 1), -vel, c->vup);
}
static double pu_(or_dom* d, int i, int j, int k) { return AT(F_(CW_P), i - 1, j, k) + AT(F_(CW_P), i, j, k); }
static double tu_dpn(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  const int nz = c->nz;
  if (k == 0) return H * (d->cf1 * pu_(d, i, j, 0) + d->cf2 * pu_(d, i, j, 1) + d->cf3 * pu_(d, i, j, 2));
  if (k == nz) return c->top_lid ? H * (d->cfn * pu_(d, i, j, nz - 1) + d->cfn1 * pu_(d, i, j, nz - 2)) : 0.0;
  return H * (d->fnm[k] * pu_(d, i, j, k) + d->fnp[k] * pu_(d, i, j, k - 1));
}
/* advect_u open_ys / open_ye: the v-flux terms of the outermost rows (KTendU::open_y_term, :193-208) */
static double tu_open_y(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *u = F_(CW_U_2), *rv = F_(CW_RV);
  const int imin = 0, imax = c->sp.nx - 1;
  const int ip = i < imax ? i : imax, im = i - 1 > imin ? i - 1 : imin;
  const double mrdy = AT(F_(CW_MSFUX), i, j, 0) * d->rdy;
  if (j == 0) {
    const double vw = H * (AT(rv, ip, 0, k) + AT(rv, im, 0, k));
    const double vb = vw < 0.0 ? vw : 0.0;
    const double dvm = AT(rv, ip, 1, k) - AT(rv, ip, 0, k), dvp = AT(rv, im, 1, k) - AT(rv, im, 0, k);
    return mrdy * (vb * (AT(u, i, 1, k) - AT(u, i, 0, k)) + H * AT(u, i, 0, k) * (dvm + dvp));
  }
  const int je = c->sp.ny;
  const double vw = H * (AT(rv, ip, je, k) + AT(rv, im, je, k));
  const double vb = vw > 0.0 ? vw : 0.0;
  const double dvm = AT(rv, ip, je, k) - AT(rv, ip, je - 1, k), dvp = AT(rv, im, je, k) - AT(rv, im, je - 1, k);
  return mrdy * (vb * (AT(u, i, je - 1, k) - AT(u, i, je - 2, k)) + H * AT(u, i, je - 1, k) * (dvm + dvp));
}
static double tend_u(const tctx* c, int i, int j, int k, int use_tendf) {
  or_dom* d = c->d;
  fld *msfux = F_(CW_MSFUX), *msfuy = F_(CW_MSFUY), *muu = F_(CW_MUU), *mu = F_(CW_MU_2);
  fld *ph = F_(CW_PH_2), *alt = F_(CW_ALT), *p = F_(CW_P), *al = F_(CW_AL), *pb = F_(CW_PB), *php = F_(CW_PHP);
  fld *rv = F_(CW_RV), *rw = F_(CW_RW), *u = F_(CW_U_2), *ru = F_(CW_RU), *mut = F_(CW_MUT);
  const double rdx = d->rdx, rdy = d->rdy;
  if (c->sp.ox && (i == 0 || i == c->sp.nx)) {
    /* open x boundary face (:210-227): the radiation condition with phase speed cb, the vertical advection unless
     * y is open too, and the held tendency */
    double t;
    if (i == 0) {
      double ub = AT(ru, 0, j, k) - CB * (d->c1h[k] * AT(mut, 0, j, 0) + d->c2h[k]);
      ub = ub < 0.0 ? ub : 0.0;
      t = 0.0 - rdx * ub * (AT(u, 1, j, k) - AT(u, 0, j, k));
    } else {
      double ub = AT(ru, i, j, k) + CB * (d->c1h[k] * AT(mut, i - 1, j, 0) + d->c2h[k]);
      ub = ub > 0.0 ? ub : 0.0;
      t = 0.0 - rdx * ub * (AT(u, i, j, k) - AT(u, i - 1, j, k));
    }
    if (!c->sp.oy) t -= d->rdnw[k] * (tu_fz(c, i, j, k + 1) - tu_fz(c, i, j, k));
    if (use_tendf) t += AT(F_(CW_RU_TENDF), i, j, k) / AT(msfuy, i, j, 0);
    return t;
  }
  double t = -(AT(msfux, i, j, 0) * rdx) * (tu_fx(c, i + 1, j, k) - tu_fx(c, i, j, k));
  if (c->do_y) {
    const int orow = c->sp.oy && (j == 0 || j == c->sp.ny - 1);
    if (!orow) t -= (AT(msfux, i, j, 0) * rdy) * (tu_fy(c, i, j + 1, k) - tu_fy(c, i, j, k));
    else t -= tu_open_y(c, i, j, k);
  }
  if (!(c->sp.oy && c->sp.x && (i == 0 || i == c->sp.nx))) t -= d->rdnw[k] * (tu_fz(c, i, j, k + 1) - tu_fz(c, i, j, k));
  const double rm = AT(msfux, i, j, 0) / AT(msfuy, i, j, 0);
  double dpx = rm * H * rdx * (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k]) *
               ((AT(ph, i, j, k + 1) - AT(ph, i - 1, j, k + 1) + AT(ph, i, j, k) - AT(ph, i - 1, j, k)) +
                (AT(alt, i, j, k) + AT(alt, i - 1, j, k)) * (AT(p, i, j, k) - AT(p, i - 1, j, k)) +
                (AT(al, i, j, k) + AT(al, i - 1, j, k)) * (AT(pb, i, j, k) - AT(pb, i - 1, j, k)));
  dpx += rm * rdx * (AT(php, i, j, k) - AT(php, i - 1, j, k)) *
         (d->rdnw[k] * (tu_dpn(c, i, j, k + 1) - tu_dpn(c, i, j, k)) -
          H * (d->c1h[k] * AT(mu, i - 1, j, 0) + d->c1h[k] * AT(mu, i, j, 0)));
  t -= cqu_(d, i, j, k) * dpx;
  const double rw4 = Q * (AT(rw, i - 1, j, k + 1) + AT(rw, i - 1, j, k) + AT(rw, i, j, k + 1) + AT(rw, i, j, k));
  const double rv4 = Q * (AT(rv, i - 1, j + 1, k) + AT(rv, i, j + 1, k) + AT(rv, i - 1, j, k) + AT(rv, i, j, k));
  if (d->o.coriolis || d->o.mapped) { /* Coriolis (:249-253; MapC::cor = mapped || coriolis) */
    fld *f = F_(CW_F), *e = F_(CW_E), *cosa = F_(CW_COSA);
    t = t + rm * H * (AT(f, i, j, 0) + AT(f, i - 1, j, 0)) * rv4 -
        H * (AT(e, i, j, 0) + AT(e, i - 1, j, 0)) * H * (AT(cosa, i, j, 0) + AT(cosa, i - 1, j, 0)) * rw4;
  }
  if (d->o.mapped) /* curvature with the map factors' gradients (:255-257) */
    t = t + H * (vxgm(d, i, j, k) + vxgm(d, i - 1, j, k)) * rv4 - AT(u, i, j, k) * RERADIUS * rw4;
  else
    t = t - AT(u, i, j, k) * RERADIUS * rw4;
  if (use_tendf) t += AT(F_(CW_RU_TENDF), i, j, k) / AT(msfuy, i, j, 0);
  return t;
}

/* --- V --- */
static double tv_fx(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *v = F_(CW_V_2), *ru = F_(CW_RU);
  const int o = ord_face(i, c->sp.nx, c->sp.x);
  if (o == 2) return Q * (AT(ru, i, j, k) + AT(ru, i, j - 1, k)) * (AT(v, i, j, k) + AT(v, i - 1, j, k));
  const double vel = H * (AT(ru, i, j, k) + AT(ru, i, j - 1, k));
  if (o == 3) return vel * flux3(AT(v, i - 2, j, k), AT(v, i - 1, j, k), AT(v, i, j, k), AT(v, i + 1, j, k), vel, c->hup);
  return vel * flux5(AT(v, i - 3, j, k), AT(v, i - 2, j, k), AT(v, i - 1, j, k), AT(v, i, j, k), AT(v, i + 1, j, k),
                     AT(v, i + 2, j, k), vel, c->hup);
}
static double tv_fy(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *v = F_(CW_V_2), *rv = F_(CW_RV);
  const int o = ord_mass(j, c->sp.ny, c->sp.y);
  if (o == 2) {
    if (j <= 1) {
      const double vb = (c->sp.sy && AT(v, i, j, k) < 0.0) ? AT(v, i, j, k) : AT(v, i, j - 1, k);
      return Q * (AT(rv, i, j, k) + AT(rv, i, j - 1, k)) * (AT(v, i, j, k) + vb);
    }
    const double vb = (c->sp.sy && AT(v, i, j - 1, k) > 0.0) ? AT(v, i, j - 1, k) : AT(v, i, j, k);
    return Q * (AT(rv, i, j, k) + AT(rv, i, j - 1, k)) * (vb + AT(v, i, j - 1, k));
  }
  const double vel = H * (AT(rv, i, j, k) + AT(rv, i, j - 1, k));
  if (o == 3) return vel * flux3(AT(v, i, j - 2, k), AT(v, i, j - 1, k), AT(v, i, j, k), AT(v, i, j + 1, k), vel, c->hup);
  return vel * flux5(AT(v, i, j - 3, k), AT(v, i, j - 2, k), AT(v, i, j - 1, k), AT(v, i, j, k), AT(v, i, j + 1, k),
                     AT(v, i, j + 2, k), vel, c->hup);
}
static double tv_fz(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *v = F_(CW_V_2), *ww = F_(CW_WW);
  if (k == 0 || k == c->nz) return 0;
  const double vel = H * (AT(ww, i, j - 1, k) + AT(ww, i, j, k));
  if (k == 1 || k == c->nz - 1) return vel * (d->fnm[k] * AT(v, i, j, k) + d->fnp[k] * AT(v, i, j, k - 1));
  return vel * flux3(AT(v, i, j, k - 2), AT(v, i, j, k - 1), AT(v, i, j, k), AT(v, i, j, k + 1), -vel, c->vup);
}
static double pv_(or_dom* d, int i, int j, int k) { return AT(F_(CW_P), i, j - 1, k) + AT(F_(CW_P), i, j, k); }
static double tv_dpn(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  const int nz = c->nz;
  if (k == 0) return H * (d->cf1 * pv_(d, i, j, 0) + d->cf2 * pv_(d, i, j, 1) + d->cf3 * pv_(d, i, j, 2));
  if (k == nz) return c->top_lid ? H * (d->cfn * pv_(d, i, j, nz - 1) + d->cfn1 * pv_(d, i, j, nz - 2)) : 0.0;
  return H * (d->fnm[k] * pv_(d, i, j, k) + d->fnp[k] * pv_(d, i, j, k - 1));
}
/* advect_v open_xs / open_xe: the u-flux terms of the outermost columns (KTendV::open_x_term, :307-323) */
static double tv_open_x(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *v = F_(CW_V_2), *ru = F_(CW_RU), *msfvy = F_(CW_MSFVY);
  const int jmin = 0, jmax = c->sp.ny - 1;
  const int jp = j < jmax ? j : jmax, jm = j - 1 > jmin ? j - 1 : jmin;
  if (i == 0) {
    const double mrdx = AT(msfvy, 0, j, 0) * d->rdx;
    const double uw = H * (AT(ru, 0, jp, k) + AT(ru, 0, jm, k));
    const double ub = uw < 0.0 ? uw : 0.0;
    const double dup = AT(ru, 1, jp, k) - AT(ru, 0, jp, k), dum = AT(ru, 1, jm, k) - AT(ru, 0, jm, k);
    return mrdx * (ub * (AT(v, 1, j, k) - AT(v, 0, j, k)) + H * AT(v, 0, j, k) * (dup + dum));
  }
  const int ie = c->sp.nx;
  const double mrdx = AT(msfvy, ie - 1, j, 0) * d->rdx;
  const double uw = H * (AT(ru, ie, jp, k) + AT(ru, ie, jm, k));
  const double ub = uw > 0.0 ? uw : 0.0;
  const double dup = AT(ru, ie, jp, k) - AT(ru, ie - 1, jp, k), dum = AT(ru, ie, jm, k) - AT(ru, ie - 1, jm, k);
  return mrdx * (ub * (AT(v, ie - 1, j, k) - AT(v, ie - 2, j, k)) + H * AT(v, ie - 1, j, k) * (dup + dum));
}
static double tend_v(const tctx* c, int i, int j, int k, int use_tendf) {
  or_dom* d = c->d;
  fld *msfvx = F_(CW_MSFVX), *msfvy = F_(CW_MSFVY), *mvi = F_(CW_MSFVX_INV), *muv = F_(CW_MUV), *mu = F_(CW_MU_2);
  fld *ph = F_(CW_PH_2), *alt = F_(CW_ALT), *p = F_(CW_P), *al = F_(CW_AL), *pb = F_(CW_PB), *php = F_(CW_PHP);
  fld *rw = F_(CW_RW), *v = F_(CW_V_2), *rv = F_(CW_RV), *mut = F_(CW_MUT);
  const double rdx = d->rdx, rdy = d->rdy;
  if (c->sp.oy && (j == 0 || j == c->sp.ny)) { /* open y boundary face (:327-340): radiation only */
    double t;
    if (j == 0) {
      double vb = AT(rv, i, 0, k) - CB * (d->c1h[k] * AT(mut, i, 0, 0) + d->c2h[k]);
      vb = vb < 0.0 ? vb : 0.0;
      t = 0.0 - rdy * vb * (AT(v, i, 1, k) - AT(v, i, 0, k));
    } else {
      double vb = AT(rv, i, j, k) + CB * (d->c1h[k] * AT(mut, i, j - 1, 0) + d->c2h[k]);
      vb = vb > 0.0 ? vb : 0.0;
      t = 0.0 - rdy * vb * (AT(v, i, j, k) - AT(v, i, j - 1, k));
    }
    if (use_tendf) t += AT(F_(CW_RV_TENDF), i, j, k) * AT(mvi, i, j, 0);
    return t;
  }
  const double rm = AT(msfvy, i, j, 0) / AT(msfvx, i, j, 0);
  double t;
  if (c->sp.ox && (i == 0 || i == c->sp.nx - 1)) { /* open x: the y flux, then the open term instead of the x flux */
    t = -(AT(msfvy, i, j, 0) * rdy) * (tv_fy(c, i, j + 1, k) - tv_fy(c, i, j, k));
    t -= tv_open_x(c, i, j, k);
  } else {
    t = -(AT(msfvy, i, j, 0) * rdx) * (tv_fx(c, i + 1, j, k) - tv_fx(c, i, j, k));
    t -= (AT(msfvy, i, j, 0) * rdy) * (tv_fy(c, i, j + 1, k) - tv_fy(c, i, j, k));
  }
  t -= rm * d->rdnw[k] * (tv_fz(c, i, j, k + 1) - tv_fz(c, i, j, k));
  double dpy = rm * H * rdy * (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k]) *
               ((AT(ph, i, j, k + 1) - AT(ph, i, j - 1, k + 1) + AT(ph, i, j, k) - AT(ph, i, j - 1, k)) +
                (AT(alt, i, j, k) + AT(alt, i, j - 1, k)) * (AT(p, i, j, k) - AT(p, i, j - 1, k)) +
                (AT(al, i, j, k) + AT(al, i, j - 1, k)) * (AT(pb, i, j, k) - AT(pb, i, j - 1, k)));
  dpy += rm * rdy * (AT(php, i, j, k) - AT(php, i, j - 1, k)) *
         (d->rdnw[k] * (tv_dpn(c, i, j, k + 1) - tv_dpn(c, i, j, k)) -
          H * (d->c1h[k] * AT(mu, i, j - 1, 0) + d->c1h[k] * AT(mu, i, j, 0)));
  t -= cqv_(d, i, j, k) * dpy;
  const double rw4 = Q * (AT(rw, i, j - 1, k + 1) + AT(rw, i, j - 1, k) + AT(rw, i, j, k + 1) + AT(rw, i, j, k));
  fld* ru = F_(CW_RU);
  const double ru4 = Q * (AT(ru, i, j, k) + AT(ru, i + 1, j, k) + AT(ru, i, j - 1, k) + AT(ru, i + 1, j - 1, k));
  if (d->o.coriolis || d->o.mapped) { /* Coriolis (:362-365) */
    fld *f = F_(CW_F), *e = F_(CW_E), *sina = F_(CW_SINA);
    t = t - rm * H * (AT(f, i, j, 0) + AT(f, i, j - 1, 0)) * ru4 +
        rm * H * (AT(e, i, j, 0) + AT(e, i, j - 1, 0)) * H * (AT(sina, i, j, 0) + AT(sina, i, j - 1, 0)) * rw4;
  }
  if (d->o.mapped) /* curvature (:367-369) */
    t = t - H * (vxgm(d, i, j, k) + vxgm(d, i, j - 1, k)) * ru4 - rm * AT(v, i, j, k) * RERADIUS * rw4;
  else
    t = t - rm * AT(v, i, j, k) * RERADIUS * rw4;
  if (use_tendf) t += AT(F_(CW_RV_TENDF), i, j, k) * AT(mvi, i, j, 0);
  return t;
}

/* --- W (levels 1..nz) --- */
static double tw_rux(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld* ru = F_(CW_RU);
  const int nz = c->nz;
  if (k < nz) return d->fnm[k] * AT(ru, i, j, k) + d->fnp[k] * AT(ru, i, j, k - 1);
  return (2.0 - d->fnm[nz - 1]) * AT(ru, i, j, nz - 1) - d->fnp[nz - 1] * AT(ru, i, j, nz - 2);
}
static double tw_rvy(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld* rv = F_(CW_RV);
  const int nz = c->nz;
  if (k < nz) return d->fnm[k] * AT(rv, i, j, k) + d->fnp[k] * AT(rv, i, j, k - 1);
  return (2.0 - d->fnm[nz - 1]) * AT(rv, i, j, nz - 1) - d->fnp[nz - 1] * AT(rv, i, j, nz - 2);
}
static double tw_fx(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld* w = F_(CW_W_2);
  const double vel = tw_rux(c, i, j, k);
  const int o = ord_face(i, c->sp.nx, c->sp.x);
  if (o == 2) return H * vel * (AT(w, i, j, k) + AT(w, i - 1, j, k));
  if (o == 3) return vel * flux3(AT(w, i - 2, j, k), AT(w, i - 1, j, k), AT(w, i, j, k), AT(w, i + 1, j, k), vel, c->hup);
  return vel * flux5(AT(w, i - 3, j, k), AT(w, i - 2, j, k), AT(w, i - 1, j, k), AT(w, i, j, k), AT(w, i + 1, j, k),
                     AT(w, i + 2, j, k), vel, c->hup);
}
static double tw_fy(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld* w = F_(CW_W_2);
  const double vel = tw_rvy(c, i, j, k);
  const int o = ord_face(j, c->sp.ny, c->sp.y);
  if (o == 2) return H * vel * (AT(w, i, j, k) + AT(w, i, j - 1, k));
  if (o == 3) return vel * flux3(AT(w, i, j - 2, k), AT(w, i, j - 1, k), AT(w, i, j, k), AT(w, i, j + 1, k), vel, c->hup);
  return vel * flux5(AT(w, i, j - 3, k), AT(w, i, j - 2, k), AT(w, i, j - 1, k), AT(w, i, j, k), AT(w, i, j + 1, k),
                     AT(w, i, j + 2, k), vel, c->hup);
}
static double tw_fz(const tctx* c, int i, int j, int m) { /* vertical flux at mass level m */
  or_dom* d = c->d;
  fld *w = F_(CW_W_2), *ww = F_(CW_WW);
  if (m == 0 || m == c->nz - 1)
    return 0.25 * (AT(ww, i, j, m + 1) + AT(ww, i, j, m)) * (AT(w, i, j, m + 1) + AT(w, i, j, m));
  const double vel = H * (AT(ww, i, j, m + 1) + AT(ww, i, j, m));
  return vel * flux3(AT(w, i, j, m - 1), AT(w, i, j, m), AT(w, i, j, m + 1), AT(w, i, j, m + 2), -vel, c->vup);
}
/* advect_w open_xs/xe (open_ys/ye) terms of the outermost columns (rows) (KTendW::open_x_term / open_y_term,
 * :416-453): fnm/fnp-interpolated ru (rv) at the w level, extrapolated at the lid */
static double tw_open_x(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *ru = F_(CW_RU), *w = F_(CW_W_2);
  const int nz = c->nz;
  const int a = i == 0 ? 0 : c->sp.nx - 1, b = i == 0 ? 1 : c->sp.nx;
  double uw, dru;
  if (k < nz) {
    uw = H * (d->fnm[k] * (AT(ru, a, j, k) + AT(ru, b, j, k)) + d->fnp[k] * (AT(ru, a, j, k - 1) + AT(ru, b, j, k - 1)));
    dru = d->fnm[k] * (AT(ru, b, j, k) - AT(ru, a, j, k)) + d->fnp[k] * (AT(ru, b, j, k - 1) - AT(ru, a, j, k - 1));
  } else {
    const double fm = 2.0 - d->fnm[nz - 1], fp = d->fnp[nz - 1];
    uw = H * (fm * (AT(ru, a, j, nz - 1) + AT(ru, b, j, nz - 1)) - fp * (AT(ru, a, j, nz - 2) + AT(ru, b, j, nz - 2)));
    dru = fm * (AT(ru, b, j, nz - 1) - AT(ru, a, j, nz - 1)) - fp * (AT(ru, b, j, nz - 2) - AT(ru, a, j, nz - 2));
  }
  if (i == 0) {
    const double ub = uw < 0.0 ? uw : 0.0;
    return d->rdx * (ub * (AT(w, 1, j, k) - AT(w, 0, j, k)) + AT(w, 0, j, k) * dru);
  }
  const double ub = uw > 0.0 ? uw : 0.0;
  return d->rdx * (ub * (AT(w, i, j, k) - AT(w, i - 1, j, k)) + AT(w, i, j, k) * dru);
}
static double tw_open_y(const tctx* c, int i, int j, int k) {
  or_dom* d = c->d;
  fld *rv = F_(CW_RV), *w = F_(CW_W_2);
  const int nz = c->nz;
  const int a = j == 0 ? 0 : c->sp.ny - 1, b = j == 0 ? 1 : c->sp.ny;
  double vw, drv;
  if (k < nz) {
    vw = H * (d->fnm[k] * (AT(rv, i, a, k) + AT(rv, i, b, k)) + d->fnp[k] * (AT(rv, i, a, k - 1) + AT(rv, i, b, k - 1)));
    drv = d->fnm[k] * (AT(rv, i, b, k) - AT(rv, i, a, k)) + d->fnp[k] * (AT(rv, i, b, k - 1) - AT(rv, i, a, k - 1));
  } else {
    const double fm = 2.0 - d->fnm[nz - 1], fp = d->fnp[nz - 1];
    vw = H * (fm * (AT(rv, i, a, nz - 1) + AT(rv, i, b, nz - 1)) - fp * (AT(rv, i, a, nz - 2) + AT(rv, i, b, nz - 2)));
    drv = fm * (AT(rv, i, b, nz - 1) - AT(rv, i, a, nz - 1)) - fp * (AT(rv, i, b, nz - 2) - AT(rv, i, a, nz - 2));
  }
  if (j == 0) {
    const double vb = vw < 0.0 ? vw : 0.0;
    return d->rdy * (vb * (AT(w, i, 1, k) - AT(w, i, 0, k)) + AT(w, i, 0, k) * drv);
  }
  const double vb = vw > 0.0 ? vw : 0.0;
  return d->rdy * (vb * (AT(w, i, j, k) - AT(w, i, j - 1, k)) + AT(w, i, j, k) * drv);
}
static double tend_w(const tctx* c, int i, int j, int k, int use_tendf, double wd_dt, double w_crit) {
  or_dom* d = c->d;
  fld *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY), *p = F_(CW_P), *mu = F_(CW_MU_2), *mub = F_(CW_MUB);
  fld *ru = F_(CW_RU), *rv = F_(CW_RV), *u = F_(CW_U_2), *v = F_(CW_V_2), *w = F_(CW_W_2), *ww = F_(CW_WW),
      *mut = F_(CW_MUT);
  const int nz = c->nz;
  const double rdx = d->rdx, rdy = d->rdy;
  double t;
  const int ocol = c->sp.ox && (i == 0 || i == c->sp.nx - 1), orow = c->sp.oy && (j == 0 || j == c->sp.ny - 1);
  if (ocol || orow) { /* WRF order: y flux, x flux, open x terms, open y terms */
    t = 0.0;
    if (c->do_y && !orow) t = t - (AT(msftx, i, j, 0) * rdy) * (tw_fy(c, i, j + 1, k) - tw_fy(c, i, j, k));
    if (!ocol) t = t - (AT(msftx, i, j, 0) * rdx) * (tw_fx(c, i + 1, j, k) - tw_fx(c, i, j, k));
    if (ocol) t = t - tw_open_x(c, i, j, k);
    if (orow) t = t - tw_open_y(c, i, j, k);
  } else {
    t = -(AT(msftx, i, j, 0) * rdx) * (tw_fx(c, i + 1, j, k) - tw_fx(c, i, j, k));
    if (c->do_y) t -= (AT(msftx, i, j, 0) * rdy) * (tw_fy(c, i, j + 1, k) - tw_fy(c, i, j, k));
  }
  const double rmsft = 1.0 / AT(msfty, i, j, 0);
  if (k < nz) {
    t -= d->rdn[k] * (tw_fz(c, i, j, k) - tw_fz(c, i, j, k - 1));
    const double cqw = cqw_(d, i, j, k), cq1 = 1.0 / (1.0 + cqw), cq2 = cqw * cq1;
    t += rmsft * G_ *
         (cq1 * d->rdn[k] * (AT(p, i, j, k) - AT(p, i, j, k - 1)) - d->c1f[k] * AT(mu, i, j, 0) -
          cq2 * (d->c1f[k] * AT(mub, i, j, 0) + d->c2f[k]));
    if (wd_dt != 0.0) {
      const double muf = d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k];
      double cfl = AT(ww, i, j, k) / muf * d->rdnw[k] * wd_dt;
      cfl = cfl < 0.0 ? -cfl : cfl;
      if (cfl > 1.0) t = t - (AT(w, i, j, k) < 0.0 ? -1.0 : 1.0) * 0.3 * (cfl - w_crit) * muf;
    }
    const double ruw = H * (d->fnm[k] * (AT(ru, i, j, k) + AT(ru, i + 1, j, k)) +
                            d->fnp[k] * (AT(ru, i, j, k - 1) + AT(ru, i + 1, j, k - 1)));
    const double rvw = H * (d->fnm[k] * (AT(rv, i, j, k) + AT(rv, i, j + 1, k)) +
                            d->fnp[k] * (AT(rv, i, j, k - 1) + AT(rv, i, j + 1, k - 1)));
    const double rmt = AT(msftx, i, j, 0) / AT(msfty, i, j, 0);
    if (d->o.coriolis || d->o.mapped) /* Coriolis (:484) */
      t = t + AT(F_(CW_E), i, j, 0) * (AT(F_(CW_COSA), i, j, 0) * ruw - rmt * AT(F_(CW_SINA), i, j, 0) * rvw);
    const double uw = H * (d->fnm[k] * (AT(u, i, j, k) + AT(u, i + 1, j, k)) +
                           d->fnp[k] * (AT(u, i, j, k - 1) + AT(u, i + 1, j, k - 1)));
    const double vw = H * (d->fnm[k] * (AT(v, i, j, k) + AT(v, i, j + 1, k)) +
                           d->fnp[k] * (AT(v, i, j, k - 1) + AT(v, i, j + 1, k - 1)));
    t = t + RERADIUS * (ruw * uw + rmt * rvw * vw);
  } else {
    t += 2.0 * d->rdn[nz - 1] * tw_fz(c, i, j, nz - 1);
    const double cqw = cqw_(d, i, j, nz - 1), cq1 = 1.0 / (1.0 + cqw), cq2 = cqw * cq1;
    t += rmsft * G_ *
         (cq1 * 2.0 * d->rdnw[nz - 1] * (-AT(p, i, j, nz - 1)) - d->c1f[nz] * AT(mu, i, j, 0) -
          cq2 * (d->c1f[nz] * AT(mub, i, j, 0) + d->c2f[nz]));
  }
  if (use_tendf) t += AT(F_(CW_RW_TENDF), i, j, k) / AT(msfty, i, j, 0);
  return t;
}

/* --- theta (and the scalar advection of advect_scalar) --- */
static double tt_fx(const tctx* c, fld* t, int i, int j, int k) {
  or_dom* d = c->d;
  fld* ru = F_(CW_RU);
  const double vel = AT(ru, i, j, k);
  const int o = ord_face(i, c->sp.nx, c->sp.x);
  if (o == 2) return H * vel * (AT(t, i, j, k) + AT(t, i - 1, j, k));
  if (o == 3) return vel * flux3(AT(t, i - 2, j, k), AT(t, i - 1, j, k), AT(t, i, j, k), AT(t, i + 1, j, k), vel, c->hup);
  return vel * flux5(AT(t, i - 3, j, k), AT(t, i - 2, j, k), AT(t, i - 1, j, k), AT(t, i, j, k), AT(t, i + 1, j, k),
                     AT(t, i + 2, j, k), vel, c->hup);
}
static double tt_fy(const tctx* c, fld* t, int i, int j, int k) {
  or_dom* d = c->d;
  fld* rv = F_(CW_RV);
  const double vel = AT(rv, i, j, k);
  const int o = ord_face(j, c->sp.ny, c->sp.y);
  if (o == 2) return H * vel * (AT(t, i, j, k) + AT(t, i, j - 1, k));
  if (o == 3) return vel * flux3(AT(t, i, j - 2, k), AT(t, i, j - 1, k), AT(t, i, j, k), AT(t, i, j + 1, k), vel, c->hup);
  return vel * flux5(AT(t, i, j - 3, k), AT(t, i, j - 2, k), AT(t, i, j - 1, k), AT(t, i, j, k), AT(t, i, j + 1, k),
                     AT(t, i, j + 2, k), vel, c->hup);
}
static double tt_fz(const tctx* c, fld* t, int i, int j, int k) {
  or_dom* d = c->d;
  fld* ww = F_(CW_WW);
  if (k == 0 || k == c->nz) return 0;
  const double vel = AT(ww, i, j, k);
  if (k == 1 || k == c->nz - 1) return vel * (d->fnm[k] * AT(t, i, j, k) + d->fnp[k] * AT(t, i, j, k - 1));
  return vel * flux3(AT(t, i, j, k - 2), AT(t, i, j, k - 1), AT(t, i, j, k), AT(t, i, j, k + 1), -vel, c->vup);
}
/* open boundaries of advect_scalar / advect_scalar_pd (kern::open_x_scalar / open_y_scalar, kernels_common.hpp:61-84):
 * the outermost column (row) takes rdx (ub (qo(inner) - qo(outer)) + q (ru(b) - ru(a))) with the inflow mean normal
 * mass flux ub of the cell; returned without sign */
static double open_x_scalar(const fld* q, const fld* qo, const fld* ru, double rdx, int i, int j, int k, int nx) {
  if (i == 0) {
    double ub = 0.5 * (AT(ru, 0, j, k) + AT(ru, 1, j, k));
    ub = ub < 0.0 ? ub : 0.0;
    return rdx * (ub * (AT(qo, 1, j, k) - AT(qo, 0, j, k)) + AT(q, 0, j, k) * (AT(ru, 1, j, k) - AT(ru, 0, j, k)));
  }
  double ub = 0.5 * (AT(ru, nx - 1, j, k) + AT(ru, nx, j, k));
  ub = ub > 0.0 ? ub : 0.0;
  return rdx * (ub * (AT(qo, nx - 1, j, k) - AT(qo, nx - 2, j, k)) +
                AT(q, nx - 1, j, k) * (AT(ru, nx, j, k) - AT(ru, nx - 1, j, k)));
}
static double open_y_scalar(const fld* q, const fld* qo, const fld* rv, double rdy, int i, int j, int k, int ny) {
  if (j == 0) {
    double vb = 0.5 * (AT(rv, i, 0, k) + AT(rv, i, 1, k));
    vb = vb < 0.0 ? vb : 0.0;
    return rdy * (vb * (AT(qo, i, 1, k) - AT(qo, i, 0, k)) + AT(q, i, 0, k) * (AT(rv, i, 1, k) - AT(rv, i, 0, k)));
  }
  double vb = 0.5 * (AT(rv, i, ny - 1, k) + AT(rv, i, ny, k));
  vb = vb > 0.0 ? vb : 0.0;
  return rdy * (vb * (AT(qo, i, ny - 1, k) - AT(qo, i, ny - 2, k)) +
                AT(q, i, ny - 1, k) * (AT(rv, i, ny, k) - AT(rv, i, ny - 1, k)));
}
static double tend_t(const tctx* c, int i, int j, int k, int use_tendf, int use_hd) {
  or_dom* d = c->d;
  fld *t = F_(CW_T_2), *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY);
  double r;
  const int ocol = c->sp.ox && (i == 0 || i == c->sp.nx - 1), orow = c->sp.oy && (j == 0 || j == c->sp.ny - 1);
  if (ocol || orow) { /* open boundary (:535-541): y flux, x flux, open x terms, open y terms, then the vertical */
    r = 0.0;
    if (c->do_y && !orow) r = r - (AT(msftx, i, j, 0) * d->rdy) * (tt_fy(c, t, i, j + 1, k) - tt_fy(c, t, i, j, k));
    if (!ocol) r = r - (AT(msftx, i, j, 0) * d->rdx) * (tt_fx(c, t, i + 1, j, k) - tt_fx(c, t, i, j, k));
    if (ocol) r = r - open_x_scalar(t, t, F_(CW_RU), d->rdx, i, j, k, c->sp.nx);
    if (orow) r = r - open_y_scalar(t, t, F_(CW_RV), d->rdy, i, j, k, c->sp.ny);
  } else {
    r = -(AT(msftx, i, j, 0) * d->rdx) * (tt_fx(c, t, i + 1, j, k) - tt_fx(c, t, i, j, k));
    if (c->do_y) r -= (AT(msftx, i, j, 0) * d->rdy) * (tt_fy(c, t, i, j + 1, k) - tt_fy(c, t, i, j, k));
  }
  r -= d->rdnw[k] * (tt_fz(c, t, i, j, k + 1) - tt_fz(c, t, i, j, k));
  if (use_tendf) r += AT(F_(CW_T_TENDF), i, j, k) / AT(msfty, i, j, 0);
  if (use_hd)
    r += (d->c1h[k] * AT(F_(CW_MUT), i, j, 0) + d->c2h[k]) * AT(F_(CW_H_DIABATIC), i, j, k) / AT(msfty, i, j, 0);
  return r;
}

/* --- geopotential (levels 1..nz) --- */
static double tph_wdwn(or_dom* d, int i, int j, int m) {
  fld *ww = F_(CW_WW), *ph = F_(CW_PH_2), *phb = F_(CW_PHB);
  return H * (AT(ww, i, j, m + 1) + AT(ww, i, j, m)) * d->rdnw[m] *
         (AT(ph, i, j, m + 1) - AT(ph, i, j, m) + AT(phb, i, j, m + 1) - AT(phb, i, j, m));
}
static double grad6(or_dom* d, int DI, int DJ, int i, int j, int k) {
  fld *ph = F_(CW_PH_2), *phb = F_(CW_PHB);
  return 45.0 * (AT(ph, i + DI, j + DJ, k) - AT(ph, i - DI, j - DJ, k)) -
         9.0 * (AT(ph, i + 2 * DI, j + 2 * DJ, k) - AT(ph, i - 2 * DI, j - 2 * DJ, k)) +
         (AT(ph, i + 3 * DI, j + 3 * DJ, k) - AT(ph, i - 3 * DI, j - 3 * DJ, k)) +
         45.0 * (AT(phb, i + DI, j + DJ, k) - AT(phb, i - DI, j - DJ, k)) -
         9.0 * (AT(phb, i + 2 * DI, j + 2 * DJ, k) - AT(phb, i - 2 * DI, j - 2 * DJ, k)) +
         (AT(phb, i + 3 * DI, j + 3 * DJ, k) - AT(phb, i - 3 * DI, j - 3 * DJ, k));
}
static double grad4(or_dom* d, int DI, int DJ, int i, int j, int k) {
  fld *ph = F_(CW_PH_2), *phb = F_(CW_PHB);
  return 8.0 * (AT(ph, i + DI, j + DJ, k) - AT(ph, i - DI, j - DJ, k)) -
         (AT(ph, i + 2 * DI, j + 2 * DJ, k) - AT(ph, i - 2 * DI, j - 2 * DJ, k)) +
         8.0 * (AT(phb, i + DI, j + DJ, k) - AT(phb, i - DI, j - DJ, k)) -
         (AT(phb, i + 2 * DI, j + 2 * DJ, k) - AT(phb, i - 2 * DI, j - 2 * DJ, k));
}
static double dfwd(or_dom* d, int DI, int DJ, int i, int j, int k) {
  fld *ph = F_(CW_PH_2), *phb = F_(CW_PHB);
  return AT(phb, i + DI, j + DJ, k) - AT(phb, i, j, k) + AT(ph, i + DI, j + DJ, k) - AT(ph, i, j, k);
}
static int ph_horder(int i, int n, int on, int is_x, int open_x) {
  if (!on) return 6;
  if (i <= 0 || i >= n - 1) return 0;
  if (i == 1 || i == n - 2) return 2;
  if (i == 2 || i == n - 3) return (is_x && !open_x) ? 0 : 4; /* open x: 4th order (open_xs/xe only) */
  return 6;
}
static double tend_ph(const tctx* c, int i, int j, int k, int use_tendf) {
  or_dom* d = c->d;
  fld *u = F_(CW_U_2), *v = F_(CW_V_2), *w = F_(CW_W_2), *mut = F_(CW_MUT), *muu = F_(CW_MUU), *muv = F_(CW_MUV);
  fld *msfty = F_(CW_MSFTY), *msfux = F_(CW_MSFUX), *msfvy = F_(CW_MSFVY);
  const int nz = c->nz;
  double t = 0;
  if (k < nz) t = t - (d->fnm[k] * tph_wdwn(d, i, j, k) + d->fnp[k] * tph_wdwn(d, i, j, k - 1));
  t = t + (d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k]) * G_ * AT(w, i, j, k) / AT(msfty, i, j, 0);
  const double r60 = 1.0 / 60.0, r12 = 1.0 / 12.0;
  if (c->do_y) {
    const double mvp = d->c1f[k] * AT(muv, i, j + 1, 0) + d->c2f[k], mvm = d->c1f[k] * AT(muv, i, j, 0) + d->c2f[k];
    const double vp = k < nz ? AT(v, i, j + 1, k) + AT(v, i, j + 1, k - 1)
                             : d->cfn * AT(v, i, j + 1, nz - 1) + d->cfn1 * AT(v, i, j + 1, nz - 2);
    const double vm = k < nz ? AT(v, i, j, k) + AT(v, i, j, k - 1)
                             : d->cfn * AT(v, i, j, nz - 1) + d->cfn1 * AT(v, i, j, nz - 2);
    const double cy = (k < nz ? 0.25 : H) * d->rdy / AT(msfty, i, j, 0);
    const int o = ph_horder(j, c->sp.ny, c->sp.y, 0, c->sp.ox);
    if (o == 6)
      t = t - cy * ((mvp * vp * AT(msfvy, i, j + 1, 0) + mvm * vm * AT(msfvy, i, j, 0)) * r60 * grad6(d, 0, 1, i, j, k));
    else if (o == 4)
      t = t - cy * ((mvp * vp * AT(msfvy, i, j + 1, 0) + mvm * vm * AT(msfvy, i, j, 0)) * r12 * grad4(d, 0, 1, i, j, k));
    else if (o == 2)
      t = t - cy * (mvp * vp * AT(msfvy, i, j + 1, 0) * dfwd(d, 0, 1, i, j, k) +
                    mvm * vm * AT(msfvy, i, j, 0) * dfwd(d, 0, 1, i, j - 1, k));
  }
  const double mup = d->c1f[k] * AT(muu, i + 1, j, 0) + d->c2f[k], mum = d->c1f[k] * AT(muu, i, j, 0) + d->c2f[k];
  const double up = k < nz ? AT(u, i + 1, j, k) + AT(u, i + 1, j, k - 1)
                           : d->cfn * AT(u, i + 1, j, nz - 1) + d->cfn1 * AT(u, i + 1, j, nz - 2);
  const double um =
      k < nz ? AT(u, i, j, k) + AT(u, i, j, k - 1) : d->cfn * AT(u, i, j, nz - 1) + d->cfn1 * AT(u, i, j, nz - 2);
  const double cx = (k < nz ? 0.25 : H) * d->rdx / AT(msfty, i, j, 0);
  const int o = ph_horder(i, c->sp.nx, c->sp.x, 1, c->sp.ox);
  if (o == 6)
    t = t - cx * ((mup * up * AT(msfux, i + 1, j, 0) + mum * um * AT(msfux, i, j, 0)) * r60 * grad6(d, 1, 0, i, j, k));
  else if (o == 2)
    t = t - cx * (mup * up * AT(msfux, i + 1, j, 0) * dfwd(d, 1, 0, i, j, k) +
                  mum * um * AT(msfux, i, j, 0) * dfwd(d, 1, 0, i - 1, j, k));
  else if (o == 4)
    t = t - cx * ((mup * up * AT(msfux, i + 1, j, 0) + mum * um * AT(msfux, i, j, 0)) * r12 * grad4(d, 1, 0, i, j, k));
  /* open boundaries (:636-663, after the advection, south/north then west/east): inflow advection of ph by the normal
   * wind interpolated to the w level (top: level nz - 1, except the west lid level, which adds nothing) */
  fld* ph = F_(CW_PH_2);
  if (c->sp.oy && (j == 0 || j == c->sp.ny - 1)) {
    const int kz = k < nz - 1 ? k : nz - 1;
    const int a = j == 0 ? 0 : c->sp.ny - 1, b = j == 0 ? 1 : c->sp.ny;
    const double vb = H * (d->fnm[kz] * (AT(v, i, b, kz) + AT(v, i, a, kz)) + d->fnp[kz] * (AT(v, i, b, kz - 1) + AT(v, i, a, kz - 1)));
    const double muf = d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k];
    if (j == 0) {
      const double vl = vb < 0.0 ? vb : 0.0;
      t = t - d->rdy * muf * (vl * (AT(ph, i, 1, k) - AT(ph, i, 0, k)));
    } else {
      const double vr = vb > 0.0 ? vb : 0.0;
      t = t - d->rdy * muf * (vr * (AT(ph, i, j, k) - AT(ph, i, j - 1, k)));
    }
  }
  if (c->sp.ox && (i == 0 || i == c->sp.nx - 1) && !(i == 0 && k == nz)) {
    const int kz = k < nz ? k : nz - 1;
    const int a = i == 0 ? 0 : c->sp.nx - 1, b = i == 0 ? 1 : c->sp.nx;
    const double ub = H * (d->fnm[kz] * (AT(u, b, j, kz) + AT(u, a, j, kz)) + d->fnp[kz] * (AT(u, b, j, kz - 1) + AT(u, a, j, kz - 1)));
    const double muf = d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k];
    fld* msftx = F_(CW_MSFTX);
    if (i == 0) {
      const double ul = ub < 0.0 ? ub : 0.0;
      t = t - (AT(msftx, i, j, 0) / AT(msfty, i, j, 0)) * d->rdx * muf * (ul * (AT(ph, 1, j, k) - AT(ph, 0, j, k)));
    } else {
      const double ur = ub > 0.0 ? ub : 0.0;
      t = t - (AT(msftx, i, j, 0) / AT(msfty, i, j, 0)) * d->rdx * muf * (ur * (AT(ph, i, j, k) - AT(ph, i - 1, j, k)));
    }
  }
  if (use_tendf) t = t + AT(F_(CW_PH_TENDF), i, j, k) / AT(msfty, i, j, 0);
  return t;
}

/* ------------------------------------------------------------------ constant-K diffusion
 * DiffusionDriver::prepare / dynamics / scalar for diff_opt 1, km_opt 1
 * (src/dyn/diffusion_driver.cpp:92-150, :153-187, :293-322) with the kernels of
 * src/dyn/diffusion/big_step_diffusion.hpp:26-336 and KIsotropicKm (km_kh.hpp:35-46). */
static double mk(const double* c1, const double* c2, fld* mut, int i, int j, int k) {
  return c1[k] * AT(mut, i, j, 0) + c2[k];
}
static double hdiff_u(or_dom* d, fld* field, fld* mut, fld* xk, const double* c1, const double* c2, int i, int j,
                      int k) {
  fld *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY), *msfux = F_(CW_MSFUX), *msfuy = F_(CW_MSFUY);
  const double rdx = d->rdx, rdy = d->rdy;
  const double mkrdxm =
      (AT(msftx, i - 1, j, 0) / AT(msfty, i - 1, j, 0)) * mk(c1, c2, mut, i - 1, j, k) * AT(xk, i - 1, j, k) * rdx;
  const double mkrdxp = (AT(msftx, i, j, 0) / AT(msfty, i, j, 0)) * mk(c1, c2, mut, i, j, k) * AT(xk, i, j, k) * rdx;
  const double mrdx = AT(msfux, i, j, 0) * AT(msfuy, i, j, 0) * rdx;
  const double mkrdym =
      ((AT(msfuy, i, j, 0) + AT(msfuy, i, j - 1, 0)) / (AT(msfux, i, j, 0) + AT(msfux, i, j - 1, 0))) * 0.25 *
      (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i - 1, j - 1, k) +
       mk(c1, c2, mut, i - 1, j, k)) *
      0.25 * (AT(xk, i, j, k) + AT(xk, i, j - 1, k) + AT(xk, i - 1, j - 1, k) + AT(xk, i - 1, j, k)) * rdy;
  const double mkrdyp =
      ((AT(msfuy, i, j, 0) + AT(msfuy, i, j + 1, 0)) / (AT(msfux, i, j, 0) + AT(msfux, i, j + 1, 0))) * 0.25 *
      (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i - 1, j + 1, k) +
       mk(c1, c2, mut, i - 1, j, k)) *
      0.25 * (AT(xk, i, j, k) + AT(xk, i, j + 1, k) + AT(xk, i - 1, j + 1, k) + AT(xk, i - 1, j, k)) * rdy;
  const double mrdy = AT(msfux, i, j, 0) * AT(msfuy, i, j, 0) * rdy;
  return mrdx * (mkrdxp * (AT(field, i + 1, j, k) - AT(field, i, j, k)) -
                 mkrdxm * (AT(field, i, j, k) - AT(field, i - 1, j, k))) +
         mrdy * (mkrdyp * (AT(field, i, j + 1, k) - AT(field, i, j, k)) -
                 mkrdym * (AT(field, i, j, k) - AT(field, i, j - 1, k)));
}
static double hdiff_v(or_dom* d, fld* field, fld* mut, fld* xk, const double* c1, const double* c2, int i, int j,
                      int k) {
  fld *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY), *msfvx = F_(CW_MSFVX), *msfvy = F_(CW_MSFVY);
  const double rdx = d->rdx, rdy = d->rdy;
  const double mkrdxm =
      ((AT(msfvx, i, j, 0) + AT(msfvx, i - 1, j, 0)) / (AT(msfvy, i, j, 0) + AT(msfvy, i - 1, j, 0))) * 0.25 *
      (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i - 1, j - 1, k) +
       mk(c1, c2, mut, i - 1, j, k)) *
      0.25 * (AT(xk, i, j, k) + AT(xk, i, j - 1, k) + AT(xk, i - 1, j - 1, k) + AT(xk, i - 1, j, k)) * rdx;
  const double mkrdxp =
      ((AT(msfvx, i, j, 0) + AT(msfvx, i + 1, j, 0)) / (AT(msfvy, i, j, 0) + AT(msfvy, i + 1, j, 0))) * 0.25 *
      (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i + 1, j - 1, k) +
       mk(c1, c2, mut, i + 1, j, k)) *
      0.25 * (AT(xk, i, j, k) + AT(xk, i, j - 1, k) + AT(xk, i + 1, j - 1, k) + AT(xk, i + 1, j, k)) * rdx;
  const double mrdx = AT(msfvx, i, j, 0) * AT(msfvy, i, j, 0) * rdx;
  const double mkrdym = (AT(msfty, i, j - 1, 0) / AT(msftx, i, j - 1, 0)) * AT(xk, i, j - 1, k) * rdy;
  const double mkrdyp = (AT(msfty, i, j, 0) / AT(msftx, i, j, 0)) * AT(xk, i, j, k) * rdy;
  const double mrdy = AT(msfvx, i, j, 0) * AT(msfvy, i, j, 0) * rdy;
  return mrdx * (mkrdxp * (AT(field, i + 1, j, k) - AT(field, i, j, k)) -
                 mkrdxm * (AT(field, i, j, k) - AT(field, i - 1, j, k))) +
         mrdy * (mkrdyp * (AT(field, i, j + 1, k) - AT(field, i, j, k)) -
                 mkrdym * (AT(field, i, j, k) - AT(field, i, j - 1, k)));
}
static double hdiff_w(or_dom* d, fld* field, fld* mut, fld* xk, const double* c1, const double* c2, int i, int j,
                      int k) {
  fld *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY), *msfux = F_(CW_MSFUX), *msfuy = F_(CW_MSFUY),
      *msfvy = F_(CW_MSFVY), *mvi = F_(CW_MSFVX_INV);
  const double rdx = d->rdx, rdy = d->rdy;
  const double mkrdxm =
      (AT(msfux, i, j, 0) / AT(msfuy, i, j, 0)) * 0.25 *
      (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i - 1, j, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i - 1, j, k)) *
      0.25 * (AT(xk, i, j, k) + AT(xk, i - 1, j, k) + AT(xk, i, j, k - 1) + AT(xk, i - 1, j, k - 1)) * rdx;
  const double mkrdxp =
      (AT(msfux, i + 1, j, 0) / AT(msfuy, i + 1, j, 0)) * 0.25 *
      (mk(c1, c2, mut, i + 1, j, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i + 1, j, k) + mk(c1, c2, mut, i, j, k)) *
      0.25 * (AT(xk, i + 1, j, k) + AT(xk, i, j, k) + AT(xk, i + 1, j, k - 1) + AT(xk, i, j, k - 1)) * rdx;
  const double mrdx = AT(msftx, i, j, 0) * AT(msfty, i, j, 0) * rdx;
  const double mkrdym =
      (AT(msfvy, i, j, 0) * AT(mvi, i, j, 0)) * 0.25 *
      (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k)) *
      0.25 * (AT(xk, i, j, k) + AT(xk, i, j - 1, k) + AT(xk, i, j, k - 1) + AT(xk, i, j - 1, k - 1)) * rdy;
  const double mkrdyp =
      (AT(msfvy, i, j + 1, 0) * AT(mvi, i, j + 1, 0)) * 0.25 *
      (mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i, j, k)) *
      0.25 * (AT(xk, i, j + 1, k) + AT(xk, i, j, k) + AT(xk, i, j + 1, k - 1) + AT(xk, i, j, k - 1)) * rdy;
  const double mrdy = AT(msftx, i, j, 0) * AT(msfty, i, j, 0) * rdy;
  return mrdx * (mkrdxp * (AT(field, i + 1, j, k) - AT(field, i, j, k)) -
                 mkrdxm * (AT(field, i, j, k) - AT(field, i - 1, j, k))) +
         mrdy * (mkrdyp * (AT(field, i, j + 1, k) - AT(field, i, j, k)) -
                 mkrdym * (AT(field, i, j, k) - AT(field, i, j - 1, k)));
}
/* KHorizDiffM1 (base == NULL) and KHorizDiff3DMP (base given) */
static double hdiff_m(or_dom* d, fld* field, fld* base, fld* mut, fld* xk, const double* c1, const double* c2, int i,
                      int j, int k) {
  fld *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY), *msfux = F_(CW_MSFUX), *msfuy = F_(CW_MSFUY),
      *msfvy = F_(CW_MSFVY), *mvi = F_(CW_MSFVX_INV);
  const double rdx = d->rdx, rdy = d->rdy;
  const double mkrdxm = (AT(msfux, i, j, 0) / AT(msfuy, i, j, 0)) * 0.5 * (AT(xk, i, j, k) + AT(xk, i - 1, j, k)) *
                        0.5 * (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i - 1, j, k)) * rdx;
  const double mkrdxp = (AT(msfux, i + 1, j, 0) / AT(msfuy, i + 1, j, 0)) * 0.5 *
                        (AT(xk, i + 1, j, k) + AT(xk, i, j, k)) * 0.5 *
                        (mk(c1, c2, mut, i + 1, j, k) + mk(c1, c2, mut, i, j, k)) * rdx;
  const double mrdx = AT(msftx, i, j, 0) * AT(msfty, i, j, 0) * rdx;
  const double mkrdym = (AT(msfvy, i, j, 0) * AT(mvi, i, j, 0)) * 0.5 * (AT(xk, i, j, k) + AT(xk, i, j - 1, k)) * 0.5 *
                        (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k)) * rdy;
  const double mkrdyp = (AT(msfvy, i, j + 1, 0) * AT(mvi, i, j + 1, 0)) * 0.5 *
                        (AT(xk, i, j + 1, k) + AT(xk, i, j, k)) * 0.5 *
                        (mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i, j, k)) * rdy;
  const double mrdy = AT(msftx, i, j, 0) * AT(msfty, i, j, 0) * rdy;
  if (!base)
    return mrdx * (mkrdxp * (AT(field, i + 1, j, k) - AT(field, i, j, k)) -
                   mkrdxm * (AT(field, i, j, k) - AT(field, i - 1, j, k))) +
           mrdy * (mkrdyp * (AT(field, i, j + 1, k) - AT(field, i, j, k)) -
                   mkrdym * (AT(field, i, j, k) - AT(field, i, j - 1, k)));
  const double dxp = AT(field, i + 1, j, k) - AT(field, i, j, k) - AT(base, i + 1, j, k) + AT(base, i, j, k);
  const double dxm = AT(field, i, j, k) - AT(field, i - 1, j, k) - AT(base, i, j, k) + AT(base, i - 1, j, k);
  const double dyp = AT(field, i, j + 1, k) - AT(field, i, j, k) - AT(base, i, j + 1, k) + AT(base, i, j, k);
  const double dym = AT(field, i, j, k) - AT(field, i, j - 1, k) - AT(base, i, j, k) + AT(base, i, j - 1, k);
  return mrdx * (mkrdxp * dxp - mkrdxm * dxm) + mrdy * (mkrdyp * dyp - mkrdym * dym);
}

/* horizontal_diffusion's index ranges (big_step_diffusion.hpp:359-395); no open boundaries */
/* horizontal_diffusion's loop limits (big_step_diffusion.hpp:359-398): one row in on the sides that are open or
 * when any side is specified */
static void hdiff_range(or_dom* d, char name, int* is, int* ie, int* js, int* je) {
  const cw_grid* g = &d->g;
  const int sp = specified(g), nx = g->nx, ny = g->ny;
  const int bx = sp || open_x(g), by = sp || open_y(g);
  *is = bx ? 1 : 0;
  *js = by ? 1 : 0;
  if (name == 'u') {
    *ie = bx ? nx : nx + 1;
    *je = by ? ny - 1 : ny;
    if (g->bc_x == CW_BC_PERIODIC) { *is = 0; *ie = nx + 1; }
  } else if (name == 'v') {
    *ie = bx ? nx - 1 : nx;
    *je = by ? ny : ny + 1;
    if (g->bc_x == CW_BC_PERIODIC) { *is = 0; *ie = nx; }
  } else {
    *ie = bx ? nx - 1 : nx;
    *je = by ? ny - 1 : ny;
    if (g->bc_x == CW_BC_PERIODIC) { *is = 0; *ie = nx; }
  }
}

/* vertical diffusion kernels, column by column */
static void vdiff_w(or_dom* d, fld* field, fld* tend, fld* mut, double kv, int i, int j) {
  fld* alt = F_(CW_ALT);
  const int nz = d->g.nz;
  double vflux[256];
  for (int k = 0; k < nz - 1; ++k)
    vflux[k] = (kv / AT(alt, i, j, k)) * d->rdnw[k] * (AT(field, i, j, k + 1) - AT(field, i, j, k));
  vflux[nz - 1] = 0;
  for (int k = 1; k < nz; ++k) {
    const double mu = d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k];
    const double alt_avg = 0.5 * (AT(alt, i, j, k) + AT(alt, i, j, k - 1));
    AT(tend, i, j, k) += d->rdn[k] * G_ * G_ / mu / alt_avg * (vflux[k] - vflux[k - 1]);
  }
}
/* KVertDiffM1 (base NULL) / KVertDiffMP1 (base given) */
static void vdiff_m(or_dom* d, fld* field, fld* base, fld* tend, fld* mut, double kv, int i, int j) {
  fld* alt = F_(CW_ALT);
  const int nz = d->g.nz;
  double vflux[256];
  for (int k = 0; k < nz - 1; ++k) {
    const double dpert = base ? AT(field, i, j, k + 1) - AT(field, i, j, k) - AT(base, i, j, k + 1) + AT(base, i, j, k)
                              : AT(field, i, j, k + 1) - AT(field, i, j, k);
    vflux[k] = kv * d->rdn[k + 1] / (0.5 * (AT(alt, i, j, k) + AT(alt, i, j, k + 1))) * dpert;
  }
  const double vf0 = vflux[0];
  vflux[nz - 1] = 0;
  AT(tend, i, j, 0) +=
      G_ * G_ / (d->c1h[0] * AT(mut, i, j, 0) + d->c2h[0]) / AT(alt, i, j, 0) * d->rdnw[0] * (vflux[0] - vf0);
  for (int k = 1; k < nz; ++k) {
    const double mu = d->c1h[k] * AT(mut, i, j, 0) + d->c2h[k];
    AT(tend, i, j, k) += G_ * G_ / mu / AT(alt, i, j, k) * d->rdnw[k] * (vflux[k] - vflux[k - 1]);
  }
}
/* KVertDiffU1 (DI = 1, DJ = 0, ubase) / KVertDiffV1 (DI = 0, DJ = 1) */
static void vdiff_uv(or_dom* d, fld* field, const double* ubase, fld* muu, fld* tend, double kv, int DI, int DJ, int i,
                     int j) {
  fld* alt = F_(CW_ALT);
  const int nz = d->g.nz;
  double vflux[256];
  for (int k = 0; k < nz - 1; ++k) {
    const double a = 0.25 * (AT(alt, i, j, k) + AT(alt, i - DI, j - DJ, k) + AT(alt, i, j, k + 1) +
                             AT(alt, i - DI, j - DJ, k + 1));
    const double dpert = AT(field, i, j, k + 1) - AT(field, i, j, k) - ubase[k + 1] + ubase[k];
    vflux[k] = kv * d->rdn[k + 1] / a * dpert;
  }
  const double vf0 = vflux[0];
  vflux[nz - 1] = 0;
  AT(tend, i, j, 0) += G_ * G_ * d->rdnw[0] / (d->c1h[0] * AT(muu, i, j, 0) + d->c2h[0]) /
                       (0.5 * (AT(alt, i - DI, j - DJ, 0) + AT(alt, i, j, 0))) * (vflux[0] - vf0);
  for (int k = 1; k < nz - 1; ++k) {
    const double mu = d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k];
    const double a = 0.5 * (AT(alt, i - DI, j - DJ, k) + AT(alt, i, j, k));
    AT(tend, i, j, k) += G_ * G_ * d->rdnw[k] / mu / a * (vflux[k] - vflux[k - 1]);
  }
}

static double prandtl(or_dom* d) { return 1.0 / d->o.pr_inv; }

/* sixth_order_diffusion (src/dyn/diffusion/sixth_order.hpp:13-183), diff_6th_opt 1 (linear) or 2 (flux-limited) */
static double d6_flux(const fld* f, int i, int j, int k, int di, int dj, int opt) {
#define F6(s) AT(f, i + (s) * di, j + (s) * dj, k)
  double dd = 10.0 * (F6(0) - F6(-1)) - 5.0 * (F6(1) - F6(-2)) + (F6(2) - F6(-3));
  if (opt == 2 && dd * (F6(0) - F6(-1)) <= 0) dd = 0;
#undef F6
  return dd;
}
static void sixth_order(or_dom* d, char kind, fld* f, fld* tend, fld* mut, double dt, const double* c1v, const double* c2v) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz, opt = d->o.diff_6th_opt;
  if (opt == 0 || d->o.diff_6th_factor == 0) return;
  const double coef = d->o.diff_6th_factor * 0.015625 / (2.0 * dt);
  const int sp = specified(g), px = g->bc_x == CW_BC_PERIODIC, ox = open_x(g), oy = open_y(g);
  /* loop limits (sixth_order.hpp:174-205): open sides start 3 rows in and end 3 (u, v along their stagger) or 4
   * rows in; 'v' with open x takes the specified limits on all four sides */
  int is = 0, js = 0, ie, je, k0 = 0;
  if (kind == 'u') {
    ie = nx + 1; je = ny;
    if (ox) { is = 3; ie = nx - 2; }
    if (oy) { js = 3; je = ny - 3; }
    if (sp) { is = 3; ie = nx - 2; js = 3; je = ny - 3; }
    if (px) { is = 0; ie = nx + 1; }
  } else if (kind == 'v') {
    ie = nx; je = ny + 1;
    if (ox) { is = 3; ie = nx - 3; }
    if (oy) { js = 3; je = ny - 2; }
    if (ox || sp) { is = 3; ie = nx - 3; js = 3; je = ny - 2; }
    if (px) { is = 0; ie = nx; }
  } else {
    ie = nx; je = ny;
    if (ox) { is = 3; ie = nx - 3; }
    if (oy) { js = 3; je = ny - 3; }
    if (sp) { is = 3; ie = nx - 3; js = 3; je = ny - 3; }
    if (px) { is = 0; ie = nx; }
    if (kind == 'w') k0 = 1;
  }
  fld *sxf, *syf;
  if (kind == 'u') { sxf = F_(CW_MSFUX); syf = F_(CW_MSFUY); }
  else if (kind == 'v') { sxf = F_(CW_MSFVX); syf = F_(CW_MSFVY); }
  else { sxf = F_(CW_MSFTX); syf = F_(CW_MSFTY); }
  for (int k = k0; k < nz; ++k)
    for (int j = js; j < je; ++j)
      for (int i = is; i < ie; ++i) {
        const double c1 = c1v[k], c2 = c2v[k];
#define M6(a, b) (c1 * AT(mut, a, b, 0) + c2)
        const double fx0 = d6_flux(f, i, j, k, 1, 0, opt), fx1 = d6_flux(f, i + 1, j, k, 1, 0, opt);
        const double fy0 = d6_flux(f, i, j, k, 0, 1, opt), fy1 = d6_flux(f, i, j + 1, k, 0, 1, opt);
        double mx0, mx1, my0, my1;
        if (kind == 'u') {
          mx0 = M6(i - 1, j); mx1 = M6(i, j);
          my0 = 0.25 * (M6(i - 1, j - 1) + M6(i, j - 1) + M6(i - 1, j) + M6(i, j));
          my1 = 0.25 * (M6(i - 1, j) + M6(i, j) + M6(i - 1, j + 1) + M6(i, j + 1));
        } else if (kind == 'v') {
          mx0 = 0.25 * (M6(i - 1, j - 1) + M6(i, j - 1) + M6(i - 1, j) + M6(i, j));
          mx1 = 0.25 * (M6(i, j - 1) + M6(i + 1, j - 1) + M6(i, j) + M6(i + 1, j));
          my0 = M6(i, j - 1); my1 = M6(i, j);
        } else {
          mx0 = 0.5 * (M6(i - 1, j) + M6(i, j)); mx1 = 0.5 * (M6(i, j) + M6(i + 1, j));
          my0 = 0.5 * (M6(i, j - 1) + M6(i, j)); my1 = 0.5 * (M6(i, j) + M6(i, j + 1));
        }
#undef M6
        const double tx = coef * AT(sxf, i, j, 0) * (mx1 * fx1 - mx0 * fx0);
        const double ty = coef * AT(syf, i, j, 0) * (my1 * fy1 - my0 * fy0);
        AT(tend, i, j, k) = AT(tend, i, j, k) + tx + ty;
      }
}

/* rk_rayleigh_damp, damp_opt 2 (src/dyn/diffusion/rayleigh_damp.hpp:26-245), column by column; sin: glibc's (libmvec's
 * on the lanes of the vectorised k loops, scalar for w) or cw_sin */
extern __m128d _ZGVbN2v_sin(__m128d);
#define RAY_LEVELS 128
static double ray_sin(const or_dom* d, double x, int lane_k, int nk, int vec) {
  if (d->pow_mode != OR_POW_GLIBC) return cw_sin(x);
  if (vec && nk > 1 && !((nk & 1) && lane_k == nk - 1)) /* vm::lane */ return _mm_cvtsd_f64(_ZGVbN2v_sin(_mm_set1_pd(x)));
  return sin(x);
}
/* the damping of one u / v / theta column: levels from the top while within zdamp, base value interpolated */
static void ray_column(or_dom* d, double ztop, const double* zl, const double* base, const double* mu_k, const double* val,
                       double* tend_k[]) {
  const int ktf = d->g.nz - 1;
  const double pii = 2.0 * asin(1.0);
  double z00[RAY_LEVELS], b00[RAY_LEVELS];
  int k1 = ktf;
  double z = ztop;
  while (k1 >= 0 && z >= (ztop - d->o.zdamp)) {
    z = zl[k1];
    z00[k1] = z;
    k1 = k1 - 1;
  }
  k1 = k1 + 2;
  for (int k = k1; k <= ktf; ++k) {
    int k2 = ktf;
    while (k2 > 0 && d->z_base[k2] > z00[k]) k2 = k2 - 1;
    if (k2 + 1 > ktf)
      b00[k] = base[k2] + (base[k2] - base[k2 - 1]) * (z00[k] - d->z_base[k2]) / (d->z_base[k2] - d->z_base[k2 - 1]);
    else
      b00[k] = base[k2] + (base[k2 + 1] - base[k2]) * (z00[k] - d->z_base[k2]) / (d->z_base[k2 + 1] - d->z_base[k2]);
  }
  const int nk = ktf - k1 + 1;
  for (int k = k1; k <= ktf; ++k) {
    const double ratio = (ztop - z00[k]) / d->o.zdamp;
    const double m = ratio < 1.0 ? ratio : 1.0;
    double dcoef = 1.0 - m;
    const double sn = ray_sin(d, 0.5 * pii * dcoef, k - k1, nk, 1);
    dcoef = sn * sn;
    *tend_k[k] = *tend_k[k] - mu_k[k] * (dcoef * d->o.dampcoef) * (val[k] - b00[k]);
  }
}
static void rayleigh_damp(or_dom* d) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  fld *ph = F_(CW_PH_2), *phb = F_(CW_PHB), *mut = F_(CW_MUT);
  const double pii = 2.0 * asin(1.0);
  double zl[RAY_LEVELS], mu[RAY_LEVELS], val[RAY_LEVELS];
  double* tk[RAY_LEVELS];
  const int px = g->bc_x == CW_BC_PERIODIC, py = g->bc_y == CW_BC_PERIODIC;
  for (int j = 0; j < ny; ++j) /* KRayleighDampU over (i, j) in [0, nx] x [0, ny) */
    for (int i = 0; i <= nx; ++i) {
      const int a = (i == nx) ? (px ? 0 : nx - 1) : i, b = (i == 0) ? (px ? nx - 1 : 0) : i - 1;
      const double ztop = 0.5 * (AT(phb, a, j, nz) + AT(phb, b, j, nz) + AT(ph, a, j, nz) + AT(ph, b, j, nz)) / G_;
      for (int k = 0; k < nz; ++k) {
        zl[k] = 0.25 * (AT(phb, a, j, k) + AT(phb, a, j, k + 1) + AT(phb, b, j, k) + AT(phb, b, j, k + 1) + AT(ph, a, j, k) +
                        AT(ph, a, j, k + 1) + AT(ph, b, j, k) + AT(ph, b, j, k + 1)) / G_;
        mu[k] = d->c1h[k] * AT(F_(CW_MUU), i, j, 0) + d->c2h[k];
        val[k] = AT(F_(CW_U_2), i, j, k);
        tk[k] = &AT(F_(CW_RU_TENDF), i, j, k);
      }
      ray_column(d, ztop, zl, d->u_base, mu, val, tk);
    }
  for (int j = 0; j <= ny; ++j) /* KRayleighDampV over [0, nx) x [0, ny] (in 2-D row ny is row 0's storage) */
    for (int i = 0; i < nx; ++i) {
      const int a = (j == ny) ? (py ? 0 : ny - 1) : j, b = (j == 0) ? (py ? ny - 1 : 0) : j - 1;
      const double ztop = 0.5 * (AT(phb, i, a, nz) + AT(phb, i, b, nz) + AT(ph, i, a, nz) + AT(ph, i, b, nz)) / G_;
      for (int k = 0; k < nz; ++k) {
        zl[k] = 0.25 * (AT(phb, i, a, k) + AT(phb, i, a, k + 1) + AT(phb, i, b, k) + AT(phb, i, b, k + 1) + AT(ph, i, a, k) +
                        AT(ph, i, a, k + 1) + AT(ph, i, b, k) + AT(ph, i, b, k + 1)) / G_;
        mu[k] = d->c1h[k] * AT(F_(CW_MUV), i, j, 0) + d->c2h[k];
        val[k] = AT(F_(CW_V_2), i, j, k);
        tk[k] = &AT(F_(CW_RV_TENDF), i, j, k);
      }
      ray_column(d, ztop, zl, d->v_base, mu, val, tk);
    }
  for (int j = 0; j < ny; ++j) /* KRayleighDampWT */
    for (int i = 0; i < nx; ++i) {
      const double ztop = (AT(phb, i, j, nz) + AT(ph, i, j, nz)) / G_;
      for (int k = 0; k <= nz; ++k) {
        const double z = (AT(phb, i, j, k) + AT(ph, i, j, k)) / G_;
        if (z >= (ztop - d->o.zdamp)) {
          const double ratio = (ztop - z) / d->o.zdamp;
          const double m = ratio < 1.0 ? ratio : 1.0;
          double dcoef = 1.0 - m;
          const double sn = ray_sin(d, 0.5 * pii * dcoef, 0, 1, 0);
          dcoef = sn * sn;
          AT(F_(CW_RW_TENDF), i, j, k) = AT(F_(CW_RW_TENDF), i, j, k) -
                                         (d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k]) * (dcoef * d->o.dampcoef) * AT(F_(CW_W_2), i, j, k);
        }
      }
      for (int k = 0; k < nz; ++k) {
        zl[k] = 0.5 * (AT(phb, i, j, k) + AT(phb, i, j, k + 1) + AT(ph, i, j, k) + AT(ph, i, j, k + 1)) / G_;
        mu[k] = d->c1h[k] * AT(mut, i, j, 0) + d->c2h[k];
        val[k] = AT(F_(CW_T_2), i, j, k);
        tk[k] = &AT(F_(CW_T_TENDF), i, j, k);
      }
      ray_column(d, ztop, zl, d->t_base, mu, val, tk);
    }
}

/* cal_dampkm (km_kh.hpp:485-567, damp_opt 1): near the model top the eddy viscosities rise to
 * dampcoef cos^2(pi/2 min(depth / zdamp, 1)) times ds^2 / dt (horizontal) and dz^2 / dt (vertical), depth below the
 * top accumulated from the diffusion metrics' rdzw / rdz (compute_diff_metrics, diff_metrics.hpp:11-33) of
 * ph_2 + phb; the columns exclude spec_bdy_width - 1 rows of specified boundaries. cos by the pow mode: glibc's
 * (libmvec's 2-lane cos on the lanes of the column loop, vm::lane) or cw_cos. */
#define DK_LEVELS 128
static double damp_cos(const or_dom* d, double x, int lane_i, int ni) {
  if (d->pow_mode != OR_POW_GLIBC) return cw_cos(x);
  if (ni > 1 && !((ni & 1) && lane_i == ni - 1)) return _mm_cvtsd_f64(_ZGVbN2v_cos(_mm_set1_pd(x)));
  return cos(x);
}
static void cal_dampkm(or_dom* d) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  int i0 = 0, i1 = nx, j0 = 0, j1 = ny;
  if (specified(g)) {
    const int w = 5; /* spec_bdy_width */
    i0 = i0 > w - 1 ? i0 : w - 1;
    i1 = i1 < nx - w + 1 ? i1 : nx - w + 1;
    j0 = j0 > w - 1 ? j0 : w - 1;
    j1 = j1 < ny - w + 1 ? j1 : ny - w + 1;
  }
  const int ni = i1 - i0;
  const double piconst = 3.1415926535897932384626433, degrad = piconst / 180.0, degrad90 = degrad * 90.0;
  const double dx = g->dx, dy = g->dy, dt = g->dt, dampcoef = d->o.dampcoef, zdamp = d->o.zdamp;
  fld *ph = F_(CW_PH_2), *phb = F_(CW_PHB), *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY);
  double zw[DK_LEVELS + 1], rdz[DK_LEVELS], rdzw[DK_LEVELS], dampk[DK_LEVELS], dampkv[DK_LEVELS];
  for (int j = j0; j < j1; ++j)
    for (int i = i0; i < i1; ++i) {
      const int lane_i = i - i0;
      for (int k = 0; k <= nz; ++k) zw[k] = (AT(ph, i, j, k) + AT(phb, i, j, k)) / G_;
      for (int k = 0; k < nz; ++k) rdzw[k] = 1.0 / (zw[k + 1] - zw[k]);
      rdz[0] = 2.0 / (zw[1] - zw[0]);
      for (int k = 1; k < nz; ++k) rdz[k] = 2.0 / (zw[k + 1] - zw[k - 1]);
      double deltaz = 0.0;
      for (int k = nz - 1; k >= 0; --k) {
        const double dx_m = dx / AT(msftx, i, j, 0), dy_m = dy / AT(msfty, i, j, 0);
        const double ds = dx_m < dy_m ? dx_m : dy_m;
        const double kmmax = ds * ds / dt;
        double dz;
        if (k == nz - 1) {
          dz = 1.0 / rdzw[k];
          deltaz = 0.5 * dz;
        } else {
          dz = 1.0 / rdz[k];
          deltaz = deltaz + dz;
          dz = 1.0 / rdzw[k];
        }
        const double kmmvmax = dz * dz / dt;
        const double ratio = deltaz / zdamp;
        const double tmp = ratio < 1.0 ? ratio : 1.0;
        const double c = damp_cos(d, degrad90 * tmp, lane_i, ni);
        dampk[k] = c * c * kmmax * dampcoef;
        dampkv[k] = c * c * kmmvmax * dampcoef;
        if (dampk[k] < dampkv[k]) dampkv[k] = dampk[k];
      }
      for (int k = 0; k < nz; ++k) {
        if (dampk[k] > AT(&d->xkmh, i, j, k)) AT(&d->xkmh, i, j, k) = dampk[k];
        if (dampk[k] > AT(&d->xkhh, i, j, k)) AT(&d->xkhh, i, j, k) = dampk[k];
        if (dampkv[k] > AT(&d->xkmv, i, j, k)) AT(&d->xkmv, i, j, k) = dampkv[k];
        if (dampkv[k] > AT(&d->xkhv, i, j, k)) AT(&d->xkhv, i, j, k) = dampkv[k];
      }
    }
}
/* km_opt 4 with diff_opt 1: compute_diff_metrics' rdzw, zx, zy (diff_metrics.hpp:11-133, with set_physical_bc3d),
 * cal_deform_and_div's defor11, defor22, defor12 (deform_div.hpp:20-156, :264-318, the outermost faces of specified /
 * open sides copied from the next ones) and the 2-D Smagorinsky eddy viscosities (KSmag2dKm km_kh.hpp:47-97 over
 * calculate_km_kh's range :585-625, zero on the outermost rows of specified boundaries) */
static void smag2d_km(or_dom* d) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const int px = g->bc_x == CW_BC_PERIODIC, py = g->bc_y == CW_BC_PERIODIC, sp = specified(g);
  const int ox = open_x(g), oy = open_y(g);
  fld *ph = F_(CW_PH_2), *phb = F_(CW_PHB), *u = F_(CW_U_2), *v = F_(CW_V_2);
  fld *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY), *msfuy = F_(CW_MSFUY), *msfvx = F_(CW_MSFVX), *msfux = F_(CW_MSFUX),
      *msfvy = F_(CW_MSFVY);
  const long nzp = nz + 1;
  double* rdzw = (double*)calloc((size_t)nx * ny * nz, sizeof(double));
  double* zx = (double*)calloc((size_t)(nx + 1) * ny * nzp, sizeof(double));
  double* zy = (double*)calloc((size_t)nx * (ny + 1) * nzp, sizeof(double));
  double* d11 = (double*)calloc((size_t)nx * ny * nz, sizeof(double));
  double* d22 = (double*)calloc((size_t)nx * ny * nz, sizeof(double));
  double* d12 = (double*)calloc((size_t)(nx + 1) * (ny + 1) * nz, sizeof(double));
#define RDZW(i, j, k) rdzw[((size_t)(k) * ny + (j)) * nx + (i)]
#define ZX(i, j, k) zx[((size_t)(k) * ny + (j)) * (nx + 1) + (i)]
#define ZY(i, j, k) zy[((size_t)(k) * (ny + 1) + (j)) * nx + (i)]
#define D11(i, j, k) d11[((size_t)(k) * ny + (j)) * nx + (i)]
#define D22(i, j, k) d22[((size_t)(k) * ny + (j)) * nx + (i)]
#define D12(i, j, k) d12[((size_t)(k) * (ny + 1) + (j)) * (nx + 1) + (i)]
  /* metrics */
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const double z0 = (AT(ph, i, j, k) + AT(phb, i, j, k)) / G_, z1 = (AT(ph, i, j, k + 1) + AT(phb, i, j, k + 1)) / G_;
        RDZW(i, j, k) = 1.0 / (z1 - z0);
      }
  const int ktop_x = px ? nz : -1, ktop_y = py ? nz : -1;
  const int ocx = sp || ox, ocy = sp || oy;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        double val;
        if (k == ktop_x && (i == 0 || i == nx)) val = 0.0;
        else if (!px && (i == 0 || (i == nx && !ocx))) val = 0.0;
        else if (!px && i == nx) {
          const int ii = nx - 1;
          val = d->rdx * (AT(phb, ii, j, k) - AT(phb, ii - 1, j, k)) / G_;
          val += d->rdx * (AT(ph, ii, j, k) - AT(ph, ii - 1, j, k)) / G_;
        } else {
          const int i0 = i == nx ? 0 : i, im1 = i == 0 ? nx - 1 : i - 1;
          val = d->rdx * (AT(phb, i0, j, k) - AT(phb, im1, j, k)) / G_;
          val += d->rdx * (AT(ph, i0, j, k) - AT(ph, im1, j, k)) / G_;
        }
        ZX(i, j, k) = val;
      }
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double val;
        if (k == ktop_y && (j == 0 || j == ny)) val = 0.0;
        else if (!py && (j == 0 || (j == ny && !ocy))) val = 0.0;
        else if (!py && j == ny) {
          const int jj = ny - 1;
          val = d->rdy * (AT(phb, i, jj, k) - AT(phb, i, jj - 1, k)) / G_;
          val += d->rdy * (AT(ph, i, jj, k) - AT(ph, i, jj - 1, k)) / G_;
        } else {
          const int j0 = j == ny ? 0 : j, jm1 = j == 0 ? ny - 1 : j - 1;
          val = d->rdy * (AT(phb, i, j0, k) - AT(phb, i, jm1, k)) / G_;
          val += d->rdy * (AT(ph, i, j0, k) - AT(ph, i, jm1, k)) / G_;
        }
        ZY(i, j, k) = val;
      }
  const double cf1 = d->cf1, cf2 = d->cf2, cf3 = d->cf3;
  const double cft2 = -0.5 * d->dnw[nz - 1] / d->dn[nz - 1], cft1 = 1.0 - cft2;
  double a0[DK_LEVELS], a1[DK_LEVELS], av[DK_LEVELS + 1];
  /* hatavg of two columns a0, a1 at the w levels (KDeformDiagAndDiv / KDeform12) */
#define HATAVG()                                                                                                   \
  do {                                                                                                             \
    for (int k = 1; k < nz; ++k) av[k] = 0.5 * (d->fnm[k] * (a0[k] + a1[k]) + d->fnp[k] * (a0[k - 1] + a1[k - 1])); \
    av[0] = 0.5 * (cf1 * a0[0] + cf2 * a0[1] + cf3 * a0[2] + cf1 * a1[0] + cf2 * a1[1] + cf3 * a1[2]);            \
    av[nz] = 0.5 * (cft1 * (a0[nz - 1] + a1[nz - 1]) + cft2 * (a0[nz - 2] + a1[nz - 2]));                         \
  } while (0)
  for (int j = 0; j < ny; ++j) /* KDeformDiagAndDiv: defor11, defor22 */
    for (int i = 0; i < nx; ++i) {
      const double mm = AT(msftx, i, j, 0) * AT(msfty, i, j, 0);
      for (int k = 0; k < nz; ++k) {
        a0[k] = AT(u, i, j, k) / AT(msfuy, i, j, 0);
        a1[k] = AT(u, i + 1, j, k) / AT(msfuy, i + 1, j, 0);
      }
      HATAVG();
      for (int k = 0; k < nz; ++k) {
        const double tmpzx = 0.25 * (ZX(i, j, k) + ZX(i + 1, j, k) + ZX(i, j, k + 1) + ZX(i + 1, j, k + 1));
        const double tmp1 = (av[k + 1] - av[k]) * tmpzx * RDZW(i, j, k);
        D11(i, j, k) = 2.0 * (mm * (d->rdx * (a1[k] - a0[k]) - tmp1));
      }
      for (int k = 0; k < nz; ++k) {
        a0[k] = AT(v, i, j, k) / AT(msfvx, i, j, 0);
        a1[k] = AT(v, i, j + 1, k) / AT(msfvx, i, j + 1, 0);
      }
      HATAVG();
      for (int k = 0; k < nz; ++k) {
        const double tmpzy = 0.25 * (ZY(i, j, k) + ZY(i, j + 1, k) + ZY(i, j, k + 1) + ZY(i, j + 1, k + 1));
        const double tmp1 = (av[k + 1] - av[k]) * tmpzy * RDZW(i, j, k);
        D22(i, j, k) = 2.0 * (mm * (d->rdy * (a1[k] - a0[k]) - tmp1));
      }
    }
  const int bxs = !px && (sp || ox), bxe = bxs, bys = !py && (sp || oy), bye = bys;
  const int i12s = bxs ? 1 : 0, i12e = bxe ? nx : nx + 1, j12s = bys ? 1 : 0, j12e = bye ? ny : ny + 1;
  double b0[DK_LEVELS], b1[DK_LEVELS], bv[DK_LEVELS + 1];
  for (int j = j12s; j < j12e; ++j) /* KDeform12 */
    for (int i = i12s; i < i12e; ++i) {
      const int im1 = i == 0 ? (px ? nx - 1 : 0) : i - 1, i0 = i == nx ? (px ? 0 : nx - 1) : i;
      const int jm1 = j == 0 ? (py ? ny - 1 : 0) : j - 1, j0 = j == ny ? (py ? 0 : ny - 1) : j;
      const double mm = 0.25 * (AT(msfux, i, jm1, 0) + AT(msfux, i, j0, 0)) * (AT(msfvy, im1, j, 0) + AT(msfvy, i0, j, 0));
      for (int k = 0; k < nz; ++k) {
        a0[k] = AT(u, i, jm1, k) / AT(msfux, i, jm1, 0);
        a1[k] = AT(u, i, j0, k) / AT(msfux, i, j0, 0);
      }
      HATAVG();
      for (int k = 0; k <= nz; ++k) bv[k] = av[k];
      for (int k = 0; k < nz; ++k) {
        b0[k] = AT(v, im1, j, k) / AT(msfvy, im1, j, 0);
        b1[k] = AT(v, i0, j, k) / AT(msfvy, i0, j, 0);
      }
      { /* hatavg of v into av (the same statement on b0, b1) */
        for (int k = 1; k < nz; ++k) av[k] = 0.5 * (d->fnm[k] * (b0[k] + b1[k]) + d->fnp[k] * (b0[k - 1] + b1[k - 1]));
        av[0] = 0.5 * (cf1 * b0[0] + cf2 * b0[1] + cf3 * b0[2] + cf1 * b1[0] + cf2 * b1[1] + cf3 * b1[2]);
        av[nz] = 0.5 * (cft1 * (b0[nz - 1] + b1[nz - 1]) + cft2 * (b0[nz - 2] + b1[nz - 2]));
      }
      for (int k = 0; k < nz; ++k) {
        const double tmpzy = 0.25 * (ZY(im1, j, k) + ZY(i0, j, k) + ZY(im1, j, k + 1) + ZY(i0, j, k + 1));
        const double tmp1_u = (bv[k + 1] - bv[k]) * 0.25 * tmpzy *
                              (RDZW(i0, j0, k) + RDZW(im1, j0, k) + RDZW(im1, jm1, k) + RDZW(i0, jm1, k));
        const double term_u = mm * (d->rdy * (a1[k] - a0[k]) - tmp1_u);
        const double tmpzx = 0.25 * (ZX(i, jm1, k) + ZX(i, j0, k) + ZX(i, jm1, k + 1) + ZX(i, j0, k + 1));
        const double tmp1_v = (av[k + 1] - av[k]) * 0.25 * tmpzx *
                              (RDZW(i0, j0, k) + RDZW(i0, jm1, k) + RDZW(im1, jm1, k) + RDZW(im1, j0, k));
        const double term_v = mm * (d->rdx * (b1[k] - b0[k]) - tmp1_v);
        D12(i, j, k) = term_u + term_v;
      }
    }
#undef HATAVG
  /* the edge copies, in the reference's order */
  for (int j = 0; j <= ny; ++j)
    for (int k = 0; k < nz; ++k) {
      if (px) D12(nx, j, k) = D12(0, j, k);
      else if (bxs) D12(0, j, k) = D12(1, j, k);
    }
  for (int i = 0; i <= nx; ++i)
    for (int k = 0; k < nz; ++k) {
      if (py) D12(i, ny, k) = D12(i, 0, k);
      else if (bys) D12(i, 0, k) = D12(i, 1, k);
    }
  if (bxe)
    for (int j = 0; j <= ny; ++j)
      for (int k = 0; k < nz; ++k) D12(nx, j, k) = D12(nx - 1, j, k);
  if (bye)
    for (int i = 0; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) D12(i, ny, k) = D12(i, ny - 1, k);
  /* KSmag2dKm */
  int is = (ox || sp) ? 1 : 0, ie = (ox || sp) ? nx - 1 : nx;
  const int js = (oy || sp) ? 1 : 0, je = (oy || sp) ? ny - 1 : ny;
  if (px) { is = 0; ie = nx; }
  const double c_s = 0.25, pr = prandtl(d), dx = g->dx, dy = g->dy;
  for (int k = 0; k < nz; ++k)
    for (int j = js; j < je; ++j)
      for (int i = is; i < ie; ++i) {
        const double dd = D11(i, j, k) - D22(i, j, k);
        double def2 = 0.25 * (dd * dd);
        const double d12a = 0.25 * (D12(i, j, k) + D12(i, j + 1, k) + D12(i + 1, j, k) + D12(i + 1, j + 1, k));
        def2 += d12a * d12a;
        const double mlen_h = sqrt(dx / AT(msftx, i, j, 0) * dy / AT(msfty, i, j, 0));
        const double tmp = sqrt(def2);
        double kmh = c_s * c_s * mlen_h * mlen_h * tmp;
        kmh = kmh < 10.0 * mlen_h ? kmh : 10.0 * mlen_h;
        AT(&d->xkmh, i, j, k) = kmh;
        AT(&d->xkmv, i, j, k) = kmh;
        AT(&d->xkhh, i, j, k) = kmh / pr;
        AT(&d->xkhv, i, j, k) = 0.0;
      }
  if (sp) {
    for (int side = 0; side < 2; ++side)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const int ic = side == 0 ? 0 : nx - 1;
          AT(&d->xkmh, ic, j, k) = AT(&d->xkmv, ic, j, k) = AT(&d->xkhh, ic, j, k) = AT(&d->xkhv, ic, j, k) = 0.0;
        }
    for (int side = 0; side < 2; ++side)
      for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k) {
          const int jc = side == 0 ? 0 : ny - 1;
          AT(&d->xkmh, i, jc, k) = AT(&d->xkmv, i, jc, k) = AT(&d->xkhh, i, jc, k) = AT(&d->xkhv, i, jc, k) = 0.0;
        }
  }
#undef RDZW
#undef ZX
#undef ZY
#undef D11
#undef D22
#undef D12
  free(rdzw);
  free(zx);
  free(zy);
  free(d11);
  free(d22);
  free(d12);
}
static void diffusion_prepare(or_dom* d) {
  const cw_grid* g = &d->g;
  const double pr = prandtl(d);
  if (d->o.km_opt == 4) {
    smag2d_km(d);
  } else {
    for (int k = 0; k < g->nz; ++k)
      for (int j = 0; j < g->ny; ++j)
        for (int i = 0; i < g->nx; ++i) {
          AT(&d->xkmh, i, j, k) = d->o.khdif;
          AT(&d->xkmv, i, j, k) = d->o.kvdif;
          AT(&d->xkhh, i, j, k) = d->o.khdif / pr;
          AT(&d->xkhv, i, j, k) = d->o.kvdif / pr;
        }
  }
  if (d->o.damp_opt == 1) cal_dampkm(d);
  fill_halo(d, &d->xkmh);
  fill_halo(d, &d->xkmv);
  fill_halo(d, &d->xkhh);
  fill_halo(d, &d->xkhv);
}

static void diffusion_dynamics(or_dom* d) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz, do_y = !two_d(g);
  int is, ie, js, je;
  fld *mut = F_(CW_MUT);
  if (d->o.diff_opt == 1) {
    hdiff_range(d, 'u', &is, &ie, &js, &je);
    for (int k = 0; k < nz; ++k)
      for (int j = js; j < je; ++j)
        for (int i = is; i < ie; ++i)
          AT(F_(CW_RU_TENDF), i, j, k) += hdiff_u(d, F_(CW_U_2), mut, &d->xkmh, d->c1h, d->c2h, i, j, k);
    if (do_y) {
      hdiff_range(d, 'v', &is, &ie, &js, &je);
      for (int k = 0; k < nz; ++k)
        for (int j = js; j < je; ++j)
          for (int i = is; i < ie; ++i)
            AT(F_(CW_RV_TENDF), i, j, k) += hdiff_v(d, F_(CW_V_2), mut, &d->xkmh, d->c1h, d->c2h, i, j, k);
    }
    hdiff_range(d, 'w', &is, &ie, &js, &je);
    for (int k = 1; k < nz; ++k)
      for (int j = js; j < je; ++j)
        for (int i = is; i < ie; ++i)
          AT(F_(CW_RW_TENDF), i, j, k) += hdiff_w(d, F_(CW_W_2), mut, &d->xkmh, d->c1f, d->c2f, i, j, k);
    hdiff_range(d, 'm', &is, &ie, &js, &je);
    for (int k = 0; k < nz; ++k)
      for (int j = js; j < je; ++j)
        for (int i = is; i < ie; ++i)
          AT(F_(CW_T_TENDF), i, j, k) += hdiff_m(d, F_(CW_T_2), F_(CW_T_INIT), mut, &d->xkhh, d->c1h, d->c2h, i, j, k);
    { /* vertical_diffusion_u (big_step_diffusion.hpp:459-479) */
      const int bx = specified(g) || open_x(g);
      int vis = bx ? 1 : 0, vie = bx ? nx : nx + 1;
      if (g->bc_x == CW_BC_PERIODIC) { vis = 0; vie = nx + 1; }
      for (int j = 0; j < ny; ++j)
        for (int i = vis; i < vie; ++i)
          vdiff_uv(d, F_(CW_U_2), d->u_base, F_(CW_MUU), F_(CW_RU_TENDF), d->o.kvdif, 1, 0, i, j);
    }
    if (do_y) { /* vertical_diffusion_v (:481-500) */
      const int by = specified(g) || open_y(g);
      const int vjs = by ? 1 : 0, vje = by ? ny : ny + 1;
      for (int j = vjs; j < vje; ++j)
        for (int i = 0; i < nx; ++i)
          vdiff_uv(d, F_(CW_V_2), d->v_base, F_(CW_MUV), F_(CW_RV_TENDF), d->o.kvdif, 0, 1, i, j);
    }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) vdiff_w(d, F_(CW_W_2), F_(CW_RW_TENDF), mut, d->o.kvdif, i, j);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) vdiff_m(d, F_(CW_T_2), F_(CW_T_INIT), F_(CW_T_TENDF), mut, 3. * d->o.kvdif, i, j);
  }
  /* the sixth-order filter after the second-order terms (diffusion_driver.cpp:266-280) */
  sixth_order(d, 'u', F_(CW_U_2), F_(CW_RU_TENDF), mut, g->dt, d->c1h, d->c2h);
  if (do_y) sixth_order(d, 'v', F_(CW_V_2), F_(CW_RV_TENDF), mut, g->dt, d->c1h, d->c2h);
  sixth_order(d, 'w', F_(CW_W_2), F_(CW_RW_TENDF), mut, g->dt, d->c1f, d->c2f);
  sixth_order(d, 'm', F_(CW_T_2), F_(CW_T_TENDF), mut, g->dt, d->c1h, d->c2h);
  if (d->o.damp_opt == 2) rayleigh_damp(d); /* after the diffusion (diffusion_driver.cpp:281-289) */
}

static void diffusion_scalar(or_dom* d, int n) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  fld *q = &d->q2[n], *tend = &d->qtf[n], *muts = F_(CW_MUTS);
  int is, ie, js, je;
  if (d->o.diff_opt == 1) {
    hdiff_range(d, 'm', &is, &ie, &js, &je);
    for (int k = 0; k < nz; ++k)
      for (int j = js; j < je; ++j)
        for (int i = is; i < ie; ++i) AT(tend, i, j, k) += hdiff_m(d, q, NULL, muts, &d->xkhh, d->c1h, d->c2h, i, j, k);
    const double kvdq = d->o.kvdif / prandtl(d);
    const int is_qv = n < d->o.n_moist && n == 0; /* qv is the first moist species */
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) vdiff_m(d, q, is_qv ? F_(CW_QV_BASE) : NULL, tend, muts, kvdq, i, j);
  }
  sixth_order(d, 'm', q, tend, muts, g->dt / 3.0, d->c1h, d->c2h); /* rk 1: dt_rk = dt / 3, muts */
}

/* ------------------------------------------------------------------ lateral boundaries
 * LateralBC (src/dyn/lateral_bc.cpp:21-196 kernels, :294-455 methods): the boundary ring,
 * slabs (pos, k, b) with pos fastest; side order S, N, W, E = slabs ys, ye, xs, xe. */
static int slab_of_side(int side) { return side < 2 ? side + 2 : side - 2; }
typedef struct {
  int ibe, jbe;
} ring_t;
static ring_t ring_for(const cw_grid* g, char var) {
  ring_t r = {var == 'u' ? g->nx : g->nx - 1, var == 'v' ? g->ny : g->ny - 1};
  return r;
}
static int ring_map(const ring_t* r, int pos, int side, int b, int* i, int* j) {
  switch (side) {
    case 0: *j = b; *i = pos; return pos >= b && pos <= r->ibe - b;
    case 1: *j = r->jbe - b; *i = pos; return pos >= b && pos <= r->ibe - b;
    case 2: *i = b; *j = pos; return pos >= b + 1 && pos <= r->jbe - b - 1;
    default: *i = r->ibe - b; *j = pos; return pos >= b + 1 && pos <= r->jbe - b - 1;
  }
}
static double slab_at(const slabset* s, int half, int sl, int pos, int k, int b) {
  const int np = s->npos[sl];
  return s->d[s->off[half * 4 + sl] + (size_t)pos + (size_t)k * np + (size_t)b * np * s->nk];
}
static double slab_val(const slabset* s, int sl, int pos, int k, int b, double dtbc) {
  return slab_at(s, 0, sl, pos, k, b) + dtbc * slab_at(s, 1, sl, pos, k, b);
}
#define RING_LOOP(r, nk, b0, nb)                                                 \
  for (int sb = 0; sb < 4 * (nb); ++sb)                                          \
    for (int k = 0; k < (nk); ++k)                                               \
      for (int pos = 0; pos < ((r).ibe > (r).jbe ? (r).ibe : (r).jbe) + 1; ++pos) { \
        const int side = sb % 4, b = (b0) + sb / 4;                             \
        int i, j;                                                                \
        if (!ring_map(&(r), pos, side, b, &i, &j)) continue;

#define RING_END }

/* KRelax: f3 (or f2) = model field; massw: times (c1*mut + c2); out += val [* msf] or direct */
static void relax_one(or_dom* d, fld* out, fld* f, int two, const double* c1, const double* c2, fld* msf,
                      const slabset* s, char var, int nk, int direct) {
  const ring_t r = ring_for(&d->g, var);
  fld* mut = F_(CW_MUT);
  RING_LOOP(r, nk, 1, 3)
  const int sl = slab_of_side(side);
#define BV(p, bb) slab_val(s, sl, (p), k, (bb), d->dtbc)
#define FV(ii, jj) (c1 ? (two ? AT(f, ii, jj, 0) : AT(f, ii, jj, k)) * (c1[k] * AT(mut, ii, jj, 0) + c2[k]) \
                       : (two ? AT(f, ii, jj, 0) : AT(f, ii, jj, k)))
  double fls0, fls1, fls2, fls3, fls4;
  fls0 = BV(pos, b) - FV(i, j);
  if (side <= 1) {
    const int im1 = i - 1 > 0 ? i - 1 : 0, ip1 = i + 1 < r.ibe ? i + 1 : r.ibe;
    const int jin = side == 0 ? j + 1 : j - 1, jout = side == 0 ? j - 1 : j + 1;
    fls1 = BV(im1, b) - FV(im1, j);
    fls2 = BV(ip1, b) - FV(ip1, j);
    fls3 = BV(i, b - 1) - FV(i, jout);
    fls4 = BV(i, b + 1) - FV(i, jin);
  } else {
    const int iin = side == 2 ? i + 1 : i - 1, iout = side == 2 ? i - 1 : i + 1;
    fls1 = BV(j - 1, b) - FV(i, j - 1);
    fls2 = BV(j + 1, b) - FV(i, j + 1);
    fls3 = BV(j, b - 1) - FV(iout, j);
    fls4 = BV(j, b + 1) - FV(iin, j);
  }
#undef BV
#undef FV
  const double val = d->fcx[b] * fls0 - d->gcx[b] * (fls1 + fls2 + fls3 + fls4 - 4.0 * fls0);
  if (two) AT(out, i, j, 0) += val;
  else if (direct)
    AT(out, i, j, k) = AT(out, i, j, k) + d->fcx[b] * fls0 - d->gcx[b] * (fls1 + fls2 + fls3 + fls4 - 4.0 * fls0);
  else AT(out, i, j, k) += msf ? val * AT(msf, i, j, 0) : val;
  RING_END
}

static void lbc_relax_dry(or_dom* d) {
  const int nz = d->g.nz;
  relax_one(d, F_(CW_RU_TENDF), F_(CW_RU), 0, NULL, NULL, F_(CW_MSFUY), &d->lbc[CW_LBC_U], 'u', nz, 0);
  relax_one(d, F_(CW_RV_TENDF), F_(CW_RV), 0, NULL, NULL, F_(CW_MSFVX), &d->lbc[CW_LBC_V], 'v', nz, 0);
  relax_one(d, F_(CW_PH_TENDF), F_(CW_PH_2), 0, d->c1f, d->c2f, NULL, &d->lbc[CW_LBC_PH], 'h', nz + 1, 0);
  relax_one(d, F_(CW_T_TENDF), F_(CW_T_2), 0, d->c1h, d->c2h, NULL, &d->lbc[CW_LBC_T], 't', nz, 0);
  relax_one(d, F_(CW_MU_TEND), F_(CW_MU_2), 1, NULL, NULL, NULL, &d->lbc[CW_LBC_MU], 'm', 1, 0);
}
/* KSpecTend */
static void spec_one(or_dom* d, fld* out, int two, const slabset* s, char var, int nk) {
  const ring_t r = ring_for(&d->g, var);
  RING_LOOP(r, nk, 0, 1)
  const double v = slab_at(s, 1, slab_of_side(side), pos, k, b);
  if (two) AT(out, i, j, 0) = v;
  else AT(out, i, j, k) = v;
  RING_END
}
static void lbc_spec_dry(or_dom* d) {
  const int nz = d->g.nz;
  spec_one(d, F_(CW_RU_TEND), 0, &d->lbc[CW_LBC_U], 'u', nz);
  spec_one(d, F_(CW_RV_TEND), 0, &d->lbc[CW_LBC_V], 'v', nz);
  spec_one(d, F_(CW_PH_TEND), 0, &d->lbc[CW_LBC_PH], 'h', nz + 1);
  spec_one(d, F_(CW_T_TEND), 0, &d->lbc[CW_LBC_T], 't', nz);
  spec_one(d, F_(CW_MU_TEND), 1, &d->lbc[CW_LBC_MU], 'm', 1);
}
/* KUpdate */
static void update_one(or_dom* d, fld* f, fld* t, int two, char var, int nk, double dts) {
  const ring_t r = ring_for(&d->g, var);
  RING_LOOP(r, nk, 0, 1)
  if (two) AT(f, i, j, 0) += dts * AT(t, i, j, 0);
  else AT(f, i, j, k) += dts * AT(t, i, j, k);
  RING_END
}
static void lbc_update_uv(or_dom* d, double dts) {
  update_one(d, F_(CW_U_2), F_(CW_RU_TEND), 0, 'u', d->g.nz, dts);
  update_one(d, F_(CW_V_2), F_(CW_RV_TEND), 0, 'v', d->g.nz, dts);
}
static void lbc_update_mu_t(or_dom* d, double dts) {
  update_one(d, F_(CW_T_2), F_(CW_T_TEND), 0, 't', d->g.nz, dts);
  update_one(d, F_(CW_MU_2), F_(CW_MU_TEND), 1, 't', 1, dts);
  update_one(d, F_(CW_MUTS), F_(CW_MU_TEND), 1, 't', 1, dts);
}
static void lbc_update_ph_w(or_dom* d, double dts) {
  const ring_t r = ring_for(&d->g, 'h');
  fld *ph = F_(CW_PH_2), *pht = F_(CW_PH_TEND), *mt = F_(CW_MU_TEND), *muts = F_(CW_MUTS), *w = F_(CW_W_2);
  RING_LOOP(r, d->g.nz + 1, 0, 1) /* KUpdatePh */
  const double mu_old = AT(muts, i, j, 0) - dts * AT(mt, i, j, 0);
  const double m_old = d->c1f[k] * mu_old + d->c2f[k], m_new = d->c1f[k] * AT(muts, i, j, 0) + d->c2f[k];
  AT(ph, i, j, k) = AT(ph, i, j, k) * m_old / m_new + dts * AT(pht, i, j, k) / m_new +
                    AT(&d->ph_save, i, j, k) * (m_old / m_new - 1.0);
  RING_END
  RING_LOOP(r, d->g.nz + 1, 0, 1) /* KZeroGrad */
  const int ic = i < 1 ? 1 : (i > r.ibe - 1 ? r.ibe - 1 : i);
  const int jc = j < 1 ? 1 : (j > r.jbe - 1 ? r.jbe - 1 : j);
  switch (side) {
    case 0: AT(w, i, j, k) = AT(w, ic, 1, k); break;
    case 1: AT(w, i, j, k) = AT(w, ic, r.jbe - 1, k); break;
    case 2: AT(w, i, j, k) = AT(w, 1, jc, k); break;
    default: AT(w, i, j, k) = AT(w, r.ibe - 1, jc, k); break;
  }
  RING_END
}
static void lbc_flow_dep(or_dom* d, int n) {
  const ring_t r = ring_for(&d->g, 'q');
  fld *f = &d->q2[n], *u = F_(CW_RU_M), *v = F_(CW_RV_M);
  RING_LOOP(r, d->g.nz, 0, 1)
  const int ic = i < 1 ? 1 : (i > r.ibe - 1 ? r.ibe - 1 : i);
  const int jc = j < 1 ? 1 : (j > r.jbe - 1 ? r.jbe - 1 : j);
  switch (side) {
    case 0: AT(f, i, j, k) = AT(v, i, j, k) < 0.0 ? AT(f, ic, 1, k) : 0.0; break;
    case 1: AT(f, i, j, k) = AT(v, i, j + 1, k) > 0.0 ? AT(f, ic, r.jbe - 1, k) : 0.0; break;
    case 2: AT(f, i, j, k) = AT(u, i, j, k) < 0.0 ? AT(f, 1, jc, k) : 0.0; break;
    default: AT(f, i, j, k) = AT(u, i + 1, j, k) > 0.0 ? AT(f, r.ibe - 1, jc, k) : 0.0; break;
  }
  RING_END
}
/* KFinal */
static void final_one(or_dom* d, fld* f, int two, fld* mu, const double* c1, const double* c2, int mucouple, fld* msf,
                      int msfcouple, const slabset* s, char var, int nk) {
  const ring_t r = ring_for(&d->g, var);
  RING_LOOP(r, nk, 0, 1)
  const double bval = slab_val(s, slab_of_side(side), pos, k, b, d->dtbc);
  const double xmsf = msfcouple ? AT(msf, i, j, 0) : 1.0;
  const double xmu = mucouple ? (c1[k] * AT(mu, i, j, 0) + c2[k]) : 1.0;
  const double v = xmsf * bval / xmu;
  if (two) AT(f, i, j, 0) = v;
  else AT(f, i, j, k) = v;
  RING_END
}
static void lbc_final(or_dom* d) {
  const int nz = d->g.nz;
  final_one(d, F_(CW_U_2), 0, F_(CW_MUUS), d->c1h, d->c2h, 1, F_(CW_MSFUY), 1, &d->lbc[CW_LBC_U], 'u', nz);
  final_one(d, F_(CW_V_2), 0, F_(CW_MUVS), d->c1h, d->c2h, 1, F_(CW_MSFVX), 1, &d->lbc[CW_LBC_V], 'v', nz);
  final_one(d, F_(CW_T_2), 0, F_(CW_MUTS), d->c1h, d->c2h, 1, F_(CW_MSFTY), 0, &d->lbc[CW_LBC_T], 't', nz);
  final_one(d, F_(CW_PH_2), 0, F_(CW_MUTS), d->c1f, d->c2f, 1, F_(CW_MSFTY), 0, &d->lbc[CW_LBC_PH], 'h', nz + 1);
  final_one(d, F_(CW_MU_2), 1, F_(CW_MUTS), d->c1h, d->c2h, 0, F_(CW_MSFTY), 0, &d->lbc[CW_LBC_MU], 'm', 1);
  for (int n = 0; n < d->o.n_scalars; ++n)
    if (d->lbcq[n].have)
      final_one(d, &d->q2[n], 0, F_(CW_MUTS), d->c1h, d->c2h, 1, F_(CW_MSFTY), 0, &d->lbcq[n], 't', nz);
}

/* ------------------------------------------------------------------ small step
 * SmallStep::run_stage (src/dyn/small_step.cpp:490-607) and its kernels (:50-453) */
typedef struct {
  int x, y, nx, ny;
} edge_t;
static int edge_mass(const edge_t* e, int i, int j) {
  return (e->x && (i == 0 || i == e->nx - 1)) || (e->y && (j == 0 || j == e->ny - 1));
}
static int edge_uface(const edge_t* e, int i, int j) {
  return (e->x && (i <= 0 || i >= e->nx)) || (e->y && (j == 0 || j == e->ny - 1));
}
static int edge_vface(const edge_t* e, int i, int j) {
  return (e->x && (i == 0 || i == e->nx - 1)) || (e->y && (j <= 0 || j >= e->ny));
}

/* p_rho_point (:97-112) */
static void p_rho_point(or_dom* d, int i, int j, int k, double smdiv, int damp) {
  fld *al = F_(CW_AL), *p = F_(CW_P), *ph = F_(CW_PH_2), *alt = F_(CW_ALT), *t = F_(CW_T_2), *mu = F_(CW_MU_2),
      *muts = F_(CW_MUTS);
  fld *pm1 = &d->pm1, *ts = &d->t_save, *c2a = &d->c2a;
  const double m = d->c1h[k] * AT(muts, i, j, 0) + d->c2h[k];
  const double a =
      -((1. / m) * (AT(alt, i, j, k) * (d->c1h[k] * AT(mu, i, j, 0)) + d->rdnw[k] * (AT(ph, i, j, k + 1) - AT(ph, i, j, k))));
  AT(al, i, j, k) = a;
  double pp = AT(c2a, i, j, k) * (AT(alt, i, j, k) * (AT(t, i, j, k) - d->c1h[k] * AT(mu, i, j, 0) * AT(ts, i, j, k)) /
                                      (m * (T0 + AT(ts, i, j, k))) -
                                  a);
  if (damp) {
    const double ptmp = pp;
    pp = pp + smdiv * (pp - AT(pm1, i, j, k));
    AT(pm1, i, j, k) = ptmp;
  } else {
    AT(pm1, i, j, k) = pp;
  }
  AT(p, i, j, k) = pp;
}

static double mh_(or_dom* d, int k, double m) { return d->c1h[k] * m + d->c2h[k]; }
static double mf_(or_dom* d, int k, double m) { return d->c1f[k] * m + d->c2f[k]; }

/* advance_uv's dp (:156-173) */
static double uv_ps(or_dom* d, int DI, int DJ, int i, int j, int k) {
  return AT(F_(CW_P), i, j, k) + AT(F_(CW_P), i - DI, j - DJ, k);
}
static double uv_dpn(or_dom* d, int DI, int DJ, int i, int j, int k) {
  const int nz = d->g.nz;
  if (k == 0)
    return H * (d->cf1 * uv_ps(d, DI, DJ, i, j, 0) + d->cf2 * uv_ps(d, DI, DJ, i, j, 1) + d->cf3 * uv_ps(d, DI, DJ, i, j, 2));
  if (k == nz)
    return d->o.top_lid ? H * (d->cf1 * uv_ps(d, DI, DJ, i, j, nz - 1) + d->cf2 * uv_ps(d, DI, DJ, i, j, nz - 2) +
                               d->cf3 * uv_ps(d, DI, DJ, i, j, nz - 3))
                        : 0.0;
  return H * (d->fnm[k] * uv_ps(d, DI, DJ, i, j, k) + d->fnp[k] * uv_ps(d, DI, DJ, i, j, k - 1));
}
static double uv_dp(or_dom* d, int DI, int DJ, int i, int j, int k, double mface, double rd, double rm) {
  fld *ph = F_(CW_PH_2), *alt = F_(CW_ALT), *p = F_(CW_P), *al = F_(CW_AL), *pb = F_(CW_PB), *php = F_(CW_PHP),
      *mu = F_(CW_MU_2);
  double dd = rm * H * rd * (d->c1h[k] * mface + d->c2h[k]) *
              (((AT(ph, i, j, k + 1) - AT(ph, i - DI, j - DJ, k + 1)) + (AT(ph, i, j, k) - AT(ph, i - DI, j - DJ, k))) +
               (AT(alt, i, j, k) + AT(alt, i - DI, j - DJ, k)) * (AT(p, i, j, k) - AT(p, i - DI, j - DJ, k)) +
               (AT(al, i, j, k) + AT(al, i - DI, j - DJ, k)) * (AT(pb, i, j, k) - AT(pb, i - DI, j - DJ, k)));
  dd += rm * rd * (AT(php, i, j, k) - AT(php, i - DI, j - DJ, k)) *
        (d->rdnw[k] * (uv_dpn(d, DI, DJ, i, j, k + 1) - uv_dpn(d, DI, DJ, i, j, k)) -
         H * (d->c1h[k] * AT(mu, i - DI, j - DJ, 0) + d->c1h[k] * AT(mu, i, j, 0)));
  return dd;
}

/* KWCommon (:295-320) */
static double wc_t2ave(or_dom* d, int i, int j, int k) {
  const double epssm = d->o.epssm;
  const double tav = H * ((1.0 + epssm) * AT(F_(CW_T_2), i, j, k) + (1.0 - epssm) * AT(&d->t_2save, i, j, k));
  return (tav + d->c1h[k] * AT(&d->muave, i, j, 0) * T0) /
         (mh_(d, k, AT(F_(CW_MUTS), i, j, 0)) * (T0 + AT(&d->t_save, i, j, k)));
}
static double wc_wdwn(or_dom* d, int i, int j, int m) {
  fld *ww = F_(CW_WW), *phs = &d->ph_save, *phb = F_(CW_PHB);
  return H * (AT(ww, i, j, m) + AT(ww, i, j, m - 1)) * d->rdnw[m - 1] *
         (AT(phs, i, j, m) - AT(phs, i, j, m - 1) + AT(phb, i, j, m) - AT(phb, i, j, m - 1));
}
static double wc_rhs(or_dom* d, int i, int j, int k, double dts) {
  const int nz = d->g.nz;
  const double epssm = d->o.epssm;
  if (k == 0) return 0;
  if (d->o.top_lid && k == nz) return 0;
  double r = dts * (AT(F_(CW_PH_TEND), i, j, k) + H * G_ * (1.0 - epssm) * AT(F_(CW_W_2), i, j, k));
  if (k < nz) r -= dts * (d->fnm[k] * wc_wdwn(d, i, j, k + 1) + d->fnp[k] * wc_wdwn(d, i, j, k));
  return AT(F_(CW_PH_2), i, j, k) + AT(F_(CW_MSFTY), i, j, 0) * r / mf_(d, k, AT(F_(CW_MUT), i, j, 0));
}

static void small_run_stage(or_dom* d, double dts, int n_small, int rk_step) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz, nyv = nys(g, ST_V), do_y = !two_d(g);
  const double epssm = d->o.epssm, smdiv = d->o.smdiv;
  const edge_t ed = {g->bc_x == CW_BC_SPECIFIED, g->bc_y == CW_BC_SPECIFIED && do_y, nx, ny};
  fld *u = F_(CW_U_2), *v = F_(CW_V_2), *w = F_(CW_W_2), *t = F_(CW_T_2), *ph = F_(CW_PH_2), *mu = F_(CW_MU_2);
  fld *u1 = F_(CW_U_1), *v1 = F_(CW_V_1), *w1 = F_(CW_W_1), *t1 = F_(CW_T_1), *ph1 = F_(CW_PH_1), *mu1 = F_(CW_MU_1);
  fld *mut = F_(CW_MUT), *muu = F_(CW_MUU), *muv = F_(CW_MUV), *muts = F_(CW_MUTS), *muus = F_(CW_MUUS),
      *muvs = F_(CW_MUVS);
  fld *mub = F_(CW_MUB), *pb = F_(CW_PB), *p = F_(CW_P), *alt = F_(CW_ALT), *ww = F_(CW_WW);
  fld *msfuy = F_(CW_MSFUY), *mvi = F_(CW_MSFVX_INV), *msfty = F_(CW_MSFTY), *msftx = F_(CW_MSFTX),
      *msfux = F_(CW_MSFUX), *msfvx = F_(CW_MSFVX), *msfvy = F_(CW_MSFVY);
  if (rk_step == 1) fld_fill(&d->mudf, 0.0); /* every point of the allocation, the halo too */
  /* KPrep */
  for (int k = 0; k < nz + 1; ++k)
    for (int j = 0; j < nyv; ++j)
      for (int i = 0; i < nx + 1; ++i) {
        const int first = rk_step == 1;
        const double mts = AT(mub, i, j, 0) + AT(mu1, i, j, 0);
        const double mus_u = first ? AT(muu, i, j, 0) : H * (mts + AT(mub, i - 1, j, 0) + AT(mu1, i - 1, j, 0));
        const double mus_v = first ? AT(muv, i, j, 0) : H * (mts + AT(mub, i, j - 1, 0) + AT(mu1, i, j - 1, 0));
        if (k == 0) {
          if (i < nx && j < ny) {
            AT(muts, i, j, 0) = mts;
            AT(&d->mu_save, i, j, 0) = AT(mu, i, j, 0);
            AT(mu, i, j, 0) = AT(mu1, i, j, 0) - AT(mu, i, j, 0);
          }
          if (j < ny) AT(muus, i, j, 0) = mus_u;
          if (i < nx && j < nyv) AT(muvs, i, j, 0) = mus_v;
        }
        if (j < ny && k < nz) {
          const double ui = AT(u, i, j, k);
          AT(&d->u_save, i, j, k) = ui;
          AT(u, i, j, k) = ((d->c1h[k] * mus_u + d->c2h[k]) * AT(u1, i, j, k) - (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k]) * ui) /
                           AT(msfuy, i, j, 0);
        }
        if (i < nx && j < nyv && k < nz) {
          const double vi = AT(v, i, j, k);
          AT(&d->v_save, i, j, k) = vi;
          AT(v, i, j, k) = ((d->c1h[k] * mus_v + d->c2h[k]) * AT(v1, i, j, k) - (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k]) * vi) *
                           AT(mvi, i, j, 0);
        }
        if (i < nx && j < ny) {
          if (k < nz) {
            const double ti = AT(t, i, j, k);
            AT(&d->t_save, i, j, k) = ti;
            AT(t, i, j, k) = (d->c1h[k] * mts + d->c2h[k]) * AT(t1, i, j, k) - (d->c1h[k] * AT(mut, i, j, 0) + d->c2h[k]) * ti;
            AT(&d->c2a, i, j, k) = CPOVCV * (AT(pb, i, j, k) + AT(p, i, j, k)) / AT(alt, i, j, k);
          }
          const double wi = AT(w, i, j, k), phi = AT(ph, i, j, k);
          AT(&d->w_save, i, j, k) = wi;
          AT(w, i, j, k) = ((d->c1f[k] * mts + d->c2f[k]) * AT(w1, i, j, k) - (d->c1f[k] * AT(mut, i, j, 0) + d->c2f[k]) * wi) /
                           AT(msfty, i, j, 0);
          AT(&d->ph_save, i, j, k) = phi;
          AT(ph, i, j, k) = AT(ph1, i, j, k) - phi;
          AT(&d->ww1, i, j, k) = (k == 0 || k == nz) ? 0.0 : AT(ww, i, j, k);
        }
      }
  fill_halo(d, u);
  fill_halo(d, v);
  fill_halo(d, ph);
  fill_halo(d, &d->t_save);
  fill_halo(d, &d->u_save);
  fill_halo(d, &d->v_save);
  fill_halo(d, mu);
  fill_halo(d, muts);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) p_rho_point(d, i, j, k, 0.0, 0); /* KPRho */
  fill_halo(d, p);
  fill_halo(d, F_(CW_AL));
  { /* KCoefW (:122-148) */
    const double cof_h = 0.5 * dts * G_ * (1.0 + epssm);
    const double cof = cof_h * cof_h;
    const double lid = d->o.top_lid ? 0.0 : 1.0;
    fld *a = &d->a, *alpha = &d->alpha, *gamma = &d->gamma, *c2a = &d->c2a;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double m = AT(mut, i, j, 0);
        AT(a, i, j, 0) = 0;
        AT(alpha, i, j, 0) = 0;
        AT(gamma, i, j, 0) = 0;
        AT(a, i, j, 1) = 0;
        AT(a, i, j, nz) = -2.0 * cof * (d->rdnw[nz - 1] * d->rdnw[nz - 1]) * AT(c2a, i, j, nz - 1) * lid /
                          (mh_(d, nz - 1, m) * mf_(d, nz - 1, m));
        for (int k = 2; k < nz; ++k)
          AT(a, i, j, k) = -cq1_(d, i, j, k) * cof * d->rdn[k] * d->rdnw[k - 1] * AT(c2a, i, j, k - 1) /
                           (mh_(d, k - 1, m) * mf_(d, k - 1, m));
        for (int k = 1; k < nz; ++k) {
          const double cq1 = cq1_(d, i, j, k);
          const double b = 1.0 + cq1 * cof * d->rdn[k] *
                                      (d->rdnw[k] * AT(c2a, i, j, k) / (mh_(d, k, m) * mf_(d, k, m)) +
                                       d->rdnw[k - 1] * AT(c2a, i, j, k - 1) / (mh_(d, k - 1, m) * mf_(d, k, m)));
          const double cc = -cq1 * cof * d->rdn[k] * d->rdnw[k] * AT(c2a, i, j, k) / (mh_(d, k, m) * mf_(d, k + 1, m));
          AT(alpha, i, j, k) = 1.0 / (b - AT(a, i, j, k) * AT(gamma, i, j, k - 1));
          AT(gamma, i, j, k) = cc * AT(alpha, i, j, k);
        }
        const double b = 1.0 + 2.0 * cof * (d->rdnw[nz - 1] * d->rdnw[nz - 1]) * AT(c2a, i, j, nz - 1) /
                                   (mh_(d, nz - 1, m) * mf_(d, nz, m));
        AT(alpha, i, j, nz) = 1.0 / (b - AT(a, i, j, nz) * AT(gamma, i, j, nz - 1));
        AT(gamma, i, j, nz) = 0;
      }
  }
  const int ui0 = g->bc_x != CW_BC_PERIODIC ? 1 : 0, ui1 = nx;
  const int vj0 = (g->bc_y != CW_BC_PERIODIC && do_y) ? 1 : 0, vj1 = ny;
  const int ox = open_x(g), oy = open_y(g);
  const double emdx = d->o.emdiv * (1. / d->rdx), emdy = do_y ? d->o.emdiv * (1. / d->rdy) : 0.0;
  fld *mudf = &d->mudf, *ru_tend = F_(CW_RU_TEND), *rv_tend = F_(CW_RV_TEND);
  for (int it = 1; it <= n_small; ++it) {
    /* KUV (:151-190); open boundaries: the boundary faces take only the large-step tendency */
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny + oy; ++j)
        for (int i = 0; i < nx + ox; ++i) {
          if (ox && (i == 0 || i == nx) && j < ny) {
            AT(u, i, j, k) = AT(u, i, j, k) + dts * AT(ru_tend, i, j, k);
          } else if (i >= ui0 && i < ui1 && !edge_uface(&ed, i, j) && j < ed.ny) {
            const double mudf_x = -emdx * (AT(mudf, i, j, 0) - AT(mudf, i - 1, j, 0)) / AT(msfuy, i, j, 0);
            AT(u, i, j, k) = AT(u, i, j, k) + dts * AT(ru_tend, i, j, k) -
                             dts * cqu_(d, i, j, k) *
                                 uv_dp(d, 1, 0, i, j, k, AT(muu, i, j, 0), d->rdx, AT(msfux, i, j, 0) / AT(msfuy, i, j, 0)) +
                             d->c1h[k] * mudf_x;
          }
          if (do_y && oy && (j == 0 || j == ny) && i < nx) {
            AT(v, i, j, k) = AT(v, i, j, k) + dts * AT(rv_tend, i, j, k);
          } else if (do_y && j >= vj0 && j < vj1 && !edge_vface(&ed, i, j) && i < ed.nx) {
            const double mudf_y = -emdy * (AT(mudf, i, j, 0) - AT(mudf, i, j - 1, 0)) * AT(mvi, i, j, 0);
            AT(v, i, j, k) = AT(v, i, j, k) + dts * AT(rv_tend, i, j, k) -
                             dts * cqv_(d, i, j, k) *
                                 uv_dp(d, 0, 1, i, j, k, AT(muv, i, j, 0), d->rdy, AT(msfvy, i, j, 0) / AT(msfvx, i, j, 0)) +
                             d->c1h[k] * mudf_y;
          }
        }
    if (d->o.lbc) lbc_update_uv(d, dts);
    fill_halo(d, u);
    if (do_y) fill_halo(d, v);
    /* KMuTDiv (:194-206) */
    fld *us = &d->u_save, *vs = &d->v_save, *dv = &d->dvdxi;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double fx = (AT(u, i + 1, j, k) + (d->c1h[k] * AT(muu, i + 1, j, 0) + d->c2h[k]) * AT(us, i + 1, j, k) /
                                                      AT(msfuy, i + 1, j, 0)) -
                            (AT(u, i, j, k) + (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k]) * AT(us, i, j, k) / AT(msfuy, i, j, 0));
          double dd = d->rdx * fx;
          if (do_y)
            dd += d->rdy * ((AT(v, i, j + 1, k) + (d->c1h[k] * AT(muv, i, j + 1, 0) + d->c2h[k]) * AT(vs, i, j + 1, k) *
                                                      AT(mvi, i, j + 1, 0)) -
                            (AT(v, i, j, k) + (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k]) * AT(vs, i, j, k) * AT(mvi, i, j, 0)));
          AT(dv, i, j, k) = AT(msftx, i, j, 0) * AT(msfty, i, j, 0) * dd;
        }
    /* KMuTCol (:208-249) */
    const int first = it == 1, last = it == n_small;
    const double rn = (double)n_small;
    fld *ww_m = F_(CW_WW_M), *mu_tend = F_(CW_MU_TEND);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (edge_mass(&ed, i, j)) {
          for (int k = 0; k <= nz; ++k) {
            const double sw = (first ? 0.0 : AT(ww_m, i, j, k)) + AT(ww, i, j, k);
            AT(ww_m, i, j, k) = last ? sw / rn + AT(&d->ww1, i, j, k) : sw;
          }
          continue;
        }
        double dmdt = 0;
        for (int k = 0; k < nz; ++k) dmdt += d->dnw[k] * AT(dv, i, j, k);
        const double mtend = AT(mu_tend, i, j, 0);
        const double mu_old = AT(mu, i, j, 0);
        const double mu_new = mu_old + dts * (dmdt + mtend);
        AT(mu, i, j, 0) = mu_new;
        AT(mudf, i, j, 0) = dmdt + mtend;
        AT(muts, i, j, 0) = AT(mut, i, j, 0) + mu_new;
        AT(&d->muave, i, j, 0) = H * ((1.0 + epssm) * mu_new + (1.0 - epssm) * mu_old);
        double ww_full = 0;
        AT(ww, i, j, 0) = 0;
        {
          const double sw = (first ? 0.0 : AT(ww_m, i, j, 0)) + 0.0;
          AT(ww_m, i, j, 0) = last ? sw / rn + AT(&d->ww1, i, j, 0) : sw;
        }
        for (int k = 0; k < nz; ++k) {
          double wpp_hi = 0;
          if (k + 1 < nz) {
            ww_full = ww_full - d->dnw[k] * (d->c1h[k] * dmdt + AT(dv, i, j, k) + d->c1h[k] * mtend) / AT(msfty, i, j, 0);
            wpp_hi = ww_full - AT(&d->ww1, i, j, k + 1);
            AT(ww, i, j, k + 1) = wpp_hi;
          } else {
            AT(ww, i, j, nz) = 0;
          }
          const double sw = (first ? 0.0 : AT(ww_m, i, j, k + 1)) + wpp_hi;
          AT(ww_m, i, j, k + 1) = last ? sw / rn + AT(&d->ww1, i, j, k + 1) : sw;
        }
      }
    /* KMuTPoint (:251-277) */
    fld *ts = &d->t_save, *t_tend = F_(CW_T_TEND), *ru_m = F_(CW_RU_M), *rv_m = F_(CW_RV_M);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double su = (first ? 0.0 : AT(ru_m, i, j, k)) + AT(u, i, j, k);
          AT(ru_m, i, j, k) =
              last ? su / rn + (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k]) * AT(us, i, j, k) / AT(msfuy, i, j, 0) : su;
          if (do_y) {
            const double sv = (first ? 0.0 : AT(rv_m, i, j, k)) + AT(v, i, j, k);
            AT(rv_m, i, j, k) =
                last ? sv / rn + (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k]) * AT(vs, i, j, k) * AT(mvi, i, j, 0) : sv;
          }
          const double tk = AT(t, i, j, k);
          AT(&d->t_2save, i, j, k) = tk;
          if (edge_mass(&ed, i, j)) continue;
          double hflux = H * d->rdx *
                         (AT(u, i + 1, j, k) * (AT(ts, i + 1, j, k) + AT(ts, i, j, k)) -
                          AT(u, i, j, k) * (AT(ts, i, j, k) + AT(ts, i - 1, j, k)));
          if (do_y)
            hflux += H * d->rdy *
                     (AT(v, i, j + 1, k) * (AT(ts, i, j + 1, k) + AT(ts, i, j, k)) -
                      AT(v, i, j, k) * (AT(ts, i, j, k) + AT(ts, i, j - 1, k)));
          const double tn = tk + AT(msfty, i, j, 0) * dts * AT(t_tend, i, j, k);
#define WDTN(kk) (((kk) == 0 || (kk) == nz) ? 0.0 : AT(ww, i, j, kk) * (d->fnm[kk] * AT(ts, i, j, kk) + d->fnp[kk] * AT(ts, i, j, (kk)-1)))
          AT(t, i, j, k) = tn - dts * AT(msfty, i, j, 0) * (AT(msftx, i, j, 0) * hflux + d->rdnw[k] * (WDTN(k + 1) - WDTN(k)));
#undef WDTN
        }
    /* KSumEdge (:281-290): east / north faces of specified and open boundaries */
    if (ed.x || ox) {
      for (int k = 0; k < nz; ++k)
        for (int jj = 0; jj < ny; ++jj) {
          const int i = nx, j = jj;
          const double su = (first ? 0.0 : AT(ru_m, i, j, k)) + AT(u, i, j, k);
          const double cpl = (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k]) * AT(us, i, j, k);
          AT(ru_m, i, j, k) = last ? su / rn + cpl / AT(msfuy, i, j, 0) : su;
        }
    }
    if (ed.y || oy) {
      for (int k = 0; k < nz; ++k)
        for (int ii = 0; ii < nx; ++ii) {
          const int i = ii, j = ny;
          const double su = (first ? 0.0 : AT(rv_m, i, j, k)) + AT(v, i, j, k);
          const double cpl = (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k]) * AT(vs, i, j, k);
          AT(rv_m, i, j, k) = last ? su / rn + cpl * AT(mvi, i, j, 0) : su;
        }
    }
    if (d->o.lbc) lbc_update_mu_t(d, dts);
    fill_halo(d, mu);
    fill_halo(d, mudf);
    fill_halo(d, muts);
    /* advance_w: KWRhs, KWExpl, KWSolve (:295-408), then KWPRho (:411-416) */
    fld *R = &d->w_rhs, *T2 = &d->t2a, *c2a = &d->c2a;
    for (int k = 0; k < nz + 1; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (edge_mass(&ed, i, j)) continue;
          AT(R, i, j, k) = wc_rhs(d, i, j, k, dts);
          if (k < nz) AT(T2, i, j, k) = wc_t2ave(d, i, j, k);
        }
    const int terrain = !d->o.flat;
    fld *ht = F_(CW_HT), *rw_tend = F_(CW_RW_TEND);
    for (int k = 0; k < nz + 1; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (edge_mass(&ed, i, j)) continue;
          if (k == 0) {
            if (terrain) {
              double ws = AT(msftx, i, j, 0) * H * d->rdx *
                          ((AT(ht, i + 1, j, 0) - AT(ht, i, j, 0)) *
                               (d->cf1 * AT(u, i + 1, j, 0) + d->cf2 * AT(u, i + 1, j, 1) + d->cf3 * AT(u, i + 1, j, 2)) +
                           (AT(ht, i, j, 0) - AT(ht, i - 1, j, 0)) *
                               (d->cf1 * AT(u, i, j, 0) + d->cf2 * AT(u, i, j, 1) + d->cf3 * AT(u, i, j, 2)));
              if (do_y)
                ws = AT(msfty, i, j, 0) * H * d->rdy *
                         ((AT(ht, i, j + 1, 0) - AT(ht, i, j, 0)) *
                              (d->cf1 * AT(v, i, j + 1, 0) + d->cf2 * AT(v, i, j + 1, 1) + d->cf3 * AT(v, i, j + 1, 2)) +
                          (AT(ht, i, j, 0) - AT(ht, i, j - 1, 0)) *
                              (d->cf1 * AT(v, i, j, 0) + d->cf2 * AT(v, i, j, 1) + d->cf3 * AT(v, i, j, 2))) +
                     ws;
              AT(w, i, j, 0) = ws;
            } else {
              AT(w, i, j, 0) = 0;
            }
            continue;
          }
          const double m = AT(mut, i, j, 0), mav = AT(&d->muave, i, j, 0);
          const double ope = 1.0 + epssm, ome = 1.0 - epssm;
          const double msft_inv = 1.0 / AT(msfty, i, j, 0);
          const double r_k = AT(R, i, j, k), r_km1 = AT(R, i, j, k - 1), ph_k = AT(ph, i, j, k), ph_km1 = AT(ph, i, j, k - 1);
          if (k < nz) {
            const double r_kp1 = AT(R, i, j, k + 1), ph_kp1 = AT(ph, i, j, k + 1);
            AT(w, i, j, k) =
                AT(w, i, j, k) + dts * AT(rw_tend, i, j, k) +
                msft_inv * cq1_(d, i, j, k) *
                    (H * dts * G_ * d->rdn[k] *
                     (AT(c2a, i, j, k) * d->rdnw[k] / mh_(d, k, m) * (ope * (r_kp1 - r_k) + ome * (ph_kp1 - ph_k)) -
                      AT(c2a, i, j, k - 1) * d->rdnw[k - 1] / mh_(d, k - 1, m) * (ope * (r_k - r_km1) + ome * (ph_k - ph_km1)))) +
                dts * G_ * msft_inv *
                    (d->rdn[k] * (AT(c2a, i, j, k) * AT(alt, i, j, k) * AT(T2, i, j, k) -
                                  AT(c2a, i, j, k - 1) * AT(alt, i, j, k - 1) * AT(T2, i, j, k - 1)) -
                     d->c1f[k] * mav);
          } else {
            const int km = nz - 1;
            double wn = AT(w, i, j, k) + dts * AT(rw_tend, i, j, k) +
                        msft_inv * (-H * dts * G_ / mh_(d, km, m) * (d->rdnw[km] * d->rdnw[km]) * 2.0 * AT(c2a, i, j, km) *
                                        (ope * (r_k - r_km1) + ome * (ph_k - ph_km1)) -
                                    dts * G_ * (2.0 * d->rdnw[km] * AT(c2a, i, j, km) * AT(alt, i, j, km) * AT(T2, i, j, km) +
                                                d->c1f[k] * mav));
            if (d->o.top_lid) wn = 0;
            AT(w, i, j, k) = wn;
          }
        }
    fld *a = &d->a, *alpha = &d->alpha, *gamma = &d->gamma;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) { /* KWSolve */
        if (edge_mass(&ed, i, j)) continue;
        const double mts = AT(muts, i, j, 0), ope = 1.0 + epssm;
        for (int k = 1; k <= nz; ++k)
          AT(w, i, j, k) = (AT(w, i, j, k) - AT(a, i, j, k) * AT(w, i, j, k - 1)) * AT(alpha, i, j, k);
        for (int k = nz - 1; k >= 1; --k) AT(w, i, j, k) = AT(w, i, j, k) - AT(gamma, i, j, k) * AT(w, i, j, k + 1);
        if (d->o.damp_opt == 3) { /* implicit Rayleigh damping of w near the top (KWSolve :393-404) */
          const double dampmag = dts * d->o.dampcoef, hdepth = d->o.zdamp, pi = 4.0 * atan(1.0), m = AT(F_(CW_MUT), i, j, 0);
          const double htop = (AT(&d->ph_save, i, j, nz) + AT(F_(CW_PHB), i, j, nz)) / G_, hbot = htop - hdepth;
          for (int k = nz; k >= 1; --k) {
            const double hk = (AT(&d->ph_save, i, j, k) + AT(F_(CW_PHB), i, j, k)) / G_;
            double dampwt = 0;
            if (hk >= hbot) {
              const double x = H * pi * (hk - hbot) / hdepth;
              const double sn = d->pow_mode == OR_POW_GLIBC ? sin(x) : cw_sin(x);
              dampwt = dampmag * sn * sn;
            }
            AT(w, i, j, k) = (AT(w, i, j, k) - dampwt * mf_(d, k, m) * AT(&d->w_save, i, j, k)) / (1.0 + dampwt);
          }
        }
        for (int k = nz; k >= 1; --k)
          AT(ph, i, j, k) = AT(R, i, j, k) + AT(msfty, i, j, 0) * H * dts * G_ * ope * AT(w, i, j, k) / mf_(d, k, mts);
      }
    if (d->o.lbc) lbc_update_ph_w(d, dts);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) p_rho_point(d, i, j, k, smdiv, 1); /* KWPRho */
    fill_halo(d, ph);
    fill_halo(d, p);
    fill_halo(d, F_(CW_AL));
  }
  fill_halo(d, muts);
  fill_halo(d, F_(CW_RU_M));
  fill_halo(d, F_(CW_RV_M));
  fill_halo(d, F_(CW_WW_M));
  { /* KFinish (:419-444) */
    fld *us = &d->u_save, *vs = &d->v_save, *ws = &d->w_save, *ts = &d->t_save, *phs = &d->ph_save, *hd = F_(CW_H_DIABATIC);
    const double hd_dt = (rk_step == 3 && d->o.n_moist > 0) ? dts * (double)n_small : 0.0;
    for (int k = 0; k < nz + 1; ++k)
      for (int j = 0; j < nyv; ++j)
        for (int i = 0; i < nx + 1; ++i) {
          if (j < ny && k < nz) {
            const double mus_u = H * (AT(muts, i, j, 0) + AT(muts, i - 1, j, 0));
            AT(u, i, j, k) = (AT(msfuy, i, j, 0) * AT(u, i, j, k) + AT(us, i, j, k) * (d->c1h[k] * AT(muu, i, j, 0) + d->c2h[k])) /
                             (d->c1h[k] * mus_u + d->c2h[k]);
          }
          if (i < nx && j < nyv && k < nz) {
            const double mus_v = H * (AT(muts, i, j, 0) + AT(muts, i, j - 1, 0));
            AT(v, i, j, k) = (AT(msfvx, i, j, 0) * AT(v, i, j, k) + AT(vs, i, j, k) * (d->c1h[k] * AT(muv, i, j, 0) + d->c2h[k])) /
                             (d->c1h[k] * mus_v + d->c2h[k]);
          }
          if (i < nx && j < ny) {
            const double m = AT(mut, i, j, 0), mts = AT(muts, i, j, 0);
            AT(w, i, j, k) = (AT(msfty, i, j, 0) * AT(w, i, j, k) + AT(ws, i, j, k) * (d->c1f[k] * m + d->c2f[k])) /
                             (d->c1f[k] * mts + d->c2f[k]);
            AT(ph, i, j, k) = AT(ph, i, j, k) + AT(phs, i, j, k);
            AT(ww, i, j, k) = AT(ww, i, j, k) + AT(&d->ww1, i, j, k);
            if (k < nz)
              AT(t, i, j, k) = (AT(t, i, j, k) - (hd_dt != 0.0 ? hd_dt * (d->c1h[k] * m + d->c2h[k]) * AT(hd, i, j, k) : 0.0) +
                                AT(ts, i, j, k) * (d->c1h[k] * m + d->c2h[k])) /
                               (d->c1h[k] * mts + d->c2h[k]);
          }
        }
  }
  for (int j = 0; j < nyv; ++j)
    for (int i = 0; i < nx + 1; ++i) { /* KFinishMu (:446-453) */
      if (i < nx && j < ny) AT(mu, i, j, 0) = AT(mu, i, j, 0) + AT(&d->mu_save, i, j, 0);
      if (j < ny) AT(muus, i, j, 0) = H * (AT(muts, i, j, 0) + AT(muts, i - 1, j, 0));
      if (i < nx && j < nyv) AT(muvs, i, j, 0) = H * (AT(muts, i, j, 0) + AT(muts, i, j - 1, 0));
    }
  fill_halo(d, u);
  fill_halo(d, v);
  fill_halo(d, w);
  fill_halo(d, t);
  fill_halo(d, ph);
  fill_halo(d, ww);
  fill_halo(d, mu);
}

/* calc_p_rho_phi, hypsometric_opt 1 (linear) or 2 (log-linear in pressure) (KPRhoPhi :456-477;
 * SmallStep::calc_p_rho_phi(_interior) :609-633) */
static double eos_pow(or_dom* d, double base, int lane_i, int lane_n) {
  if (d->pow_mode == OR_POW_GLIBC) {
    const int lane = lane_n > 1 && !((lane_n & 1) && lane_i == lane_n - 1); /* vm::lane, backend.hpp:144 */
    if (lane) return _mm_cvtsd_f64(_ZGVbN2vv_pow(_mm_set1_pd(base), _mm_set1_pd(CPOVCV)));
    return pow(base, CPOVCV);
  }
  return cw_pow(base, CPOVCV);
}
static double hypso_log(or_dom* d, double x, int lane_i, int lane_n) {
  if (d->pow_mode == OR_POW_GLIBC) {
    const int lane = lane_n > 1 && !((lane_n & 1) && lane_i == lane_n - 1); /* vm::lane, backend.hpp:144 */
    if (lane) return _mm_cvtsd_f64(_ZGVbN2v_log(_mm_set1_pd(x)));
    return log(x);
  }
  return cw_log(x);
}
static void calc_p_rho_phi_range(or_dom* d, int i0, int i1, int j0, int j1) {
  fld *al = F_(CW_AL), *p = F_(CW_P), *ph = F_(CW_PH_2), *t = F_(CW_T_2), *mu = F_(CW_MU_2), *muts = F_(CW_MUTS),
      *alb = F_(CW_ALB), *pb = F_(CW_PB), *phb = F_(CW_PHB);
  const int n = i1 - i0, hypso = d->o.hypsometric_opt;
  const double ptop = d->p_top;
  for (int k = 0; k < d->g.nz; ++k)
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i) {
        double a;
        if (hypso == 2) {
          const double m = AT(muts, i, j, 0);
          const double pfu = d->c3f[k + 1] * m + d->c4f[k + 1] + ptop, pfd = d->c3f[k] * m + d->c4f[k] + ptop;
          const double phm = d->c3h[k] * m + d->c4h[k] + ptop;
          a = (AT(ph, i, j, k + 1) - AT(ph, i, j, k) + AT(phb, i, j, k + 1) - AT(phb, i, j, k)) / phm /
                  hypso_log(d, pfd / pfu, i - i0, n) - AT(alb, i, j, k);
        } else {
          a = -1.0 / (d->c1h[k] * AT(muts, i, j, 0) + d->c2h[k]) *
              (AT(alb, i, j, k) * (d->c1h[k] * AT(mu, i, j, 0)) + d->rdnw[k] * (AT(ph, i, j, k + 1) - AT(ph, i, j, k)));
        }
        AT(al, i, j, k) = a;
        const double base = R_D * (T0 + AT(t, i, j, k)) / (P1000MB * (a + AT(alb, i, j, k)));
        AT(p, i, j, k) = P1000MB * eos_pow(d, base, i - i0, n) - AT(pb, i, j, k);
      }
  fill_halo(d, p);
  fill_halo(d, al);
}

/* ------------------------------------------------------------------ scalar transport
 * ScalarTransport::run_stage / update (src/dyn/scalars.cpp:302-461), Fluxes (:42-140) */
typedef struct {
  or_dom* d;
  fld *q, *qo;
  spec_t sp;
  double dt, hup, vup;
  int nz, do_y, pd;
} sflux;
static double sf_f5(const sflux* f, double a, double b, double c, double dd, double e, double ff, double v) {
  return f->pd ? flux5_pd(a, b, c, dd, e, ff, v, f->hup) : flux5(a, b, c, dd, e, ff, v, f->hup);
}
static double sf_f3(const sflux* f, double a, double b, double c, double dd, double v, double up) {
  return f->pd ? flux3_pd(a, b, c, dd, v, up) : flux3(a, b, c, dd, v, up);
}
static double sf_fx(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  fld* q = f->q;
  const double vel = AT(F_(CW_RU_M), i, j, k);
  const int o = ord_face(i, f->sp.nx, f->sp.x);
  if (o == 2) return H * vel * (AT(q, i, j, k) + AT(q, i - 1, j, k));
  if (o == 3) return vel * sf_f3(f, AT(q, i - 2, j, k), AT(q, i - 1, j, k), AT(q, i, j, k), AT(q, i + 1, j, k), vel, f->hup);
  return vel * sf_f5(f, AT(q, i - 3, j, k), AT(q, i - 2, j, k), AT(q, i - 1, j, k), AT(q, i, j, k), AT(q, i + 1, j, k),
                     AT(q, i + 2, j, k), vel);
}
static double sf_fy(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  fld* q = f->q;
  const double vel = AT(F_(CW_RV_M), i, j, k);
  const int o = ord_face(j, f->sp.ny, f->sp.y);
  if (o == 2) return H * vel * (AT(q, i, j, k) + AT(q, i, j - 1, k));
  if (o == 3) return vel * sf_f3(f, AT(q, i, j - 2, k), AT(q, i, j - 1, k), AT(q, i, j, k), AT(q, i, j + 1, k), vel, f->hup);
  return vel * sf_f5(f, AT(q, i, j - 3, k), AT(q, i, j - 2, k), AT(q, i, j - 1, k), AT(q, i, j, k), AT(q, i, j + 1, k),
                     AT(q, i, j + 2, k), vel);
}
static double sf_fz(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  fld* q = f->q;
  if (k == 0 || k == f->nz) return 0;
  const double vel = AT(F_(CW_WW_M), i, j, k);
  if (k == 1 || k == f->nz - 1) return vel * (d->fnm[k] * AT(q, i, j, k) + d->fnp[k] * AT(q, i, j, k - 1));
  return vel * sf_f3(f, AT(q, i, j, k - 2), AT(q, i, j, k - 1), AT(q, i, j, k), AT(q, i, j, k + 1), -vel, f->vup);
}
static double sf_mh(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  return d->c1h[k] * AT(F_(CW_MUTS), i, j, 0) + d->c2h[k];
}
static double sf_fxl(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  fld* msfty = F_(CW_MSFTY);
  const double dx = 2.0 / (AT(msfty, i, j, 0) + AT(msfty, i - 1, j, 0)) / d->rdx,
               mu = H * (sf_mh(f, i, j, k) + sf_mh(f, i - 1, j, k)), vel = AT(F_(CW_RU_M), i, j, k);
  const double cr = (f->sp.x && i == 1) ? (vel / mu) * f->dt / dx : vel * f->dt / dx / mu;
  return mu * (dx / f->dt) * flux_upwind(AT(f->qo, i - 1, j, k), AT(f->qo, i, j, k), cr);
}
static double sf_fyl(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  fld* msftx = F_(CW_MSFTX);
  const double dy = 2.0 / (AT(msftx, i, j, 0) + AT(msftx, i, j - 1, 0)) / d->rdy,
               mu = H * (sf_mh(f, i, j, k) + sf_mh(f, i, j - 1, k)), vel = AT(F_(CW_RV_M), i, j, k);
  const double cr = vel * f->dt / dy / mu;
  return mu * (dy / f->dt) * flux_upwind(AT(f->qo, i, j - 1, k), AT(f->qo, i, j, k), cr);
}
static double sf_fzl(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  if (k == 0 || k == f->nz) return 0;
  const double dz = 2.0 / (d->rdnw[k] + d->rdnw[k - 1]), mu = sf_mh(f, i, j, k), vel = AT(F_(CW_WW_M), i, j, k);
  const double cr = vel * f->dt / dz / mu;
  return mu * (dz / f->dt) * flux_upwind(AT(f->qo, i, j, k - 1), AT(f->qo, i, j, k), cr);
}
/* spec zone of a specified boundary (not advected); the outermost cells of an open boundary are */
static int sf_spec_cell(const sflux* f, int i, int j) {
  return (f->sp.sx && (i == 0 || i == f->sp.nx - 1)) || (f->sp.sy && (j == 0 || j == f->sp.ny - 1));
}
static int sf_open_col(const sflux* f, int i) { return f->sp.ox && (i == 0 || i == f->sp.nx - 1); }
static int sf_open_row(const sflux* f, int j) { return f->sp.oy && (j == 0 || j == f->sp.ny - 1); }
/* Fluxes::open_terms (:110-116): x, then y; fo = the scalar itself (advect_scalar) or scalar_old (advect_scalar_pd) */
static double sf_open_terms(const sflux* f, double r, int i, int j, int k, const fld* fo) {
  or_dom* d = f->d;
  if (sf_open_col(f, i)) r = r - open_x_scalar(f->q, fo, F_(CW_RU_M), d->rdx, i, j, k, f->sp.nx);
  if (sf_open_row(f, j)) r = r - open_y_scalar(f->q, fo, F_(CW_RV_M), d->rdy, i, j, k, f->sp.ny);
  return r;
}
static double sf_adv(const sflux* f, int i, int j, int k) {
  or_dom* d = f->d;
  fld* msftx = F_(CW_MSFTX);
  if (sf_spec_cell(f, i, j)) return 0;
  double r;
  if (sf_open_col(f, i) || sf_open_row(f, j)) { /* y flux, x flux, open x, open y, vertical */
    r = 0.0;
    if (f->do_y && !sf_open_row(f, j)) r = r - (AT(msftx, i, j, 0) * d->rdy) * (sf_fy(f, i, j + 1, k) - sf_fy(f, i, j, k));
    if (!sf_open_col(f, i)) r = r - (AT(msftx, i, j, 0) * d->rdx) * (sf_fx(f, i + 1, j, k) - sf_fx(f, i, j, k));
    r = sf_open_terms(f, r, i, j, k, f->q);
  } else {
    r = -(AT(msftx, i, j, 0) * d->rdx) * (sf_fx(f, i + 1, j, k) - sf_fx(f, i, j, k));
    if (f->do_y) r -= (AT(msftx, i, j, 0) * d->rdy) * (sf_fy(f, i, j + 1, k) - sf_fy(f, i, j, k));
  }
  return r - d->rdnw[k] * (sf_fz(f, i, j, k + 1) - sf_fz(f, i, j, k));
}
static double m_full(or_dom* d, int k, double mub, double mu) { return d->c1h[k] * (mub + mu) + d->c2h[k]; }

static void scalar_update(or_dom* d, int n, int pd, double dt_rk) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz, do_y = !two_d(g);
  sflux f = {d, &d->q2[n], &d->q1[n], spec_of(g), dt_rk, d->o.h_adv_order == 5 ? 1.0 : 0.0,
             d->o.v_adv_order == 3 ? 1.0 : 0.0, nz, do_y, pd};
  fld *mub = F_(CW_MUB), *mu1 = F_(CW_MU_1), *mu2 = F_(CW_MU_2), *msfty = F_(CW_MSFTY), *msftx = F_(CW_MSFTX);
  fld *q1 = &d->q1[n], *qn = &d->q_new[n], *tendf = &d->qtf[n];
  if (!pd) {
    for (int k = 0; k < nz; ++k) /* KUpdate (:145-156) */
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          double tend = sf_adv(&f, i, j, k) * AT(msfty, i, j, 0);
          tend += AT(tendf, i, j, k);
          AT(qn, i, j, k) = (m_full(d, k, AT(mub, i, j, 0), AT(mu1, i, j, 0)) * AT(q1, i, j, k) + dt_rk * tend) /
                            m_full(d, k, AT(mub, i, j, 0), AT(mu2, i, j, 0));
        }
  } else {
    for (int k = 0; k < nz; ++k) /* KPreUpdatePD (:174-180) */
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double m = m_full(d, k, AT(mub, i, j, 0), AT(mu1, i, j, 0));
          AT(q1, i, j, k) = (m * AT(q1, i, j, k) + dt_rk * AT(tendf, i, j, k)) / m;
        }
    fill_halo(d, q1);
    fld *dhx = &d->dhx[n], *lox = &d->lox[n], *dhy = &d->dhy[n], *loy = &d->loy[n], *dhz = &d->dhz[n], *loz = &d->loz[n];
    for (int k = 0; k < nz; ++k) /* KFacePDX/Y/Z (:185-208) */
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx + 1; ++i) {
          const double l = sf_fxl(&f, i, j, k);
          AT(dhx, i, j, k) = sf_fx(&f, i, j, k) - l;
          AT(lox, i, j, k) = l;
        }
    if (do_y)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny + 1; ++j)
          for (int i = 0; i < nx; ++i) {
            const double l = sf_fyl(&f, i, j, k);
            AT(dhy, i, j, k) = sf_fy(&f, i, j, k) - l;
            AT(loy, i, j, k) = l;
          }
    for (int k = 0; k < nz + 1; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double l = sf_fzl(&f, i, j, k);
          AT(dhz, i, j, k) = sf_fz(&f, i, j, k) - l;
          AT(loz, i, j, k) = l;
        }
    fld* sc = &d->scale[n];
    for (int k = 0; k < nz; ++k) /* KScalePD (:215-241) */
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const int edge = (f.sp.x && (i == 0 || i == nx - 1)) || (f.sp.y && (j == 0 || j == ny - 1));
          if (edge) {
            AT(sc, i, j, k) = 1;
            continue;
          }
          const double mxy = AT(msftx, i, j, 0) * AT(msfty, i, j, 0);
          double hlow = d->rdx * (AT(lox, i + 1, j, k) - AT(lox, i, j, k));
          if (do_y) hlow += d->rdy * (AT(loy, i, j + 1, k) - AT(loy, i, j, k));
          const double ph_low = ((d->c1h[k] * AT(mub, i, j, 0) + d->c2h[k]) + d->c1h[k] * AT(mu1, i, j, 0)) * AT(q1, i, j, k) -
                                dt_rk * (mxy * hlow + AT(msfty, i, j, 0) * d->rdnw[k] * (AT(loz, i, j, k + 1) - AT(loz, i, j, k)));
          const double fxp = AT(dhx, i + 1, j, k), fxm = AT(dhx, i, j, k);
          double hout = d->rdx * ((fxp > 0 ? fxp : 0.0) - (fxm < 0 ? fxm : 0.0));
          if (do_y) {
            const double fyp = AT(dhy, i, j + 1, k), fym = AT(dhy, i, j, k);
            hout += d->rdy * ((fyp > 0 ? fyp : 0.0) - (fym < 0 ? fym : 0.0));
          }
          const double fzp = AT(dhz, i, j, k + 1), fzm = AT(dhz, i, j, k);
          const double out = mxy * hout + AT(msfty, i, j, 0) * d->rdnw[k] * ((fzp < 0 ? fzp : 0.0) - (fzm > 0 ? fzm : 0.0));
          const double flux_out = dt_rk * out;
          double s = 1;
          if (flux_out > ph_low) {
            s = ph_low / (flux_out + 1e-20);
            if (s < 0) s = 0;
          }
          AT(sc, i, j, k) = s;
        }
    fill_halo(d, sc);
#define DXL(ii, jj, kk) (AT(dhx, ii, jj, kk) * (AT(dhx, ii, jj, kk) > 0 ? AT(sc, (ii)-1, jj, kk) : (AT(dhx, ii, jj, kk) < 0 ? AT(sc, ii, jj, kk) : 1.0)))
#define DYL(ii, jj, kk) (AT(dhy, ii, jj, kk) * (AT(dhy, ii, jj, kk) > 0 ? AT(sc, ii, (jj)-1, kk) : (AT(dhy, ii, jj, kk) < 0 ? AT(sc, ii, jj, kk) : 1.0)))
#define DZL(ii, jj, kk) (((kk) == 0 || (kk) == nz) ? 0.0 : AT(dhz, ii, jj, kk) * (AT(dhz, ii, jj, kk) > 0 ? AT(sc, ii, jj, kk) : (AT(dhz, ii, jj, kk) < 0 ? AT(sc, ii, jj, (kk)-1) : 1.0)))
    for (int k = 0; k < nz; ++k) /* KUpdatePD (:244-291) */
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (sf_spec_cell(&f, i, j)) {
            AT(qn, i, j, k) = m_full(d, k, AT(mub, i, j, 0), AT(mu1, i, j, 0)) * AT(q1, i, j, k) /
                              m_full(d, k, AT(mub, i, j, 0), AT(mu2, i, j, 0));
            continue;
          }
          double tend;
          if (sf_open_col(&f, i) || sf_open_row(&f, j)) { /* open terms, vertical, x (not outer columns), y */
            tend = sf_open_terms(&f, 0.0, i, j, k, f.qo);
            tend = tend - d->rdnw[k] * (DZL(i, j, k + 1) - DZL(i, j, k) + AT(loz, i, j, k + 1) - AT(loz, i, j, k));
            if (!sf_open_col(&f, i))
              tend -= AT(msftx, i, j, 0) * (d->rdx * (DXL(i + 1, j, k) - DXL(i, j, k) + AT(lox, i + 1, j, k) - AT(lox, i, j, k)));
            if (do_y && !sf_open_row(&f, j))
              tend -= AT(msftx, i, j, 0) * (d->rdy * (DYL(i, j + 1, k) - DYL(i, j, k) + AT(loy, i, j + 1, k) - AT(loy, i, j, k)));
          } else {
            tend = -d->rdnw[k] * (DZL(i, j, k + 1) - DZL(i, j, k) + AT(loz, i, j, k + 1) - AT(loz, i, j, k));
            tend -= AT(msftx, i, j, 0) * (d->rdx * (DXL(i + 1, j, k) - DXL(i, j, k) + AT(lox, i + 1, j, k) - AT(lox, i, j, k)));
            if (do_y)
              tend -= AT(msftx, i, j, 0) * (d->rdy * (DYL(i, j + 1, k) - DYL(i, j, k) + AT(loy, i, j + 1, k) - AT(loy, i, j, k)));
          }
          AT(qn, i, j, k) = (m_full(d, k, AT(mub, i, j, 0), AT(mu1, i, j, 0)) * AT(q1, i, j, k) +
                             dt_rk * (tend * AT(msfty, i, j, 0))) /
                            m_full(d, k, AT(mub, i, j, 0), AT(mu2, i, j, 0));
        }
#undef DXL
#undef DYL
#undef DZL
  }
  /* swap(q_2, q_new) */
  fld tmp = d->q2[n];
  d->q2[n] = d->q_new[n];
  d->q_new[n] = tmp;
}

static void relax_scalar(or_dom* d, int n) {
  if (!d->lbcq[n].have) return;
  relax_one(d, &d->qtf[n], &d->q2[n], 0, d->c1h, d->c2h, NULL, &d->lbcq[n], 'q', d->g.nz, 1);
}
static void spec_scalar(or_dom* d, int n) {
  if (!d->lbcq[n].have) return;
  spec_one(d, &d->qtf[n], 0, &d->lbcq[n], 'q', d->g.nz);
}

static void scalars_run_stage(or_dom* d, int rk, double dt_rk) {
  const int ns = d->o.n_scalars;
  if (ns == 0) return;
  if (rk == 1) {
    if (d->o.diff_opt == 1 || d->o.diff_6th_opt != 0)
      for (int n = 0; n < ns; ++n) diffusion_scalar(d, n);
    if (d->o.lbc)
      for (int n = 0; n < ns; ++n) relax_scalar(d, n);
  }
  if (d->o.lbc)
    for (int n = 0; n < ns; ++n) spec_scalar(d, n);
  for (int pass = 0; pass < 2; ++pass) /* plain species, then positive-definite ones */
    for (int n = 0; n < ns; ++n) {
      const int moist = n < d->o.n_moist;
      const int pd = rk == 3 && (moist ? d->o.moist_adv_opt : d->o.scalar_adv_opt) == 1;
      if (pd != pass) continue;
      scalar_update(d, n, pd, dt_rk);
      if (d->o.lbc && !d->lbcq[n].have) lbc_flow_dep(d, n);
    }
  for (int n = 0; n < ns; ++n) fill_halo(d, &d->q2[n]);
}

/* ------------------------------------------------------------------ set_w_surface
 * KSetWSurface / set_w_surface (src/dyn/rk3.cpp:173-200), fill = false */
static void set_w_surface(or_dom* d) {
  const cw_grid* g = &d->g;
  fld *w = F_(CW_W_2), *u = F_(CW_U_2), *v = F_(CW_V_2), *ht = F_(CW_HT), *msftx = F_(CW_MSFTX), *msfty = F_(CW_MSFTY);
  fill_halo(d, u);
  fill_halo(d, v);
  for (int j = 0; j < g->ny; ++j)
    for (int i = 0; i < g->nx; ++i) {
      const double ws =
          AT(msfty, i, j, 0) * 0.5 * d->rdy *
              ((AT(ht, i, j + 1, 0) - AT(ht, i, j, 0)) * (d->cf1 * AT(v, i, j + 1, 0) + d->cf2 * AT(v, i, j + 1, 1) + d->cf3 * AT(v, i, j + 1, 2)) +
               (AT(ht, i, j, 0) - AT(ht, i, j - 1, 0)) * (d->cf1 * AT(v, i, j, 0) + d->cf2 * AT(v, i, j, 1) + d->cf3 * AT(v, i, j, 2))) +
          AT(msftx, i, j, 0) * 0.5 * d->rdx *
              ((AT(ht, i + 1, j, 0) - AT(ht, i, j, 0)) * (d->cf1 * AT(u, i + 1, j, 0) + d->cf2 * AT(u, i + 1, j, 1) + d->cf3 * AT(u, i + 1, j, 2)) +
               (AT(ht, i, j, 0) - AT(ht, i - 1, j, 0)) * (d->cf1 * AT(u, i, j, 0) + d->cf2 * AT(u, i, j, 1) + d->cf3 * AT(u, i, j, 2)));
      AT(w, i, j, 0) = ws;
    }
  fill_halo(d, w);
}

/* ------------------------------------------------------------------ RK3::step (src/dyn/rk3.cpp:166-250) */
static void zero_cells(or_dom* d, fld* f) {
  const cw_layout* L = &f->L;
  for (int k = 0; k < L->nz; ++k)
    for (int j = 0; j < L->ny; ++j)
      for (int i = 0; i < L->nx; ++i) AT(f, i, j, k) = 0;
}

static void tendencies(or_dom* d, int rk) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz, do_y = !two_d(g);
  tctx c = {d, spec_of(g), d->o.h_adv_order == 5 ? 1.0 : 0.0, d->o.v_adv_order == 3 ? 1.0 : 0.0, nz, do_y, d->o.top_lid};
  const int dd_on = d->o.diff_opt == 1 || d->o.diff_6th_opt != 0 || d->o.damp_opt == 2; /* DiffusionConfig::on */
  if (rk == 1) { /* zero_tendf (large_step.cpp:888-894) */
    zero_cells(d, F_(CW_PH_TENDF));
    zero_cells(d, F_(CW_RU_TENDF));
    zero_cells(d, F_(CW_RV_TENDF));
    zero_cells(d, F_(CW_RW_TENDF));
    zero_cells(d, F_(CW_T_TENDF));
    for (int n = 0; n < d->o.n_scalars; ++n) zero_cells(d, &d->qtf[n]);
  }
  if (d->o.lbc) zero_cells(d, F_(CW_MU_TEND));
  if (dd_on && rk == 1) diffusion_dynamics(d);
  if (d->o.lbc && rk == 1) lbc_relax_dry(d);
  const int use_tendf = d->o.lbc || dd_on;
  /* open boundaries: the boundary faces are advanced too (radiation condition) */
  const int ui0 = (g->bc_x != CW_BC_PERIODIC && !open_x(g)) ? 1 : 0, ui1 = open_x(g) ? nx + 1 : nx;
  const int vj0 = (g->bc_y != CW_BC_PERIODIC && do_y && !open_y(g)) ? 1 : 0, vj1 = open_y(g) ? ny + 1 : ny;
  const double wd_dt = d->o.w_damping == 1 ? g->dt : 0.0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = ui0; i < ui1; ++i) AT(F_(CW_RU_TEND), i, j, k) = tend_u(&c, i, j, k, use_tendf);
  if (do_y)
    for (int k = 0; k < nz; ++k)
      for (int j = vj0; j < vj1; ++j)
        for (int i = 0; i < nx; ++i) AT(F_(CW_RV_TEND), i, j, k) = tend_v(&c, i, j, k, use_tendf);
  for (int k = 1; k < nz + 1; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        AT(F_(CW_RW_TEND), i, j, k) = tend_w(&c, i, j, k, use_tendf, wd_dt, d->o.w_crit_cfl);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) AT(F_(CW_T_TEND), i, j, k) = tend_t(&c, i, j, k, use_tendf, d->o.n_moist > 0);
  for (int k = 1; k < nz + 1; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) AT(F_(CW_PH_TEND), i, j, k) = tend_ph(&c, i, j, k, d->o.lbc);
  if (d->o.lbc) lbc_spec_dry(d);
}

static void copy_fld(fld* dst, const fld* src) { memcpy(dst->a, src->a, (size_t)src->L.total * sizeof(double)); }

/* ------------------------------------------------------------------ microphysics coupling
 * PhysicsCoupling::step for mp_physics = 1 (src/dyn/physics_coupling.cpp:262-456): moist_physics_prep_em (KPrep
 * :42-60, KSaveQc :78-81), Kessler (src/phys/mp_kessler/kessler.hpp:47-159) on the columns outside the spec zone,
 * moist_physics_finish_em (KFinish :63-76), halos. Species 0, 1, 2 are qv, qc, qr. pow and exp by the mode:
 * glibc (libmvec's 2-lane functions on the lanes of WRF's vectorised loops, vm::lane) or cw_pow / cw_exp. */
static int vm_lane(int i, int n) { return n > 1 && !((n & 1) && i == n - 1); }
static double mp_pow(const or_dom* d, double a, double b, int i, int n) {
  if (d->pow_mode != OR_POW_GLIBC) return cw_pow(a, b);
  if (vm_lane(i, n)) return _mm_cvtsd_f64(_ZGVbN2vv_pow(_mm_set1_pd(a), _mm_set1_pd(b)));
  return pow(a, b);
}
static double mp_rpow(const or_dom* d, double a, double b) { return d->pow_mode == OR_POW_GLIBC ? pow(a, b) : cw_pow(a, b); }
static double mp_exp(const or_dom* d, double a, int i, int n) {
  if (d->pow_mode != OR_POW_GLIBC) return cw_exp(a);
  if (vm_lane(i, n)) return _mm_cvtsd_f64(_ZGVbN2v_exp(_mm_set1_pd(a)));
  return exp(a);
}
static double c_max(double a, double b) { return a < b ? b : a; } /* std::max */
static double c_min(double a, double b) { return b < a ? b : a; } /* std::min */

#define KS_LEVELS 128
typedef struct {
  fld *th, *rho, *pii, *z, *dz8w;
} mp_work;

static void kessler_column(or_dom* d, const mp_work* w, int i, int j, double dt, int i0, int ni) {
  fld *qv = &d->q2[0], *qc = &d->q2[1], *qr = &d->q2[2], *t = w->th;
  const int nz = d->g.nz;
  const double xlv = 2.5e6, cp = CP, ep2 = R_D / 461.6, svp1 = 0.6112, svp2 = 17.67, svp3 = 29.65, svpt0 = 273.15,
               rhowater = 1000.0;
  double vt[KS_LEVELS] = {0}, prodk[KS_LEVELS] = {0}, vtden[KS_LEVELS] = {0}, rdzk[KS_LEVELS] = {0},
         rhok[KS_LEVELS] = {0}, factor[KS_LEVELS] = {0}, rdzw[KS_LEVELS] = {0}, prod[KS_LEVELS] = {0};
  const double f5 = svp2 * (svpt0 - svp3) * xlv / cp;
  const double c1 = 0.001, c2 = 0.001, c3 = 2.2, c4 = 0.875, max_cr_sedimentation = 0.75;
  double crmax = 0;
  for (int k = 0; k < nz; ++k) {
    prodk[k] = AT(qr, i, j, k);
    rhok[k] = AT(w->rho, i, j, k);
    const double qrr = c_max(0, AT(qr, i, j, k) * 0.001 * rhok[k]);
    vtden[k] = sqrt(rhok[0] / rhok[k]);
    vt[k] = 36.34 * mp_rpow(d, qrr, 0.1364) * vtden[k];
    rdzw[k] = 1.0 / AT(w->dz8w, i, j, k);
    crmax = c_max(vt[k] * dt * rdzw[k], crmax);
  }
  for (int k = 0; k < nz - 1; ++k) rdzk[k] = 1.0 / (AT(w->z, i, j, k + 1) - AT(w->z, i, j, k));
  rdzk[nz - 1] = 1.0 / (AT(w->z, i, j, nz - 1) - AT(w->z, i, j, nz - 2));
  int nfall = (int)round(0.5 + crmax / max_cr_sedimentation);
  nfall = 1 < nfall ? nfall : 1;
  double dtfall = dt / nfall, time_sediment = dt;
  fld *rainnc = F_(CW_RAINNC), *rainncv = F_(CW_RAINNCV);
  while (nfall > 0) {
    time_sediment = time_sediment - dtfall;
    for (int k = 0; k < nz - 1; ++k) factor[k] = dtfall * rdzk[k] / rhok[k];
    factor[nz - 1] = dtfall * rdzk[nz - 1];
    const double ppt = rhok[0] * prodk[0] * vt[0] * dtfall / rhowater;
    AT(rainncv, i, j, 0) = ppt * 1000.0;
    AT(rainnc, i, j, 0) = AT(rainnc, i, j, 0) + ppt * 1000.0;
    for (int k = 0; k < nz - 1; ++k)
      prodk[k] = prodk[k] - factor[k] * (rhok[k] * prodk[k] * vt[k] - rhok[k + 1] * prodk[k + 1] * vt[k + 1]);
    prodk[nz - 1] = prodk[nz - 1] - factor[nz - 1] * prodk[nz - 1] * vt[nz - 1];
    if (nfall > 1) {
      nfall = nfall - 1;
      crmax = 0;
      for (int k = 0; k < nz; ++k) {
        const double qrr = c_max(0, prodk[k] * 0.001 * rhok[k]);
        vt[k] = 36.34 * mp_pow(d, qrr, 0.1364, k, nz) * vtden[k];
        crmax = c_max(vt[k] * time_sediment * rdzw[k], crmax);
      }
      int nfall_new = (int)round(0.5 + crmax / max_cr_sedimentation);
      nfall_new = 1 < nfall_new ? nfall_new : 1;
      if (nfall_new != nfall) {
        nfall = nfall_new;
        dtfall = time_sediment / nfall;
      }
    } else {
      for (int k = 0; k < nz; ++k) prod[k] = prodk[k];
      nfall = 0;
    }
  }
  const int li = i - i0;
  for (int k = 0; k < nz; ++k) {
    const double factorn = 1.0 / (1.0 + c3 * dt * mp_pow(d, c_max(0.0, AT(qr, i, j, k)), c4, li, ni));
    const double qrprod = AT(qc, i, j, k) * (1.0 - factorn) + factorn * c1 * dt * c_max(AT(qc, i, j, k) - c2, 0.0);
    const double rcgs = 0.001 * AT(w->rho, i, j, k);
    AT(qc, i, j, k) = c_max(AT(qc, i, j, k) - qrprod, 0.0);
    AT(qr, i, j, k) = (AT(qr, i, j, k) + prod[k] - AT(qr, i, j, k));
    AT(qr, i, j, k) = c_max(AT(qr, i, j, k) + qrprod, 0.0);
    const double pii = AT(w->pii, i, j, k);
    const double temp = pii * AT(t, i, j, k);
    const double pressure = 1.000e+05 * mp_pow(d, pii, 1004.0 / 287.0, li, ni);
    const double gam = 2.5e+06 / (1004.0 * pii);
    const double es = 1000.0 * svp1 * mp_exp(d, svp2 * (temp - svpt0) / (temp - svp3), li, ni);
    const double qvs = ep2 * es / (pressure - es);
    prod[k] = (AT(qv, i, j, k) - qvs) / (1.0 + pressure / (pressure - es) * qvs * f5 / ((temp - svp3) * (temp - svp3)));
    const double dim_qvs_qv = c_max(0.0, qvs - AT(qv, i, j, k));
    const double rq = rcgs * AT(qr, i, j, k);
    const double ern_num = (1.6 + 124.9 * mp_pow(d, rq, 0.2046, li, ni)) * mp_pow(d, rq, 0.525, li, ni);
    const double ern_den = 2.55e8 / (pressure * qvs) + 5.4e5;
    const double ern_term1 = dt * (ern_num / ern_den) * (dim_qvs_qv / (rcgs * qvs));
    const double ern_term2 = c_max(-prod[k] - AT(qc, i, j, k), 0.0);
    const double ern = c_min(ern_term1, c_min(ern_term2, AT(qr, i, j, k)));
    const double product = c_max(prod[k], -AT(qc, i, j, k));
    AT(t, i, j, k) = AT(t, i, j, k) + gam * (product - ern);
    AT(qv, i, j, k) = c_max(AT(qv, i, j, k) - product + ern, 0.0);
    AT(qc, i, j, k) = AT(qc, i, j, k) + product;
    AT(qr, i, j, k) = AT(qr, i, j, k) - ern;
  }
}

static void physics_step(or_dom* d) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const double dt = g->dt, rvrd = 461.6 / R_D, lim = d->o.mp_tend_lim;
  mp_work w;
  fld th, rho, pii, z, dz8w, hd_old, qv_old;
  fld* all[] = {&th, &rho, &pii, &z, &dz8w, &hd_old, &qv_old};
  for (size_t n = 0; n < sizeof all / sizeof all[0]; ++n) fld_alloc(all[n], g, ST_M, 3, 0);
  w.th = &th; w.rho = &rho; w.pii = &pii; w.z = &z; w.dz8w = &dz8w;
  fld *t = F_(CW_T_2), *ph = F_(CW_PH_2), *phb = F_(CW_PHB), *al = F_(CW_AL), *alb = F_(CW_ALB), *p = F_(CW_P),
      *pb = F_(CW_PB), *hd = F_(CW_H_DIABATIC), *qv = &d->q2[0];
  const int pz = specified(g) ? 1 : 0;
  const int pi0 = g->bc_x == CW_BC_PERIODIC ? 0 : pz, pni = nx - 2 * pi0;
  for (int k = 0; k < nz; ++k)  /* KPrep (qc_diabatic and the other WRF diagnostics are not kept) */
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double zw0 = (AT(ph, i, j, k) + AT(phb, i, j, k)) / G_;
        const double zw1 = (AT(ph, i, j, k + 1) + AT(phb, i, j, k + 1)) / G_;
        AT(&dz8w, i, j, k) = zw1 - zw0;
        AT(&z, i, j, k) = 0.5 * (zw0 + zw1);
        const double q = AT(qv, i, j, k);
        const double thv = (AT(t, i, j, k) + T0) / (1.0 + rvrd * q);
        AT(&th, i, j, k) = thv;
        AT(&hd_old, i, j, k) = thv;
        AT(&qv_old, i, j, k) = q;
        AT(&rho, i, j, k) = 1.0 / (AT(al, i, j, k) + AT(alb, i, j, k));
        AT(&pii, i, j, k) = mp_pow(d, (AT(p, i, j, k) + AT(pb, i, j, k)) / P1000MB, R_D / CP, i - pi0, pni);
      }
  const int sx = g->bc_x == CW_BC_SPECIFIED ? 1 : 0, sy = g->bc_y == CW_BC_SPECIFIED ? 1 : 0;
  for (int j = sy; j < ny - sy; ++j)
    for (int i = sx; i < nx - sx; ++i) kessler_column(d, &w, i, j, dt, sx, nx - 2 * sx);
  for (int k = 0; k < nz; ++k)  /* KFinish */
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double thn = AT(&th, i, j, k), th_old = AT(&hd_old, i, j, k), q = AT(qv, i, j, k), q_old = AT(&qv_old, i, j, k);
        double mpten = thn - th_old;
        mpten = mpten < lim * dt ? mpten : lim * dt;
        mpten = mpten > -lim * dt ? mpten : -lim * dt;
        const double qvten = q - q_old;
        AT(t, i, j, k) = th_old * (1.0 + rvrd * q_old) + mpten * (1.0 + rvrd * q) + rvrd * qvten * thn - T0;
        AT(hd, i, j, k) = (mpten * (1.0 + rvrd * q) + rvrd * qvten * thn) / dt;
      }
  fill_halo(d, t);
  fill_halo(d, hd);
  for (int n = 0; n < d->o.n_moist; ++n) fill_halo(d, &d->q2[n]);
  for (size_t n = 0; n < sizeof all / sizeof all[0]; ++n) fld_free(all[n]);
}

/* LargeStep::cfl_max (src/dyn/large_step.cpp:672-687, :865-877): Reducer maxima from -1e308 over levels 1..nz-1 of
 * the mass points, then 0 unless positive */
static void cfl_max(or_dom* d, int rk) {
  const cw_grid* g = &d->g;
  double v = -1e308, h = -1e308;
  for (int k = 1; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const double x = AT(F_(CW_WW), i, j, k) / (d->c1f[k] * AT(F_(CW_MUT), i, j, 0) + d->c2f[k]) * d->rdnw[k] * g->dt;
        const double xv = x < 0 ? -x : x;
        v = xv > v ? xv : v;
        double a = AT(F_(CW_U_2), i, j, k) * d->rdx * AT(F_(CW_MSFUX), i, j, 0) * g->dt;
        double b = AT(F_(CW_V_2), i, j, k) * d->rdy * AT(F_(CW_MSFVY), i, j, 0) * g->dt;
        a = a < 0 ? -a : a;
        b = b < 0 ? -b : b;
        const double xh = b > a ? b : a;
        h = xh > h ? xh : h;
      }
  d->cfl[2 * (rk - 1)] = v > 0.0 ? v : 0.0;
  d->cfl[2 * (rk - 1) + 1] = h > 0.0 ? h : 0.0;
}

static void rk3_step(or_dom* d) {
  const cw_grid* g = &d->g;
  if (d->o.lbc) d->dtbc += g->dt;
  copy_fld(F_(CW_U_1), F_(CW_U_2));
  copy_fld(F_(CW_V_1), F_(CW_V_2));
  copy_fld(F_(CW_W_1), F_(CW_W_2));
  copy_fld(F_(CW_T_1), F_(CW_T_2));
  copy_fld(F_(CW_PH_1), F_(CW_PH_2));
  copy_fld(F_(CW_MU_1), F_(CW_MU_2));
  fill_halo(d, F_(CW_MU_1));
  for (int n = 0; n < d->o.n_scalars; ++n) copy_fld(&d->q1[n], &d->q2[n]);
  const double dt = g->dt, dts = dt / d->n_sound;
  for (int rk = 1; rk <= 3; ++rk) {
    const double dt_rk = rk == 1 ? dt / 3.0 : (rk == 2 ? 0.5 * dt : dt);
    const double dts_rk = rk == 1 ? dt_rk : dts;
    const int ns = rk == 1 ? 1 : (rk == 2 ? d->n_sound / 2 : d->n_sound);
    large_prep(d);
    if (rk == 1 && d->o.diff_opt == 1) diffusion_prepare(d);
    tendencies(d, rk);
    cfl_max(d, rk);
    small_run_stage(d, dts_rk, ns, rk);
    scalars_run_stage(d, rk, dt_rk);
    calc_p_rho_phi_range(d, 0, g->nx, 0, g->ny);
  }
  if (d->o.mp_physics == 1) {  /* solve_em after the RK loop (rk3.cpp:150-158) */
    physics_step(d);
    const int sz = 1;
    const int px = g->bc_x == CW_BC_PERIODIC, py = g->bc_y == CW_BC_PERIODIC;
    if (d->o.lbc) calc_p_rho_phi_range(d, px ? 0 : sz, px ? g->nx : g->nx - sz, py ? 0 : sz, py ? g->ny : g->ny - sz);
    else calc_p_rho_phi_range(d, 0, g->nx, 0, g->ny);
  }
  if (d->o.lbc) {
    lbc_final(d);
    const int sz = 1;
    const int px = g->bc_x == CW_BC_PERIODIC, py = g->bc_y == CW_BC_PERIODIC;
    calc_p_rho_phi_range(d, px ? 0 : sz, px ? g->nx : g->nx - sz, py ? 0 : sz, py ? g->ny : g->ny - sz);
  }
  if (!d->o.flat) set_w_surface(d);
}

/* ------------------------------------------------------------------ API */
or_dom* or_create(const cw_grid* g, const cw_options* o) {
  or_dom* d = (or_dom*)calloc(1, sizeof(or_dom));
  d->g = *g;
  d->o = *o;
  if ((o->damp_opt < 0 || o->damp_opt > 3) || (o->hypsometric_opt != 1 && o->hypsometric_opt != 2) ||
      o->diff_6th_opt < 0 || o->diff_6th_opt > 2 ||
      (o->mp_physics != 0 && (o->mp_physics != 1 || o->n_moist < 3 || g->nz > KS_LEVELS)) ||
      (o->diff_opt != 0 && (o->diff_opt != 1 || (o->km_opt != 1 && o->km_opt != 4)))) {
    free(d);
    return NULL;
  }
  d->n_sound = o->time_step_sound > 0 ? o->time_step_sound
                                      : (int)fmax(2 * ((int)(300.0 * g->dt / fmin(g->dx, g->dy) - 0.01) + 1), 4);
  for (int id = 0; id < CW_Q_1; ++id) {
    char s;
    int rank, uni;
    field_kind(o, id, &s, &rank, &uni);
    fld_alloc(&d->f[id], g, s, rank, uni);
  }
  /* BaseState defaults: m = 1, cosa = 1, f = e = sina = ht = 0 (src/dyn/state.cpp:67-84) */
  const int ones[] = {CW_MSFTX, CW_MSFTY, CW_MSFUX, CW_MSFUY, CW_MSFVX, CW_MSFVY, CW_MSFVX_INV, CW_COSA};
  for (size_t n = 0; n < sizeof ones / sizeof ones[0]; ++n) fld_fill(&d->f[ones[n]], 1.0);
  const int ns = o->n_scalars;
  d->q1 = (fld*)calloc(ns + 1, sizeof(fld));
  d->q2 = (fld*)calloc(ns + 1, sizeof(fld));
  d->qtf = (fld*)calloc(ns + 1, sizeof(fld));
  d->q_new = (fld*)calloc(ns + 1, sizeof(fld));
  d->scale = (fld*)calloc(ns + 1, sizeof(fld));
  d->dhx = (fld*)calloc(ns + 1, sizeof(fld));
  d->lox = (fld*)calloc(ns + 1, sizeof(fld));
  d->dhy = (fld*)calloc(ns + 1, sizeof(fld));
  d->loy = (fld*)calloc(ns + 1, sizeof(fld));
  d->dhz = (fld*)calloc(ns + 1, sizeof(fld));
  d->loz = (fld*)calloc(ns + 1, sizeof(fld));
  d->lbcq = (slabset*)calloc(ns + 1, sizeof(slabset));
  for (int n = 0; n < ns; ++n) {
    fld_alloc(&d->q1[n], g, ST_M, 3, 0);
    fld_alloc(&d->q2[n], g, ST_M, 3, 0);
    fld_alloc(&d->qtf[n], g, ST_M, 3, 0);
    fld_alloc(&d->q_new[n], g, ST_M, 3, 0);
    fld_alloc(&d->scale[n], g, ST_M, 3, 0);
    fld_alloc(&d->dhx[n], g, ST_U, 3, 0);
    fld_alloc(&d->lox[n], g, ST_U, 3, 0);
    fld_alloc(&d->dhy[n], g, ST_V, 3, 0);
    fld_alloc(&d->loy[n], g, ST_V, 3, 0);
    fld_alloc(&d->dhz[n], g, ST_W, 3, 0);
    fld_alloc(&d->loz[n], g, ST_W, 3, 0);
  }
  fld_alloc(&d->u_save, g, ST_U, 3, 0);
  fld_alloc(&d->v_save, g, ST_V, 3, 0);
  fld_alloc(&d->w_save, g, ST_W, 3, 0);
  fld_alloc(&d->t_save, g, ST_M, 3, 0);
  fld_alloc(&d->ph_save, g, ST_W, 3, 0);
  fld_alloc(&d->ww1, g, ST_W, 3, 0);
  fld_alloc(&d->c2a, g, ST_M, 3, 0);
  fld_alloc(&d->pm1, g, ST_M, 3, 0);
  fld_alloc(&d->t_2save, g, ST_M, 3, 0);
  fld_alloc(&d->a, g, ST_W, 3, 0);
  fld_alloc(&d->alpha, g, ST_W, 3, 0);
  fld_alloc(&d->gamma, g, ST_W, 3, 0);
  fld_alloc(&d->mu_save, g, ST_M, 2, 0);
  fld_alloc(&d->mudf, g, ST_M, 2, 0);
  fld_alloc(&d->muave, g, ST_M, 2, 0);
  fld_alloc(&d->w_rhs, g, ST_W, 3, 0);
  fld_alloc(&d->t2a, g, ST_M, 3, 0);
  fld_alloc(&d->dvdxi, g, ST_M, 3, 0);
  fld_alloc(&d->xkmh, g, ST_M, 3, 0);
  fld_alloc(&d->xkmv, g, ST_M, 3, 0);
  fld_alloc(&d->xkhh, g, ST_M, 3, 0);
  fld_alloc(&d->xkhv, g, ST_M, 3, 0);
  const int nz = g->nz;
  double** arr[] = {&d->znu, &d->znw, &d->dnw, &d->dn, &d->rdnw, &d->rdn, &d->fnm, &d->fnp, &d->c1h, &d->c2h, &d->c3h,
                    &d->c4h, &d->c1f, &d->c2f, &d->c3f, &d->c4f, &d->u_base, &d->v_base, &d->t_base, &d->qv_base_1d,
                    &d->z_base};
  for (size_t n = 0; n < sizeof arr / sizeof arr[0]; ++n) *arr[n] = (double*)calloc(nz + 2, sizeof(double));
  d->rdx = 1.0 / g->dx;
  d->rdy = two_d(g) ? 0.0 : 1.0 / g->dy;
  /* LateralBC: slabs and fcx/gcx (lateral_bc.cpp:198-233) */
  if (o->lbc) {
    const int width = 5, spec_zone = 1, relax_zone = 4;
    const int nk[5] = {nz, nz, nz, nz + 1, 1};
    for (int v = 0; v < 5; ++v) {
      slabset* s = &d->lbc[v];
      s->nk = nk[v];
      for (int sd = 0; sd < 4; ++sd)
        s->npos[sd] = sd < 2 ? (v == CW_LBC_V ? g->ny + 1 : g->ny) : (v == CW_LBC_U ? g->nx + 1 : g->nx);
      size_t off = 0;
      for (int half = 0; half < 2; ++half)
        for (int sd = 0; sd < 4; ++sd) {
          s->off[half * 4 + sd] = off;
          off += (size_t)s->npos[sd] * s->nk * width;
        }
      s->d = (double*)calloc(off, sizeof(double));
    }
    for (int n = 0; n < ns; ++n) {
      slabset* s = &d->lbcq[n];
      s->nk = nz;
      for (int sd = 0; sd < 4; ++sd) s->npos[sd] = sd < 2 ? g->ny : g->nx;
      size_t off = 0;
      for (int half = 0; half < 2; ++half)
        for (int sd = 0; sd < 4; ++sd) {
          s->off[half * 4 + sd] = off;
          off += (size_t)s->npos[sd] * nz * width;
        }
      s->d = (double*)calloc(off, sizeof(double));
    }
    for (int loop = spec_zone + 1; loop <= spec_zone + relax_zone; ++loop) {
      const double num = (double)(spec_zone + relax_zone - loop), den = (double)(relax_zone - 1);
      d->fcx[loop - 1] = 0.1 / g->dt * num / den;
      d->gcx[loop - 1] = 1.0 / g->dt / 50.0 * num / den;
    }
  }
  return d;
}

void or_destroy(or_dom* d) {
  if (!d) return;
  for (int id = 0; id < CW_Q_1; ++id) fld_free(&d->f[id]);
  for (int n = 0; n < d->o.n_scalars; ++n) {
    fld_free(&d->q1[n]); fld_free(&d->q2[n]); fld_free(&d->qtf[n]); fld_free(&d->q_new[n]); fld_free(&d->scale[n]);
    fld_free(&d->dhx[n]); fld_free(&d->lox[n]); fld_free(&d->dhy[n]); fld_free(&d->loy[n]); fld_free(&d->dhz[n]);
    fld_free(&d->loz[n]);
    free(d->lbcq[n].d);
  }
  free(d->q1); free(d->q2); free(d->qtf); free(d->q_new); free(d->scale); free(d->dhx); free(d->lox); free(d->dhy);
  free(d->loy); free(d->dhz); free(d->loz); free(d->lbcq);
  fld* in[] = {&d->u_save, &d->v_save, &d->w_save, &d->t_save, &d->ph_save, &d->ww1, &d->c2a, &d->pm1, &d->t_2save,
               &d->a, &d->alpha, &d->gamma, &d->mu_save, &d->mudf, &d->muave, &d->w_rhs, &d->t2a, &d->dvdxi,
               &d->xkmh, &d->xkmv, &d->xkhh, &d->xkhv};
  for (size_t n = 0; n < sizeof in / sizeof in[0]; ++n) fld_free(in[n]);
  double* arr[] = {d->znu, d->znw, d->dnw, d->dn, d->rdnw, d->rdn, d->fnm, d->fnp, d->c1h, d->c2h, d->c3h,
                   d->c4h, d->c1f, d->c2f, d->c3f, d->c4f, d->u_base, d->v_base, d->t_base, d->qv_base_1d, d->z_base};
  for (size_t n = 0; n < sizeof arr / sizeof arr[0]; ++n) free(arr[n]);
  for (int v = 0; v < 5; ++v) free(d->lbc[v].d);
  free(d);
}

static fld* field_ptr(or_dom* d, int field, int n) {
  if (field >= 0 && field < CW_Q_1) return &d->f[field];
  if (n < 0 || n >= d->o.n_scalars) return NULL;
  if (field == CW_Q_1) return &d->q1[n];
  if (field == CW_Q_2) return &d->q2[n];
  if (field == CW_Q_TENDF) return &d->qtf[n];
  return NULL;
}
int or_layout(or_dom* d, int field, int n, cw_layout* out) {
  fld* f = field_ptr(d, field, n);
  if (!f) return -1;
  *out = f->L;
  return 0;
}
double* or_field(or_dom* d, int field, int n) {
  fld* f = field_ptr(d, field, n);
  return f ? f->a : NULL;
}
int or_set_vertical(or_dom* d, const cw_vertical* v) {
  const int nz = d->g.nz;
#define CP1(dst, src, cnt) \
  do { if (src) memcpy(dst, src, (size_t)(cnt) * sizeof(double)); else memset(dst, 0, (size_t)(cnt) * sizeof(double)); } while (0)
  CP1(d->znu, v->znu, nz); CP1(d->dnw, v->dnw, nz); CP1(d->rdnw, v->rdnw, nz); CP1(d->c1h, v->c1h, nz);
  CP1(d->c2h, v->c2h, nz); CP1(d->c3h, v->c3h, nz); CP1(d->c4h, v->c4h, nz);
  CP1(d->znw, v->znw, nz + 1); CP1(d->dn, v->dn, nz + 1); CP1(d->rdn, v->rdn, nz + 1); CP1(d->fnm, v->fnm, nz + 1);
  CP1(d->fnp, v->fnp, nz + 1); CP1(d->c1f, v->c1f, nz + 1); CP1(d->c2f, v->c2f, nz + 1); CP1(d->c3f, v->c3f, nz + 1);
  CP1(d->c4f, v->c4f, nz + 1);
  CP1(d->u_base, v->u_base, nz); CP1(d->v_base, v->v_base, nz); CP1(d->t_base, v->t_base, nz);
  CP1(d->qv_base_1d, v->qv_base_1d, nz); CP1(d->z_base, v->z_base, nz);
#undef CP1
  d->cf1 = v->cf1; d->cf2 = v->cf2; d->cf3 = v->cf3; d->cfn = v->cfn; d->cfn1 = v->cfn1;
  d->rdx = v->rdx; d->rdy = v->rdy; d->p_top = v->p_top;
  return 0;
}
static int set_slab(slabset* s, int side, const double* values, const double* tends, size_t count) {
  const size_t n = (size_t)s->npos[side] * s->nk * 5;
  if (count != n) return -1;
  memcpy(s->d + s->off[side], values, n * sizeof(double));
  memcpy(s->d + s->off[4 + side], tends, n * sizeof(double));
  s->have = 1;
  return 0;
}
int or_set_lbc(or_dom* d, int var, int side, const double* values, const double* tends, size_t count) {
  if (!d->o.lbc || var < 0 || var > 4 || side < 0 || side > 3) return -1;
  return set_slab(&d->lbc[var], side, values, tends, count);
}
int or_set_lbc_scalar(or_dom* d, int n, int side, const double* values, const double* tends, size_t count) {
  if (!d->o.lbc || n < 0 || n >= d->o.n_scalars || side < 0 || side > 3) return -1;
  return set_slab(&d->lbcq[n], side, values, tends, count);
}
int or_set_lbc_time(or_dom* d, double dtbc) {
  d->dtbc = dtbc;
  return 0;
}
void or_set_pow_mode(or_dom* d, int mode) { d->pow_mode = mode; }
int or_n_sound(or_dom* d) { return d->n_sound; }
int or_step(or_dom* d, int nsteps) {
  for (int n = 0; n < nsteps; ++n) rk3_step(d);
  return 0;
}
const char* or_last_error(or_dom* d) { return d ? d->err : ""; }

/* ------------------------------------------------------------------ diagnostics
 * dyn::Diagnostics::compute (src/dyn/diagnostics.cpp:56-80) with the functors of :18-51, reduced in the
 * reference CPU build's order (Reducer::run, src/core/backend.hpp:836-860): per level k a running sum from
 * 0.0 over j (outer) and i (inner), or a running maximum from -1e308, then the levels folded in order. */
#define RVOVRD (461.6 / 287.0)
static double dg_absnan(double v) { return (v != v || v - v != 0.0) ? INFINITY : (v < 0 ? -v : v); }

static double dg_max_abs(const fld* f, int nx, int ny, int nz) {
  double acc = -1e308;
  for (int k = 0; k < nz; ++k) {
    double a = -1e308;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double v = dg_absnan(AT(f, i, j, k));
        a = v > a ? v : a;
      }
    acc = a > acc ? a : acc;
  }
  return acc;
}

static double dg_thp(const or_dom* d, int i, int j, int k, double sign, int moist) {
  double th = AT(&d->f[CW_T_2], i, j, k);
  if (moist) th = (th + T0) / (1.0 + RVOVRD * AT(&d->q2[0], i, j, k)) - T0;
  const double v = th - AT(&d->f[CW_T_INIT], i, j, k);
  return v != v ? INFINITY : sign * v;
}

static double dg_energy(const or_dom* d, int i, int j, int k) {
  const fld *u = &d->f[CW_U_2], *v = &d->f[CW_V_2], *w = &d->f[CW_W_2], *t = &d->f[CW_T_2], *p = &d->f[CW_P];
  const fld *ph = &d->f[CW_PH_2], *mu = &d->f[CW_MU_2], *mub = &d->f[CW_MUB], *pb = &d->f[CW_PB], *phb = &d->f[CW_PHB];
  const double m = d->c1h[k] * (AT(mu, i, j, 0) + AT(mub, i, j, 0)) + d->c2h[k];
  const double uc = 0.5 * (AT(u, i, j, k) + AT(u, i + 1, j, k));
  const double vc = 0.5 * (AT(v, i, j, k) + AT(v, i, j + 1, k));
  const double wc = 0.5 * (AT(w, i, j, k) + AT(w, i, j, k + 1));
  const double base = (AT(p, i, j, k) + AT(pb, i, j, k)) / P1000MB;
  const double rcp = R_D / CP;
  const double T = (AT(t, i, j, k) + T0) * (d->pow_mode == OR_POW_GLIBC ? pow(base, rcp) : cw_pow(base, rcp));
  const double phm = 0.5 * (AT(ph, i, j, k) + AT(ph, i, j, k + 1) + AT(phb, i, j, k) + AT(phb, i, j, k + 1));
  return -d->dnw[k] * m * (0.5 * (uc * uc + vc * vc + wc * wc) + CV * T + phm);
}

int or_diagnostics(or_dom* d, double out[9]) {
  const cw_grid* g = &d->g;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  out[0] = dg_max_abs(&d->f[CW_U_2], nxs(g, ST_U), ny, nz);
  out[1] = dg_max_abs(&d->f[CW_V_2], nx, nys(g, ST_V), nz);
  out[2] = dg_max_abs(&d->f[CW_W_2], nx, ny, nz + 1);
  double mq = 0;
  for (int n = 0; n < d->o.n_scalars; ++n) {
    const double v = dg_max_abs(&d->q2[n], nx, ny, nz);
    mq = mq < v ? v : mq;
  }
  out[8] = mq;
  const int moist = d->o.n_moist > 0; /* species 0 is qv (State::P_QV) */
  double mx = -1e308, mn = -1e308, sm = 0, se = 0;
  for (int k = 0; k < nz; ++k) {
    double a = -1e308, b = -1e308, s = 0.0, e = 0.0;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double vp = dg_thp(d, i, j, k, 1.0, moist), vm = dg_thp(d, i, j, k, -1.0, moist);
        a = vp > a ? vp : a;
        b = vm > b ? vm : b;
        const double m = d->c1h[k] * (AT(&d->f[CW_MU_2], i, j, 0) + AT(&d->f[CW_MUB], i, j, 0)) + d->c2h[k];
        s = s + -d->dnw[k] * m * (AT(&d->f[CW_T_2], i, j, k) + T0);
        e = e + dg_energy(d, i, j, k);
      }
    mx = a > mx ? a : mx;
    mn = b > mn ? b : mn;
    sm = sm + s;
    se = se + e;
  }
  double dm = 0.0, s0 = 0.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) s0 = s0 + (AT(&d->f[CW_MU_2], i, j, 0) + AT(&d->f[CW_MUB], i, j, 0));
  dm = dm + s0;
  const double area = g->dx * (two_d(g) ? 1.0 : g->dy) / G_;
  out[3] = -mn;
  out[4] = mx;
  out[5] = area * dm;
  out[6] = area * sm;
  out[7] = area * se;
  return 0;
}

int or_cfl_max(or_dom* d, double out[6]) {
  memcpy(out, d->cfl, sizeof d->cfl);
  return 0;
}
