// SPDX-License-Identifier: GPL-3.0-or-later
// Host-side inputs of a domain (cw_case) and the seeded synthetic case generators.
//
// Straka density current: a restatement of CPPWRF's ideal-case set-up for "straka" -- the dry sounding
// (cases::Sounding, src/cases/cases.cpp:17-86), the uniform_z eta levels (:194-201), the level
// coefficients (BaseState::set_levels, src/dyn/state.cpp:86-116), the hydrostatic initial state
// (cases::initialize, cases.cpp:224-287) and the 1-D base profiles (src/cases/model.cpp:149-177) -- with
// the same operation order, so the reference's regression goldens can be reproduced from it.
//
// Limited-area case: a from-scratch generator (see cw_gen_lam below) for a 3-D domain with terrain,
// the hybrid sigma-pressure coordinate, moist species and specified lateral boundaries.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <stdexcept>
#include <string>
#include <vector>

#include "cw_fields.hpp"

namespace cw {
namespace cst {
constexpr double g = 9.81;
constexpr double r_d = 287.0;
constexpr double cp = 7.0 * r_d / 2.0;
constexpr double cv = cp - r_d;
constexpr double cvpm = -cv / cp;
constexpr double rcp = r_d / cp;
constexpr double p1000mb = 100000.0;
constexpr double t0 = 300.0;
constexpr double r_v = 461.6;
constexpr double rvovrd = r_v / r_d;
constexpr double ep_2 = r_d / r_v;
}  // namespace cst
}  // namespace cw

struct cw_case {
  cw_grid g{};
  cw_options o{};
  std::vector<std::vector<double>> f;   // CW_U_1 .. CW_COSA
  std::vector<std::vector<double>> q1, q2, qtf;
  std::vector<cw_layout> L;
  cw_layout Lq{};
  // vertical arrays
  std::vector<double> znu, znw, dnw, dn, rdnw, rdn, fnm, fnp, c1h, c2h, c3h, c4h, c1f, c2f, c3f, c4f, u_base, v_base,
      t_base, qv_base_1d, z_base;
  double cf1 = 0, cf2 = 0, cf3 = 0, cfn = 0, cfn1 = 0, rdx = 0, rdy = 0, p_top = 0;
  // boundary slabs: [var][side] values / tends; scalars [n][side]
  std::vector<double> lv[5][4], lt[5][4];
  std::vector<std::vector<double>> qv[4], qt[4];
  std::vector<char> q_have;
  double dtbc = 0;

  double& at(int id, int i, int j, int k) {
    const cw_layout& l = L[id];
    return f[id][size_t(l.offset + i * l.si + j * l.sj + k * l.sk)];
  }
  size_t idx(const cw_layout& l, int i, int j, int k) const { return size_t(l.offset + i * l.si + j * l.sj + k * l.sk); }
  double& at_q(int n, int i, int j, int k) { return q2[size_t(n)][idx(Lq, i, j, k)]; }
};

namespace {

// HaloLine (src/core/halo.cpp:52-88) on a host array: x pass over the rows, y pass over the full x extent
void host_fill_halo(const cw_grid& g, const cw_layout& L, double* base, bool odd_x, bool odd_y) {
  if (L.uniform) return;
  double* p = base + L.offset;
  auto line = [&](double* q, int64_t sn, int n, bool face, bool periodic, bool odd, bool flat, int lo, int hi, int a) {
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
    double v = q[src * sn];
    if (!periodic && !flat && src == i) return;
    if (!periodic && !flat && odd) v = -v;
    q[i * sn] = v;
  };
  const bool ux = L.stagger == 'U', vy = L.stagger == 'V';
  for (int k = 0; k < L.nz; ++k)
    for (int a = 0; a < (ux ? 8 : 6); ++a)
      for (int j = 0; j < L.ny; ++j)
        line(p + j * L.sj + k * L.sk, 1, g.nx, ux, g.bc_x == CW_BC_PERIODIC, odd_x, cw::flat_x(g), L.wi0, L.wi1, a);
  if (cw::two_d(g)) return;
  for (int k = 0; k < L.nz; ++k)
    for (int i = L.wi0; i < L.wi1; ++i)
      for (int a = 0; a < (vy ? 8 : 6); ++a)
        line(p + i + k * L.sk, L.sj, g.ny, vy, g.bc_y == CW_BC_PERIODIC, odd_y, cw::flat_y(g), L.wj0, L.wj1, a);
}

void fill_q_halo(cw_case* c, int n) { host_fill_halo(c->g, c->Lq, c->q2[size_t(n)].data(), false, false); }

void fill_default_halo(cw_case* c, int id) {
  const cw_layout& L = c->L[id];
  const bool three = L.rank == 3;
  host_fill_halo(c->g, L, c->f[id].data(), three && L.stagger == 'U', three && L.stagger == 'V');
}

// cases::Sounding (src/cases/cases.cpp:17-86), dry or moist
struct Sounding {
  std::vector<double> pi_, w_;
  double dz_;
  double (*th_)(double, const void*);
  double (*qv_)(double, const void*);
  const void* ctx;
  double theta(double z) const { return th_(z, ctx); }
  double qv(double z) const { return qv_ ? qv_(z, ctx) : 0.0; }
  double theta_rho(double z) const {
    if (!qv_) return theta(z);
    const double q = qv(z);
    return theta(z) * (1.0 + cw::cst::rvovrd * q) / (1.0 + q);
  }
  Sounding(double (*th_fn)(double, const void*), double (*qv_fn)(double, const void*), const void* c, double p_surf,
           double zmax, double dz)
      : dz_(dz), th_(th_fn), qv_(qv_fn), ctx(c) {
    using namespace cw::cst;
    const int n = int(std::ceil(zmax / dz)) + 2;
    pi_.resize(n);
    pi_[0] = std::pow(p_surf / p1000mb, rcp);
    for (int m = 1; m < n; ++m) {
      const double z0 = (m - 1) * dz, z1 = m * dz;
      const double f = (1.0 / theta_rho(z0) + 4.0 / theta_rho(0.5 * (z0 + z1)) + 1.0 / theta_rho(z1)) / 6.0;
      pi_[m] = pi_[m - 1] - g / cp * f * dz;
    }
    if (qv_) {
      auto rq = [&](int m) {
        const double z = m * dz, pi = pi_[m], pp = p1000mb * std::pow(pi, 1.0 / rcp);
        return pp / (r_d * theta(z) * (1.0 + rvovrd * qv(z)) * pi) * qv(z);
      };
      w_.assign(n, 0.0);
      for (int m = n - 2; m >= 0; --m) w_[m] = w_[m + 1] + 0.5 * g * dz * (rq(m) + rq(m + 1));
    }
  }
  double p(double z) const {
    using namespace cw::cst;
    const double s = z / dz_;
    const int m = int(std::floor(s));
    if (m < 0 || m + 1 >= int(pi_.size())) throw std::runtime_error("Sounding::p out of range");
    const double z0 = m * dz_, h = z - z0;
    const double f = (1.0 / theta_rho(z0) + 4.0 / theta_rho(z0 + 0.5 * h) + 1.0 / theta_rho(z)) / 6.0;
    const double pi = pi_[m] - g / cp * f * h;
    return p1000mb * std::pow(pi, 1.0 / rcp);
  }
  double z_of_p(double pp) const {
    double lo = 0, hi = (pi_.size() - 2) * dz_;
    if (pp > p(lo) || pp < p(hi)) throw std::runtime_error("Sounding::z_of_p out of range");
    for (int it = 0; it < 200 && hi - lo > 1e-9; ++it) {
      const double mid = 0.5 * (lo + hi);
      (p(mid) > pp ? lo : hi) = mid;
    }
    return 0.5 * (lo + hi);
  }
  // the weight of the water vapour above z (Pa), linear between the table's points
  double vapour_load(double z) const {
    if (!qv_) return 0.0;
    const double s = z / dz_;
    const int m = int(std::floor(s));
    if (m < 0 || m + 1 >= int(w_.size())) throw std::runtime_error("Sounding::vapour_load out of range");
    const double a = s - m;
    return (1.0 - a) * w_[m] + a * w_[m + 1];
  }
  double pd(double z) const { return p(z) - vapour_load(z); }  // dry-air pressure
  double z_of_pd(double pp) const {
    if (!qv_) return z_of_p(pp);
    double lo = 0, hi = (pi_.size() - 2) * dz_;
    if (pp > pd(lo) || pp < pd(hi)) throw std::runtime_error("Sounding::z_of_pd out of range");
    for (int it = 0; it < 200 && hi - lo > 1e-9; ++it) {
      const double mid = 0.5 * (lo + hi);
      (pd(mid) > pp ? lo : hi) = mid;
    }
    return 0.5 * (lo + hi);
  }
};

// BaseState::set_levels, hybrid_opt = 0 (src/dyn/state.cpp:86-116)
void set_levels(cw_case* c, const std::vector<double>& e) {
  const int nz = c->g.nz;
  if (int(e.size()) != nz + 1) throw std::runtime_error("set_levels: need nz+1 eta levels");
  for (int k = 0; k <= nz; ++k) c->znw[k] = e[k];
  for (int k = 0; k < nz; ++k) {
    c->dnw[k] = c->znw[k + 1] - c->znw[k];
    c->rdnw[k] = 1.0 / c->dnw[k];
    c->znu[k] = 0.5 * (c->znw[k + 1] + c->znw[k]);
  }
  for (int k = 1; k < nz; ++k) {
    c->dn[k] = 0.5 * (c->dnw[k] + c->dnw[k - 1]);
    c->rdn[k] = 1.0 / c->dn[k];
    c->fnp[k] = 0.5 * c->dnw[k] / c->dn[k];
    c->fnm[k] = 0.5 * c->dnw[k - 1] / c->dn[k];
  }
  const double cof1 = (2. * c->dn[1] + c->dn[2]) / (c->dn[1] + c->dn[2]) * c->dnw[0] / c->dn[1];
  const double cof2 = c->dn[1] / (c->dn[1] + c->dn[2]) * c->dnw[0] / c->dn[2];
  c->cf1 = c->fnp[1] + cof1;
  c->cf2 = c->fnm[1] - cof1 - cof2;
  c->cf3 = cof2;
  c->cfn = (0.5 * c->dnw[nz - 1] + c->dn[nz - 1]) / c->dn[nz - 1];
  c->cfn1 = -0.5 * c->dnw[nz - 1] / c->dn[nz - 1];
  for (int k = 0; k < nz; ++k) { c->c1h[k] = 1; c->c2h[k] = 0; c->c3h[k] = c->znu[k]; c->c4h[k] = 0; }
  for (int k = 0; k <= nz; ++k) { c->c1f[k] = 1; c->c2f[k] = 0; c->c3f[k] = c->znw[k]; c->c4f[k] = 0; }
}


}  // namespace

extern "C" {

int cw_default_options(cw_options* o) {
  if (!o) return -1;
  std::memset(o, 0, sizeof *o);
  o->khdif = 0; o->kvdif = 0; o->pr_inv = 3.0;
  o->top_lid = 0; o->h_adv_order = 5; o->v_adv_order = 3; o->w_damping = 0; o->w_crit_cfl = 1.0;
  o->epssm = 0.1; o->smdiv = 0.1; o->emdiv = 0.01;
  o->damp_opt = 0; o->hypsometric_opt = 1; o->zdamp = 5000.0; o->dampcoef = 0.2;
  o->time_step_sound = 0;
  o->moist_adv_opt = 1; o->scalar_adv_opt = 1; o->tke_adv_opt = 1;
  o->diff_opt = 0; o->km_opt = 1;
  o->flat = 1; o->n_moist = 0; o->n_scalars = 0; o->lbc = 0; o->precision = CW_FP64;
  o->mp_physics = 0; o->mp_tend_lim = 10.0;
  o->diff_6th_opt = 0; o->diff_6th_factor = 0.12; o->coriolis = 0; o->mapped = 0;
  return 0;
}

int cw_layout_of(const cw_grid* g, const cw_options* o, int field, cw_layout* out) {
  if (!g || !o || !out) return -1;
  try {
    if (field >= 0 && field < CW_Q_1) *out = cw::field_layout(*g, *o, field);
    else if (field >= CW_Q_1 && field <= CW_Q_TENDF) *out = cw::layout_make(*g, 'M', 3, false);
    else return -1;
  } catch (...) {
    return -1;
  }
  return 0;
}

int cw_case_create(const cw_grid* g, const cw_options* o, cw_case** out) {
  if (!g || !o || !out) return -1;
  if (cw::unsupported(*g, *o)) return -2;
  try {
    cw_case* c = new cw_case;
    c->g = *g;
    c->o = *o;
    c->f.resize(CW_Q_1);
    c->L.resize(CW_Q_1);
    for (int id = 0; id < CW_Q_1; ++id) {
      c->L[id] = cw::field_layout(*g, *o, id);
      c->f[id].assign(size_t(c->L[id].total), 0.0);
    }
    for (int id : {CW_MSFTX, CW_MSFTY, CW_MSFUX, CW_MSFUY, CW_MSFVX, CW_MSFVY, CW_MSFVX_INV, CW_COSA})
      std::fill(c->f[id].begin(), c->f[id].end(), 1.0);
    c->Lq = cw::layout_make(*g, 'M', 3, false);
    c->q1.assign(o->n_scalars, std::vector<double>(size_t(c->Lq.total), 0.0));
    c->q2 = c->q1;
    c->qtf = c->q1;
    const int nz = g->nz;
    for (auto* a : {&c->znu, &c->dnw, &c->rdnw, &c->c1h, &c->c2h, &c->c3h, &c->c4h, &c->u_base, &c->v_base, &c->t_base,
                    &c->qv_base_1d, &c->z_base})
      a->assign(nz, 0.0);
    for (auto* a : {&c->znw, &c->dn, &c->rdn, &c->fnm, &c->fnp, &c->c1f, &c->c2f, &c->c3f, &c->c4f}) a->assign(nz + 1, 0.0);
    c->rdx = 1.0 / g->dx;
    c->rdy = cw::two_d(*g) ? 0.0 : 1.0 / g->dy;
    c->p_top = g->p_top;
    if (o->lbc) {
      for (int v = 0; v < 5; ++v)
        for (int s = 0; s < 4; ++s) {
          const size_t n = size_t(cw::lbc_npos(*g, v, s)) * cw::lbc_nk(*g, v) * cw::kLbcWidth;
          c->lv[v][s].assign(n, 0.0);
          c->lt[v][s].assign(n, 0.0);
        }
      for (int s = 0; s < 4; ++s) {
        const size_t n = size_t(s < 2 ? g->ny : g->nx) * nz * cw::kLbcWidth;
        c->qv[s].assign(o->n_scalars, std::vector<double>(n, 0.0));
        c->qt[s].assign(o->n_scalars, std::vector<double>(n, 0.0));
      }
      c->q_have.assign(o->n_scalars, 0);
    }
    *out = c;
  } catch (...) {
    return -3;
  }
  return 0;
}

int cw_case_destroy(cw_case* c) {
  delete c;
  return 0;
}

int cw_case_clone(const cw_case* c, cw_case** out) {
  if (!c || !out) return -1;
  try {
    *out = new cw_case(*c);
  } catch (...) {
    return -3;
  }
  return 0;
}

int cw_case_config(const cw_case* c, cw_grid* g, cw_options* o) {
  if (!c) return -1;
  if (g) *g = c->g;
  if (o) *o = c->o;
  return 0;
}

int cw_case_field(cw_case* c, int field, int n, double** data, cw_layout* layout) {
  if (!c) return -1;
  if (field >= 0 && field < CW_Q_1) {
    if (data) *data = c->f[field].data();
    if (layout) *layout = c->L[field];
    return 0;
  }
  if (n < 0 || n >= c->o.n_scalars) return -1;
  std::vector<double>* v = field == CW_Q_1 ? &c->q1[n] : field == CW_Q_2 ? &c->q2[n] : field == CW_Q_TENDF ? &c->qtf[n] : nullptr;
  if (!v) return -1;
  if (data) *data = v->data();
  if (layout) *layout = c->Lq;
  return 0;
}

int cw_case_vertical(cw_case* c, cw_vertical* v) {
  if (!c || !v) return -1;
  *v = cw_vertical{c->znu.data(), c->dnw.data(), c->rdnw.data(), c->c1h.data(), c->c2h.data(), c->c3h.data(),
                   c->c4h.data(), c->znw.data(), c->dn.data(), c->rdn.data(), c->fnm.data(), c->fnp.data(),
                   c->c1f.data(), c->c2f.data(), c->c3f.data(), c->c4f.data(), c->u_base.data(), c->v_base.data(),
                   c->t_base.data(), c->qv_base_1d.data(), c->z_base.data(), c->cf1, c->cf2, c->cf3, c->cfn, c->cfn1,
                   c->rdx, c->rdy, c->p_top, cw::cst::t0};
  return 0;
}

int cw_case_lbc(cw_case* c, int is_scalar, int var, int side, double** values, double** tends, size_t* count) {
  if (!c || !c->o.lbc || side < 0 || side > 3) return -1;
  if (!is_scalar) {
    if (var < 0 || var > 4) return -1;
    if (values) *values = c->lv[var][side].data();
    if (tends) *tends = c->lt[var][side].data();
    if (count) *count = c->lv[var][side].size();
    return 0;
  }
  if (var < 0 || var >= c->o.n_scalars) return -1;
  if (!c->q_have[var]) {
    if (count) *count = 0;
    return 1;  // no boundary data for this scalar (flow_dep_bdy)
  }
  if (values) *values = c->qv[side][var].data();
  if (tends) *tends = c->qt[side][var].data();
  if (count) *count = c->qv[side][var].size();
  return 0;
}

int cw_case_lbc_time(cw_case* c, double* dtbc) {
  if (!c || !dtbc) return -1;
  *dtbc = c->dtbc;
  return 0;
}

int cw_default_ideal_params(cw_ideal_params* p, int kind) {
  if (!p || kind < 0 || kind > 4) return -1;
  p->kind = kind;
  p->theta0 = p->n_bv = p->u0 = p->xc = p->zc = p->xr = p->zr = p->amplitude = p->radius = p->a = CW_DEFAULT;
  p->p_surf = 1.0e5;
  return 0;
}

namespace {
struct IdealCtx {
  int kind;
  double theta0, n_bv, u0;
  // squall2d: Weisman & Klemp (1982) sounding (make_case, src/cases/cases.cpp:135-173)
  double theta_tr = 343.0, z_tr = 12000.0, t_tr = 213.0, qv_max = 0.014;
  const std::vector<double>* qtab = nullptr;  // qv on a 50 m table (nullptr: no vapour)
  double dzt = 50.0;
  int nt = 0;
};
double ideal_theta(double z, const void* v) {
  using namespace cw::cst;
  const IdealCtx* c = static_cast<const IdealCtx*>(v);
  if (c->kind == CW_IDEAL_REST_STATE || c->kind == CW_IDEAL_IGW) return c->theta0 * std::exp(c->n_bv * c->n_bv * z / g);
  if (c->kind == CW_IDEAL_SQUALL2D)
    return z <= c->z_tr ? c->theta0 + (c->theta_tr - c->theta0) * std::pow(z / c->z_tr, 1.25)
                        : c->theta_tr * std::exp(g / (cp * c->t_tr) * (z - c->z_tr));
  return 300.0;
}
double squall_rh(const IdealCtx* c, double z) { return z <= c->z_tr ? 1.0 - 0.75 * std::pow(z / c->z_tr, 1.25) : 0.25; }
// the case's qv(z): linear in the table (qv = 0 without one)
double ideal_qv(double z, const void* v) {
  const IdealCtx* c = static_cast<const IdealCtx*>(v);
  if (!c->qtab) return 0.0;
  const double f = std::clamp(z / c->dzt, 0.0, double(c->nt - 1) - 1e-9);
  const int n = int(f);
  const std::vector<double>& q = *c->qtab;
  return q[n] + (f - n) * (q[n + 1] - q[n]);
}
// the qv table of squall2d: qv = min(qv_max, RH ep_2 e_s / (p - e_s)) with p from a sounding that carries the
// previous iteration's qv (8 fixed-point iterations; cases.cpp:149-167)
void squall_qv_table(IdealCtx& c, double p_surf, double zmax, std::vector<double>& tab) {
  using namespace cw::cst;
  c.nt = int(zmax / c.dzt) + 2;
  tab.assign(size_t(c.nt), 0.0);
  for (int it = 0; it < 8; ++it) {
    c.qtab = it == 0 ? nullptr : &tab;
    Sounding snd(ideal_theta, it == 0 ? nullptr : ideal_qv, &c, p_surf, zmax, 0.5);
    std::vector<double> q(size_t(c.nt));
    for (int n = 0; n < c.nt; ++n) {
      const double z = std::min(n * c.dzt, zmax), pz = snd.p(z), T = ideal_theta(z, &c) * std::pow(pz / p1000mb, rcp);
      const double es = 611.2 * std::exp(17.67 * (T - 273.15) / (T - 29.65));
      q[size_t(n)] = std::min(c.qv_max, squall_rh(&c, z) * ep_2 * es / (pz - es));
    }
    tab = q;
  }
  c.qtab = &tab;
}
double or_default(double v, double d) { return v < -1e299 ? d : v; }
}  // namespace

// cases::make_case + init_ideal + cases::initialize for the ideal cases (flat terrain; src/cases/cases.cpp:90-192,
// :224-287, model.cpp:88-179). The grid's p_top becomes the dry sounding's pressure at ztop (model.cpp:96-99).
// With moist species (species 0 is qv, State::P_QV >= 0) the full state is WRF's moist one (initialize_moist,
// cases.cpp:292-353): dry-mass mu' from the vapour load, hydrostatic p' with moisture loading, theta_m; qv = 0
// unless the case has vapour (squall2d). The other scalars start at zero; the caller fills them.
int cw_gen_ideal(cw_case* c, const cw_ideal_params* pp) {
  if (!c || !pp) return -1;
  using namespace cw::cst;
  try {
    cw_grid& G = c->g;
    if (!c->o.flat || c->o.lbc) return -2;
    const int kind = pp->kind;
    const bool moist = c->o.n_moist > 0;
    if (kind == CW_IDEAL_SQUALL2D && !moist) return -2;
    const double pi = std::numbers::pi;
    const double xcenter = 0.5 * G.nx * G.dx;
    IdealCtx ctx{kind, 300.0, 0.01, 0.0};
    std::vector<double> qtab;
    double xc = 0, zc = 0, xr = 0, zr = 0, amp = 0, rad = 0, aa = 0, u_env = 0;
    switch (kind) {
      case CW_IDEAL_REST_STATE:
        ctx.theta0 = or_default(pp->theta0, 300.0);
        ctx.n_bv = or_default(pp->n_bv, 0.01);
        u_env = or_default(pp->u0, 0.0);
        break;
      case CW_IDEAL_STRAKA:
        xc = or_default(pp->xc, xcenter); zc = or_default(pp->zc, 3000.0);
        xr = or_default(pp->xr, 4000.0); zr = or_default(pp->zr, 2000.0);
        amp = or_default(pp->amplitude, -15.0);
        break;
      case CW_IDEAL_WARM_BUBBLE:
        xc = or_default(pp->xc, xcenter); zc = or_default(pp->zc, 2000.0);
        rad = or_default(pp->radius, 2000.0); amp = or_default(pp->amplitude, 2.0);
        break;
      case CW_IDEAL_IGW:
        ctx.theta0 = 300.0;
        ctx.n_bv = or_default(pp->n_bv, 0.01);
        u_env = or_default(pp->u0, 20.0);
        amp = or_default(pp->amplitude, 0.01);
        aa = or_default(pp->a, 5000.0);
        xc = or_default(pp->xc, 100000.0);
        break;
      case CW_IDEAL_SQUALL2D:  // no wind: u_shear tanh(z / 3 km) - u_shift = 0
        ctx.theta0 = or_default(pp->theta0, 300.0);
        xc = or_default(pp->xc, xcenter); zc = or_default(pp->zc, 1400.0);
        xr = or_default(pp->xr, 10000.0); zr = or_default(pp->zr, 1400.0);
        amp = or_default(pp->amplitude, 2.0);
        squall_qv_table(ctx, pp->p_surf, G.ztop * 1.2 + 1000.0, qtab);
        break;
      default: return -1;
    }
    const double Hz = G.ztop;
    // theta'(x, y, z, exner) of make_case (cases.cpp:103-134); libm::pow(v, 2) is v * v (gcc's fold)
    auto theta_pert = [&](double x, double z, double exner) -> double {
      switch (kind) {
        case CW_IDEAL_STRAKA: {
          const double a = (x - xc) / xr, b = (z - zc) / zr;
          const double L = std::sqrt(a * a + b * b);
          return L <= 1.0 ? amp * 0.5 * (std::cos(pi * L) + 1.0) / exner : 0.0;
        }
        case CW_IDEAL_WARM_BUBBLE: {
          const double a = (x - xc) / rad, b = (z - zc) / rad;
          const double L = std::sqrt(a * a + b * b);
          if (!(L <= 1.0)) return 0.0;
          const double cl = std::cos(0.5 * pi * L);
          return amp * (cl * cl);
        }
        case CW_IDEAL_IGW: {
          const double t = (x - xc) / aa;
          return amp * std::sin(pi * z / Hz) / (1.0 + t * t);
        }
        case CW_IDEAL_SQUALL2D: {
          const double a = (x - xc) / xr, b = (z - zc) / zr;
          const double L = std::sqrt(a * a + b * b);
          if (!(L <= 1.0)) return 0.0;
          const double cl = std::cos(0.5 * pi * L);
          return amp * (cl * cl);
        }
        default: return 0.0;
      }
    };
    // the dry sounding (eta levels, base state) and, with moisture, the moist one of the full state
    IdealCtx dry = ctx;
    dry.qtab = nullptr;
    Sounding snd(ideal_theta, nullptr, &dry, pp->p_surf, G.ztop * 1.2 + 1000.0, 0.5);
    G.p_top = snd.p(G.ztop);
    c->p_top = G.p_top;
    const int nz = G.nz;
    std::vector<double> eta(nz + 1);  // make_eta_levels, uniform_z
    {
      const double ps = snd.p(0.0), pt = snd.p(G.ztop);
      for (int k = 0; k <= nz; ++k) eta[k] = (snd.p(G.ztop * k / nz) - pt) / (ps - pt);
      eta[0] = 1.0;
      eta[nz] = 0.0;
    }
    set_levels(c, eta);
    const double mub = pp->p_surf - G.p_top;
    std::vector<double> pb(nz), tb(nz), alb(nz), phb(nz + 1), zm(nz), exn(nz);
    for (int k = 0; k < nz; ++k) {
      pb[k] = c->c3h[k] * mub + c->c4h[k] + G.p_top;
      tb[k] = snd.theta(snd.z_of_p(pb[k]));
      alb[k] = (r_d / p1000mb) * tb[k] * std::pow(pb[k] / p1000mb, cvpm);
      exn[k] = std::pow(pb[k] / p1000mb, rcp);
    }
    phb[0] = 0.0;
    for (int k = 0; k < nz; ++k) phb[k + 1] = phb[k] - c->dnw[k] * (c->c1h[k] * mub + c->c2h[k]) * alb[k];
    for (int k = 0; k < nz; ++k) zm[k] = 0.5 * (phb[k] + phb[k + 1]) / g;
    c->f[CW_MUB][0] = mub;
    for (int k = 0; k < nz; ++k) {
      c->f[CW_PB][k] = pb[k];
      c->f[CW_ALB][k] = alb[k];
      c->f[CW_T_INIT][k] = tb[k] - t0;
    }
    for (int k = 0; k <= nz; ++k) c->f[CW_PHB][k] = phb[k];
    const int nx = G.nx, ny = G.ny;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double x = (i + 0.5) * G.dx;
          const double t = tb[k] + theta_pert(x, zm[k], exn[k]);
          const double alt = (r_d / p1000mb) * t * std::pow(pb[k] / p1000mb, cvpm);
          const double al = alt - alb[k];
          c->at(CW_T_2, i, j, k) = t - t0;
          c->at(CW_AL, i, j, k) = al;
          c->at(CW_ALT, i, j, k) = alt;
        }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double ph = 0.0;
        c->at(CW_PH_2, i, j, 0) = 0.0;
        for (int k = 0; k < nz; ++k) {
          ph -= c->dnw[k] * ((c->c1h[k] * mub + c->c2h[k]) * c->at(CW_AL, i, j, k));
          c->at(CW_PH_2, i, j, k + 1) = ph;
        }
      }
    const cw_layout& Lu = c->L[CW_U_2];
    for (int k = 0; k < Lu.nz; ++k)
      for (int j = 0; j < Lu.ny; ++j)
        for (int i = 0; i < Lu.nx; ++i)
          c->at(CW_U_2, i, j, k) = (G.bc_x == CW_BC_SYMMETRIC && (i == 0 || i == G.nx)) ? 0.0 : u_env;
    for (int id : {CW_T_2, CW_AL, CW_ALT, CW_PH_2, CW_U_2, CW_V_2, CW_W_2, CW_P, CW_MU_2}) fill_default_halo(c, id);
    c->f[CW_U_1] = c->f[CW_U_2];
    c->f[CW_V_1] = c->f[CW_V_2];
    c->f[CW_W_1] = c->f[CW_W_2];
    c->f[CW_T_1] = c->f[CW_T_2];
    c->f[CW_PH_1] = c->f[CW_PH_2];
    c->f[CW_MU_1] = c->f[CW_MU_2];
    if (moist) {  // initialize_moist (cases.cpp:292-353), use_theta_m = 1
      Sounding msnd(ideal_theta, ideal_qv, &ctx, pp->p_surf, G.ztop * 1.2 + 1000.0, 0.5);
      const double pd_surf = pp->p_surf - msnd.vapour_load(0.0);
      const double mu1 = pd_surf - G.p_top - mub;
      std::vector<double> qv(nz), thd(nz), th(nz), p(nz);
      for (int k = 0; k < nz; ++k) {
        const double p_level = c->c3h[k] * (pd_surf - G.p_top) + c->c4h[k] + G.p_top;
        const double z = msnd.z_of_pd(p_level);
        qv[k] = msnd.qv(z);
        thd[k] = msnd.theta(z);
      }
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double x = (i + 0.5) * G.dx;
          for (int k = 0; k < nz; ++k) th[k] = thd[k] + theta_pert(x, zm[k], exn[k]);
          auto eos = [&](int k, double pk) {  // alt = R_d/p0 theta (1 + rvovrd qv) ((p + pb)/p0)^cvpm
            const double qvf = 1.0 + rvovrd * qv[k];
            const double alt = (r_d / p1000mb) * th[k] * qvf * std::pow((pk + pb[k]) / p1000mb, cvpm);
            c->at(CW_ALT, i, j, k) = alt;
            c->at(CW_AL, i, j, k) = alt - alb[k];
            c->at(CW_P, i, j, k) = pk;
          };
          int k = nz - 1;  // hydrostatic p' from the top with the moisture load
          double qvf1 = 0.5 * (qv[k] + qv[k]);
          double qvf2 = 1.0 / (1.0 + qvf1);
          qvf1 = qvf1 * qvf2;
          double pk = -0.5 * ((c->c1f[nz] * mu1) + qvf1 * (c->c1f[nz] * mub + c->c2f[nz])) / c->rdnw[k] / qvf2;
          eos(k, pk);
          for (k = nz - 2; k >= 0; --k) {
            qvf1 = 0.5 * (qv[k] + qv[k + 1]);
            qvf2 = 1.0 / (1.0 + qvf1);
            qvf1 = qvf1 * qvf2;
            pk = pk - ((c->c1f[k + 1] * mu1) + qvf1 * (c->c1f[k + 1] * mub + c->c2f[k + 1])) / qvf2 / c->rdn[k + 1];
            eos(k, pk);
          }
          double ph = 0.0;
          c->at(CW_PH_2, i, j, 0) = 0.0;
          for (k = 0; k < nz; ++k) {
            ph = ph - c->dnw[k] * (((c->c1h[k] * mub + c->c2h[k]) + c->c1h[k] * mu1) * c->at(CW_AL, i, j, k) +
                                   c->c1h[k] * mu1 * alb[k]);
            c->at(CW_PH_2, i, j, k + 1) = ph;
          }
          for (k = 0; k < nz; ++k) {
            c->at(CW_T_2, i, j, k) = th[k] * (1.0 + rvovrd * qv[k]) - t0;  // theta_m - t0
            c->at_q(0, i, j, k) = qv[k];
          }
          c->at(CW_MU_2, i, j, 0) = mu1;
        }
      for (int k = 0; k < nz; ++k) c->f[CW_QV_BASE][k] = qv[k];
      for (int id : {CW_T_2, CW_AL, CW_ALT, CW_PH_2, CW_P, CW_MU_2}) fill_default_halo(c, id);
      fill_q_halo(c, 0);
      c->f[CW_T_1] = c->f[CW_T_2];
      c->f[CW_PH_1] = c->f[CW_PH_2];
      c->f[CW_MU_1] = c->f[CW_MU_2];
      c->q1[0] = c->q2[0];
    }
    for (int k = 0; k < nz; ++k) {  // model.cpp:149-177: the column (0, 0)
      c->u_base[k] = c->at(CW_U_2, 0, 0, k);
      c->v_base[k] = c->at(CW_V_2, 0, 0, k);
      c->t_base[k] = c->f[CW_T_INIT][k];
      c->qv_base_1d[k] = c->f[CW_QV_BASE][k];
      c->z_base[k] = 0.5 * (phb[k] + phb[k + 1]) / g;
    }
  } catch (const std::exception&) {
    return -3;
  }
  return 0;
}

int cw_default_lam_params(cw_lam_params* p) {
  if (!p) return -1;
  p->seed = 1;
  p->t_surf = 290.0;
  p->lapse = 0.0065;
  p->t_strat = 216.65;
  p->p_surf = 1.0e5;
  p->hill_height = 1500.0;
  p->hill_halfwidth = -1.0;  // < 0: a tenth of the domain's width
  p->orog_max = 800.0;
  p->u_mean = 10.0;
  p->u_pert = 2.0;
  p->rh_mean = 0.70;
  p->rh_pert = 0.15;
  p->q_patch_max = 1.0e-3;
  p->theta_pert = 0.0;
  p->wind_pert = 0.0;
  p->etac = 0.2;
  p->hybrid_opt = 2;
  return 0;
}

namespace {
// splitmix64: the generator's only source of randomness
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * 0x1.0p-53; }  // [0, 1)
};
// a smooth random field in [-1, 1]: a few Fourier modes with random phases, amplitudes ~ |k|^-slope
struct Noise {
  struct Mode { double kx, ky, kz, ph, a; };
  std::vector<Mode> m;
  double norm = 1;
  Noise(Rng& r, double Lx, double Ly, double Lz, int nmodes, double slope, int kmax) {
    const double pi = std::numbers::pi;
    double sum = 0;
    for (int n = 0; n < nmodes; ++n) {
      const int ix = 1 + int(r.uniform() * kmax), iy = int(r.uniform() * (kmax + 1)), iz = int(r.uniform() * 3);
      const double kk = std::sqrt(double(ix * ix + iy * iy));
      Mode md{2 * pi * ix / Lx * (r.uniform() < 0.5 ? -1 : 1), Ly > 0 ? 2 * pi * iy / Ly : 0.0, Lz > 0 ? pi * iz / Lz : 0.0,
              2 * pi * r.uniform(), std::pow(kk, -slope)};
      sum += md.a;
      m.push_back(md);
    }
    norm = sum > 0 ? 1.0 / sum : 1.0;
  }
  double operator()(double x, double y, double z) const {
    double v = 0;
    for (const Mode& md : m) v += md.a * std::cos(md.kx * x + md.ky * y + md.kz * z + md.ph);
    return v * norm;
  }
};
}  // namespace

// A limited-area domain with terrain, the hybrid sigma-pressure coordinate, moisture and specified boundaries.
//   Vertical: stretched eta levels; hybrid_opt 2 coefficients with etac as WRF computes them (the formula of
//   CPPWRF's src/cases/wrf_ideal.cpp:275-306). Base state: a dry T(z) profile, T_surf - lapse z up to the
//   isothermal t_strat, in hydrostatic balance; the base fields at each column's hybrid pressure levels as
//   WRF's real-data base state is formed (pb from c3h, c4h and mub; t_init, alb from T(pb); phb integrated
//   from g ht, the discrete relation of src/cases/real_case.cpp:269-280). Terrain: a Gaussian hill in the
//   middle plus seeded spectral orography (power ~ k^-3), 0 .. orog_max. State: theta_m from the base
//   theta and qv = RH qsat (RH = rh_mean +- rh_pert, seeded); p' = 0, mu' = 0, al and ph' from the
//   equation of state and the discrete hydrostatic relation (as cases::initialize); u = u_mean + noise,
//   v = noise (+- u_pert); w from the kinematic surface condition, filled up with znw^2 (start_em);
//   species 1.. of the moist set (qc, qr, qi, qs) and tracers: seeded patches up to q_patch_max.
//   Boundaries: slabs of the initial state, coupled as WRF's boundary file holds them (u, v with the face
//   column masses, t, ph, qv with the column mass), tendencies 0; qv has boundary data, the other
//   scalars take flow_dep_bdy.
int cw_gen_lam(cw_case* c, const cw_lam_params* pp) {
  if (!c || !pp) return -1;
  using namespace cw::cst;
  try {
    cw_grid& G = c->g;
    const cw_options& o = c->o;
    if (o.flat || cw::two_d(G)) return -2;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const double p_top = G.p_top > 0 ? G.p_top : 5000.0;
    G.p_top = p_top;
    c->p_top = p_top;
    Rng rng{pp->seed * 0x2545f4914f6cdd1dULL + 12345};
    // ---- dry reference profile T(z), p(z) and its inverse T(p)
    const double Ts = pp->t_surf, lap = pp->lapse, Tst = pp->t_strat, ps0 = pp->p_surf;
    const double z_tr = (Ts - Tst) / lap, ex = g / (r_d * lap);
    const double p_tr = ps0 * std::pow(Tst / Ts, ex);
    auto p_of_z = [&](double z) {
      return z < z_tr ? ps0 * std::pow((Ts - lap * z) / Ts, ex) : p_tr * std::exp(-g * (z - z_tr) / (r_d * Tst));
    };
    auto T_of_p = [&](double p) { return p >= p_tr ? Ts * std::pow(p / ps0, 1.0 / ex) : Tst; };
    // ---- eta levels (stretched) and the coefficients of set_levels
    std::vector<double> eta(nz + 1);
    {
      const double zs = 0.4, den = 1.0 - std::exp(-1.0 / zs);
      for (int k = 0; k <= nz; ++k) eta[k] = (std::exp(-double(k) / nz / zs) - std::exp(-1.0 / zs)) / den;
      eta[0] = 1.0;
      eta[nz] = 0.0;
    }
    set_levels(c, eta);
    // ---- hybrid coefficients (hybrid_opt 2; 0 keeps set_levels' terrain-following values)
    if (pp->hybrid_opt == 2) {
      const double etac = pp->etac;
      const double B1 = 2. * (etac * etac) * (1. - etac);
      const double B2 = -etac * (4. - 3. * etac - etac * etac * etac);
      const double B3 = 2. * (1. - etac * etac * etac);
      const double B4 = -(1. - etac * etac);
      const double B5 = (1. - etac) * (1. - etac) * ((1. - etac) * (1. - etac));
      std::vector<double>& znw = c->znw;
      for (int k = 0; k <= nz; ++k) {
        double v = (B1 + B2 * znw[k] + B3 * (znw[k] * znw[k]) + B4 * (znw[k] * znw[k] * znw[k])) / B5;
        if (znw[k] < etac) v = 0.;
        if (k == 0) v = 1.;
        else if (k == nz) v = 0.;
        c->c3f[k] = v;
      }
      for (int k = 0; k <= nz; ++k) c->c4f[k] = (znw[k] - c->c3f[k]) * (p1000mb - p_top);
      for (int k = 0; k < nz; ++k) {
        c->c3h[k] = (c->c3f[k + 1] + c->c3f[k]) * 0.5;
        c->c4h[k] = (c->znu[k] - c->c3h[k]) * (p1000mb - p_top);
      }
      for (int k = 1; k < nz; ++k) c->c1f[k] = (c->c3h[k] - c->c3h[k - 1]) / (c->znu[k] - c->znu[k - 1]);
      c->c1f[0] = 1.;
      c->c1f[nz] = 0.;
      for (int k = 0; k <= nz; ++k) c->c2f[k] = (1. - c->c1f[k]) * (p1000mb - p_top);
      for (int k = 0; k < nz; ++k) {
        c->c1h[k] = (c->c3f[k + 1] - c->c3f[k]) / (znw[k + 1] - znw[k]);
        c->c2h[k] = (1. - c->c1h[k]) * (p1000mb - p_top);
      }
    } else {
      for (int k = 0; k < nz; ++k) c->c4h[k] = 0.0;
    }
    // ---- terrain
    const double Lx = nx * G.dx, Ly = ny * G.dy;
    const double hw = pp->hill_halfwidth > 0 ? pp->hill_halfwidth : 0.1 * std::min(Lx, Ly);
    Noise orog(rng, Lx, Ly, 0.0, 24, 1.5, 6);
    std::vector<double> oro(size_t(nx) * ny);
    double omin = 1e300, omax = -1e300;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) oro[size_t(j) * nx + i] = orog((i + 0.5) * G.dx, (j + 0.5) * G.dy, 0.0);
    for (double v : oro) {
      omin = std::min(omin, v);
      omax = std::max(omax, v);
    }
    auto ht_at = [&](int i, int j) {
      const double x = (i + 0.5) * G.dx - 0.5 * Lx, y = (j + 0.5) * G.dy - 0.5 * Ly;
      const double hill = pp->hill_height * std::exp(-(x * x + y * y) / (hw * hw));
      const double o2 = pp->orog_max * (oro[size_t(j) * nx + i] - omin) / std::max(omax - omin, 1e-30);
      return hill + o2;
    };
    // ---- base state
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double ht = ht_at(i, j);
        c->at(CW_HT, i, j, 0) = ht;
        const double p_surf = p_of_z(ht);
        const double mub = p_surf - p_top;
        c->at(CW_MUB, i, j, 0) = mub;
        double phb = g * ht;
        c->at(CW_PHB, i, j, 0) = phb;
        for (int k = 0; k < nz; ++k) {
          const double pb = c->c3h[k] * mub + c->c4h[k] + p_top;
          const double temp = T_of_p(pb);
          const double t_init = temp * std::pow(p1000mb / pb, r_d / cp) - t0;
          const double alb = (r_d / p1000mb) * (t_init + t0) * std::pow(pb / p1000mb, cvpm);
          c->at(CW_PB, i, j, k) = pb;
          c->at(CW_T_INIT, i, j, k) = t_init;
          c->at(CW_ALB, i, j, k) = alb;
          phb = phb - c->dnw[k] * (c->c1h[k] * mub + c->c2h[k]) * alb;
          c->at(CW_PHB, i, j, k + 1) = phb;
        }
      }
    // ---- state
    Noise nrh(rng, Lx, Ly, G.ztop > 0 ? G.ztop : 20000.0, 16, 1.0, 5);
    Noise nu(rng, Lx, Ly, 15000.0, 16, 1.0, 4), nv(rng, Lx, Ly, 15000.0, 16, 1.0, 4), nth(rng, Lx, Ly, 15000.0, 16, 1.0, 4);
    std::vector<double> qv(size_t(nx) * ny * nz, 0.0);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double pb = c->at(CW_PB, i, j, k), th = c->at(CW_T_INIT, i, j, k) + t0;
          const double z = 0.5 * (c->at(CW_PHB, i, j, k) + c->at(CW_PHB, i, j, k + 1)) / g;
          const double T = th * std::pow(pb / p1000mb, r_d / cp);
          double rh = pp->rh_mean + pp->rh_pert * nrh((i + 0.5) * G.dx, (j + 0.5) * G.dy, z);
          rh = std::min(1.0, std::max(0.0, rh));
          const double es = 611.2 * std::exp(17.67 * (T - 273.15) / (T - 29.65));
          const double q = o.n_moist > 0 ? std::max(0.0, rh * ep_2 * es / std::max(pb - es, 1.0)) : 0.0;
          qv[(size_t(k) * ny + j) * nx + i] = q;
          const double thp = pp->theta_pert * nth((i + 0.5) * G.dx, (j + 0.5) * G.dy, z);
          const double thm = (th + thp) * (1.0 + rvovrd * q);
          const double alt = (r_d / p1000mb) * thm * std::pow(pb / p1000mb, cvpm);
          c->at(CW_T_2, i, j, k) = thm - t0;
          c->at(CW_ALT, i, j, k) = alt;
          c->at(CW_AL, i, j, k) = alt - c->at(CW_ALB, i, j, k);
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double mub = c->at(CW_MUB, i, j, 0);
        double ph = 0.0;
        c->at(CW_PH_2, i, j, 0) = 0.0;
        for (int k = 0; k < nz; ++k) {
          ph -= c->dnw[k] * ((c->c1h[k] * mub + c->c2h[k]) * c->at(CW_AL, i, j, k));
          c->at(CW_PH_2, i, j, k + 1) = ph;
        }
      }
    const double up = pp->u_pert + pp->wind_pert;
    const cw_layout& Lu = c->L[CW_U_2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < Lu.ny; ++j)
        for (int i = 0; i < Lu.nx; ++i)
          c->at(CW_U_2, i, j, k) = pp->u_mean + up * nu(i * G.dx, (j + 0.5) * G.dy, (k + 0.5) * 300.0);
    const cw_layout& Lv = c->L[CW_V_2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < Lv.ny; ++j)
        for (int i = 0; i < Lv.nx; ++i) c->at(CW_V_2, i, j, k) = up * nv((i + 0.5) * G.dx, j * G.dy, (k + 0.5) * 300.0);
    // moist species and tracers
    const int ns = o.n_scalars;
    for (int n = 0; n < ns; ++n) {
      std::vector<double>& q2 = c->q2[n];
      const cw_layout& L = c->Lq;
      if (n == 0 && o.n_moist > 0) {
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) q2[c->idx(L, i, j, k)] = qv[(size_t(k) * ny + j) * nx + i];
        continue;
      }
      // patches: Gaussian blobs, cloud species in the lower / ice species in the upper troposphere
      const int nb = 4;
      struct Blob { double x, y, z, r, rz, a; };
      std::vector<Blob> blobs;
      const bool ice = n == 3 || n == 4;
      for (int b = 0; b < nb; ++b)
        blobs.push_back(Blob{Lx * (0.15 + 0.7 * rng.uniform()), Ly * (0.15 + 0.7 * rng.uniform()),
                             (ice ? 6000.0 : 1500.0) + 3000.0 * rng.uniform(), (3 + 5 * rng.uniform()) * G.dx,
                             800.0 + 1200.0 * rng.uniform(), pp->q_patch_max * (0.2 + 0.8 * rng.uniform())});
#pragma omp parallel for collapse(2) schedule(static)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const double x = (i + 0.5) * G.dx, y = (j + 0.5) * G.dy;
            const double z = 0.5 * (c->at(CW_PHB, i, j, k) + c->at(CW_PHB, i, j, k + 1)) / g;
            double v = 0;
            for (const Blob& b : blobs) {
              const double d2 = ((x - b.x) * (x - b.x) + (y - b.y) * (y - b.y)) / (b.r * b.r) + (z - b.z) * (z - b.z) / (b.rz * b.rz);
              v += b.a * std::exp(-d2);
            }
            q2[c->idx(L, i, j, k)] = std::min(v, pp->q_patch_max);
          }
    }
    // qv_base (3-D): the base state is dry
    // w: the kinematic surface condition from u, v and the terrain, znw^2 upward (start_em, rk3.cpp:173-200)
    for (int id : {CW_U_2, CW_V_2, CW_T_2, CW_AL, CW_ALT, CW_PH_2, CW_W_2, CW_P, CW_MU_2, CW_MUB, CW_PB, CW_ALB, CW_T_INIT,
                   CW_PHB, CW_HT, CW_QV_BASE})
      fill_default_halo(c, id);
    for (int n = 0; n < ns; ++n) host_fill_halo(G, c->Lq, c->q2[n].data(), false, false);
    // cf1..cf3 of set_levels (hybrid coefficients do not change them)
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        auto ht = [&](int ii, int jj) { return c->at(CW_HT, ii, jj, 0); };
        auto U = [&](int ii, int jj, int kk) { return c->at(CW_U_2, ii, jj, kk); };
        auto V = [&](int ii, int jj, int kk) { return c->at(CW_V_2, ii, jj, kk); };
        const double cf1 = c->cf1, cf2 = c->cf2, cf3 = c->cf3;
        const double ws =
            c->at(CW_MSFTY, i, j, 0) * 0.5 * c->rdy *
                ((ht(i, j + 1) - ht(i, j)) * (cf1 * V(i, j + 1, 0) + cf2 * V(i, j + 1, 1) + cf3 * V(i, j + 1, 2)) +
                 (ht(i, j) - ht(i, j - 1)) * (cf1 * V(i, j, 0) + cf2 * V(i, j, 1) + cf3 * V(i, j, 2))) +
            c->at(CW_MSFTX, i, j, 0) * 0.5 * c->rdx *
                ((ht(i + 1, j) - ht(i, j)) * (cf1 * U(i + 1, j, 0) + cf2 * U(i + 1, j, 1) + cf3 * U(i + 1, j, 2)) +
                 (ht(i, j) - ht(i - 1, j)) * (cf1 * U(i, j, 0) + cf2 * U(i, j, 1) + cf3 * U(i, j, 2)));
        c->at(CW_W_2, i, j, 0) = ws;
        for (int k = 1; k <= nz; ++k) c->at(CW_W_2, i, j, k) = ws * c->znw[k] * c->znw[k];
      }
    fill_default_halo(c, CW_W_2);
    c->f[CW_U_1] = c->f[CW_U_2];
    c->f[CW_V_1] = c->f[CW_V_2];
    c->f[CW_W_1] = c->f[CW_W_2];
    c->f[CW_T_1] = c->f[CW_T_2];
    c->f[CW_PH_1] = c->f[CW_PH_2];
    c->f[CW_MU_1] = c->f[CW_MU_2];
    for (int n = 0; n < ns; ++n) c->q1[n] = c->q2[n];
    for (int k = 0; k < nz; ++k) {
      c->u_base[k] = c->at(CW_U_2, 0, 0, k);
      c->v_base[k] = c->at(CW_V_2, 0, 0, k);
      c->t_base[k] = c->at(CW_T_INIT, 0, 0, k);
      c->qv_base_1d[k] = 0.0;
      c->z_base[k] = 0.5 * (c->at(CW_PHB, 0, 0, k) + c->at(CW_PHB, 0, 0, k + 1)) / g;
    }
    // ---- boundary slabs (pos, k, b) of the coupled initial state; tendencies 0
    if (o.lbc) {
      auto mub = [&](int i, int j) { return c->at(CW_MUB, i, j, 0); };
      auto mut = [&](int i, int j) { return c->at(CW_MU_2, i, j, 0) + mub(i, j); };
      auto muu = [&](int i, int j) {  // KMu with the doubled edge column
        const int a = i == 0 ? 0 : i - 1, b = i == nx ? nx - 1 : i;
        return 0.5 * (c->at(CW_MU_2, b, j, 0) + c->at(CW_MU_2, a, j, 0) + mub(b, j) + mub(a, j));
      };
      auto muv = [&](int i, int j) {
        const int a = j == 0 ? 0 : j - 1, b = j == ny ? ny - 1 : j;
        return 0.5 * (c->at(CW_MU_2, i, b, 0) + c->at(CW_MU_2, i, a, 0) + mub(i, b) + mub(i, a));
      };
      for (int var = 0; var < 5; ++var)
        for (int side = 0; side < 4; ++side) {
          std::vector<double>& vals = c->lv[var][side];
          const int npos = cw::lbc_npos(G, var, side), nk = cw::lbc_nk(G, var);
          const int ibe = var == CW_LBC_U ? nx : nx - 1, jbe = var == CW_LBC_V ? ny : ny - 1;
          for (int b = 0; b < cw::kLbcWidth; ++b)
            for (int k = 0; k < nk; ++k)
              for (int pos = 0; pos < npos; ++pos) {
                int i, j;
                switch (side) {
                  case CW_XS: i = b; j = pos; break;
                  case CW_XE: i = ibe - b; j = pos; break;
                  case CW_YS: i = pos; j = b; break;
                  default: i = pos; j = jbe - b; break;
                }
                double v = 0;
                switch (var) {
                  case CW_LBC_U: v = c->at(CW_U_2, i, j, k) * (c->c1h[k] * muu(i, j) + c->c2h[k]); break;
                  case CW_LBC_V: v = c->at(CW_V_2, i, j, k) * (c->c1h[k] * muv(i, j) + c->c2h[k]); break;
                  case CW_LBC_T: v = c->at(CW_T_2, i, j, k) * (c->c1h[k] * mut(i, j) + c->c2h[k]); break;
                  case CW_LBC_PH: v = c->at(CW_PH_2, i, j, k) * (c->c1f[k] * mut(i, j) + c->c2f[k]); break;
                  default: v = c->at(CW_MU_2, i, j, 0); break;
                }
                vals[pos + size_t(k) * npos + size_t(b) * npos * nk] = v;
              }
        }
      if (o.n_moist > 0) {  // qv
        c->q_have[0] = 1;
        for (int side = 0; side < 4; ++side) {
          std::vector<double>& vals = c->qv[side][0];
          const int npos = side < 2 ? ny : nx;
          for (int b = 0; b < cw::kLbcWidth; ++b)
            for (int k = 0; k < nz; ++k)
              for (int pos = 0; pos < npos; ++pos) {
                int i, j;
                switch (side) {
                  case CW_XS: i = b; j = pos; break;
                  case CW_XE: i = nx - 1 - b; j = pos; break;
                  case CW_YS: i = pos; j = b; break;
                  default: i = pos; j = ny - 1 - b; break;
                }
                vals[pos + size_t(k) * npos + size_t(b) * npos * nz] =
                    c->q2[0][c->idx(c->Lq, i, j, k)] * (c->c1h[k] * mut(i, j) + c->c2h[k]);
              }
        }
      }
    }
  } catch (const std::exception&) {
    return -3;
  }
  return 0;
}

}  // extern "C"
