// SPDX-License-Identifier: GPL-3.0-or-later
// RK3B200: a drop-in for CPPWRF's dyn::RK3 (src/dyn/rk3.hpp:36-77) that runs the step on a B200 through this
// library's C ABI (include/cw_dycore.h). Header-only: a CPPWRF build includes it (with CPPWRF's src/ and this
// repository's include/ on the include path) and links libcw_dycore.so; the driver loop then reads
//
//     cppwrf_b200::RK3B200 rk(grid, large_step_params, acoustic_params, time_step_sound, scalar_params);
//     rk.set_lateral_bc(&bc);  rk.set_diffusion(&dd);           // as with dyn::RK3
//     for (...) rk.step(state, tend, base);                      // src/main.cpp:98, unchanged
//
// The fields of State / Tendencies / BaseState keep CPPWRF's layout (Layout::make), which is also the C ABI's,
// so they move as whole allocations. step() is RK3::step (src/dyn/rk3.cpp:86-170): the caller's State,
// Tendencies and boundary slabs are uploaded, one step runs on the device, State and Tendencies come back, and
// LateralBC::dtbc advances by dt as LateralBC::advance_time would. With pow interposed by cw_pow on the CPU side
// the results equal RK3::step's bit for bit (the plain FP64 form). The BaseState is uploaded at the first step;
// call reload_base() after changing it. The fields must be host memory (CPPWRF's CPU build); with device-resident
// fields (its CUDA build) copy through cw_field_device_ptr instead.
//
// Supported as by cw_create: diff_opt 0 / 1 with km_opt 1 / 4, the sixth-order filter, damp_opt 0-3,
// hypsometric_opt 1 / 2, specified / open / periodic / symmetric boundaries, Kessler microphysics
// (enable_physics with mp_physics 1). Column physics (set_column_physics) is not: it throws.
#pragma once

#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "cw_dycore.h"
#include "dyn/diffusion_driver.hpp"
#include "dyn/lateral_bc.hpp"
#include "dyn/rk3.hpp"
#include "dyn/state.hpp"

namespace cppwrf_b200 {

namespace dyn = cppwrf::dyn;

class RK3B200 {
 public:
  RK3B200(const cppwrf::Grid& g, const dyn::LargeStepParams& lp, const dyn::AcousticParams& ap, int time_step_sound,
          const dyn::ScalarParams& sp = {})
      : g_(g), lp_(lp), ap_(ap), sp_(sp), tss_(time_step_sound) {
    if (g.patched()) throw std::runtime_error("RK3B200: a decomposed (patched) grid is not supported");
    n_sound_ = time_step_sound > 0 ? time_step_sound : dyn::RK3::auto_sound_steps(g.dt, g.dx, g.dy);
  }
  ~RK3B200() { cw_destroy(h_); }
  RK3B200(const RK3B200&) = delete;
  RK3B200& operator=(const RK3B200&) = delete;

  static int auto_sound_steps(double dt, double dx, double dy) { return dyn::RK3::auto_sound_steps(dt, dx, dy); }
  int n_sound() const { return n_sound_; }
  // RK3::set_dt (rk3.cpp:79-84): the large step and the acoustic step count of the next steps
  void set_dt(double dt, int n_sound) {
    if (n_sound < 2 || n_sound % 2) throw std::runtime_error("time_step_sound must be even and >= 2");
    g_.dt = dt;
    n_sound_ = n_sound;
    if (h_) check(cw_set_dt(h_, dt, n_sound), "cw_set_dt");
  }
  // RK3::on_cfl: the vertical and horizontal CFL maxima of each stage, reported after the step in stage order
  std::function<void(cppwrf::real, cppwrf::real)> on_cfl;
  void enable_physics(const dyn::PhysicsParams& pp) {
    if (pp.mp_physics != 0 && pp.mp_physics != 1) throw std::runtime_error("RK3B200: only mp_physics 0 and 1 (Kessler)");
    mp_physics_ = pp.mp_physics;
    mp_tend_lim_ = pp.mp_tend_lim;
  }
  void set_lateral_bc(dyn::LateralBC* bc) { bc_ = bc; }
  void set_diffusion(dyn::DiffusionDriver* d) { dd_ = d; }
  void set_column_physics(void*) { throw std::runtime_error("RK3B200: column physics is not supported"); }
  void reload_base() { base_loaded_ = false; }
  cw_handle* handle() const { return h_; }

  void step(dyn::State& s, dyn::Tendencies& t, const dyn::BaseState& b) {
    if (!h_) create(s, b);
    if (!base_loaded_) load_base(b);
    for_fields(s, t, [&](int id, int n, cppwrf::real* base, const cppwrf::Layout& L) {
      check(cw_upload(h_, id, n, base, size_t(L.total)), "cw_upload");
    });
    if (bc_) load_boundaries(s);
    check(cw_step(h_, 1), "cw_step");
    for_fields(s, t, [&](int id, int n, cppwrf::real* base, const cppwrf::Layout& L) {
      check(cw_download(h_, id, n, base, size_t(L.total)), "cw_download");
    });
    if (bc_) bc_->advance_time(g_.dt);
    if (on_cfl) {
      double v[3], hz[3];
      check(cw_cfl_max(h_, 0, v, hz), "cw_cfl_max");
      for (int rk = 0; rk < 3; ++rk) on_cfl(cppwrf::real(v[rk]), cppwrf::real(hz[rk]));
    }
  }

 private:
  static void check(int rc, const char* what) {
    if (rc != 0) {
      const char* e = cw_last_error(nullptr);
      throw std::runtime_error(std::string("RK3B200: ") + what + " failed: " + (e ? e : ""));
    }
  }
  void check_h(int rc, const char* what) const {
    if (rc != 0) throw std::runtime_error(std::string("RK3B200: ") + what + " failed: " + cw_last_error(h_));
  }

  void create(const dyn::State& s, const dyn::BaseState& b) {
    cw_grid cg{};
    cg.nx = g_.nx; cg.ny = g_.ny; cg.nz = g_.nz; cg.dx = g_.dx; cg.dy = g_.dy; cg.dt = g_.dt; cg.ztop = g_.ztop;
    cg.p_top = g_.p_top; cg.bc_x = int(g_.bc_x); cg.bc_y = int(g_.bc_y);
    cw_options o{};
    check(cw_default_options(&o), "cw_default_options");
    o.khdif = lp_.khdif; o.kvdif = lp_.kvdif; o.pr_inv = lp_.pr_inv; o.top_lid = lp_.top_lid ? 1 : 0;
    o.h_adv_order = lp_.h_adv_order; o.v_adv_order = lp_.v_adv_order; o.w_damping = lp_.w_damping;
    o.w_crit_cfl = lp_.w_crit_cfl;
    o.epssm = ap_.epssm; o.smdiv = ap_.smdiv; o.emdiv = ap_.emdiv; o.damp_opt = ap_.damp_opt;
    o.hypsometric_opt = ap_.hypsometric_opt; o.zdamp = ap_.zdamp; o.dampcoef = ap_.dampcoef;
    o.moist_adv_opt = sp_.moist_adv_opt; o.scalar_adv_opt = sp_.scalar_adv_opt; o.tke_adv_opt = sp_.tke_adv_opt;
    o.time_step_sound = n_sound_;
    o.diff_opt = 0;
    if (dd_) {  // DiffusionConfig (diffusion_driver.hpp:24-49)
      const dyn::DiffusionConfig& c = dd_->config();
      o.diff_opt = c.diff_opt; o.km_opt = c.km_opt; o.damp_opt = c.damp_opt > 0 && c.damp_opt < 3 ? c.damp_opt : o.damp_opt;
      if (c.damp_opt == 1 || c.damp_opt == 2) { o.zdamp = c.zdamp; o.dampcoef = c.dampcoef; }
      // prandtl: the library takes 1 / pr_inv of LargeStepParams (a driver sets both from the namelist's pr_inv)
      o.khdif = c.khdif; o.kvdif = c.kvdif;
      o.diff_6th_opt = c.diff_6th_opt; o.diff_6th_factor = c.diff_6th_factor;
    }
    o.flat = b.flat ? 1 : 0;
    o.mapped = b.mapped ? 1 : 0;
    o.coriolis = b.coriolis ? 1 : 0;
    o.n_moist = s.n_moist;
    o.n_scalars = s.n_scalars();
    o.lbc = bc_ ? 1 : 0;
    o.precision = CW_FP64;
    o.mp_physics = mp_physics_;
    o.mp_tend_lim = mp_tend_lim_;
    check(cw_create(&cg, &o, &h_), "cw_create");
    check_h(cw_set_autotune(h_, 1), "cw_set_autotune");  // the first six steps pick the kernels' shapes (same values)
    if (on_cfl) check_h(cw_set_cfl_diagnostics(h_, 1), "cw_set_cfl_diagnostics");
  }

  void load_base(const dyn::BaseState& b) {
    const int nz = g_.nz;
    auto arr = [&](const cppwrf::Array1& a, int n) {
      std::vector<double> out(static_cast<size_t>(n));
      for (int k = 0; k < n; ++k) out[static_cast<size_t>(k)] = a[k];
      return out;
    };
    std::vector<double> znu = arr(b.znu, nz), dnw = arr(b.dnw, nz), rdnw = arr(b.rdnw, nz), c1h = arr(b.c1h, nz),
                        c2h = arr(b.c2h, nz), c3h = arr(b.c3h, nz), c4h = arr(b.c4h, nz);
    std::vector<double> znw = arr(b.znw, nz + 1), dn = arr(b.dn, nz + 1), rdn = arr(b.rdn, nz + 1),
                        fnm = arr(b.fnm, nz + 1), fnp = arr(b.fnp, nz + 1), c1f = arr(b.c1f, nz + 1),
                        c2f = arr(b.c2f, nz + 1), c3f = arr(b.c3f, nz + 1), c4f = arr(b.c4f, nz + 1);
    std::vector<double> ub = arr(b.u_base, nz), vb = arr(b.v_base, nz), tb = arr(b.t_base, nz),
                        qb = arr(b.qv_base_1d, nz), zb = arr(b.z_base, nz);
    cw_vertical v{};
    v.znu = znu.data(); v.dnw = dnw.data(); v.rdnw = rdnw.data(); v.c1h = c1h.data(); v.c2h = c2h.data();
    v.c3h = c3h.data(); v.c4h = c4h.data();
    v.znw = znw.data(); v.dn = dn.data(); v.rdn = rdn.data(); v.fnm = fnm.data(); v.fnp = fnp.data();
    v.c1f = c1f.data(); v.c2f = c2f.data(); v.c3f = c3f.data(); v.c4f = c4f.data();
    v.u_base = ub.data(); v.v_base = vb.data(); v.t_base = tb.data(); v.qv_base_1d = qb.data(); v.z_base = zb.data();
    v.cf1 = b.cf1; v.cf2 = b.cf2; v.cf3 = b.cf3; v.cfn = b.cfn; v.cfn1 = b.cfn1; v.rdx = b.rdx; v.rdy = b.rdy;
    v.p_top = b.p_top; v.t0 = b.t0;
    check_h(cw_set_vertical(h_, &v), "cw_set_vertical");
    auto up = [&](int id, const auto& f) {
      const cppwrf::Layout& L = f.layout();
      check_h(cw_upload(h_, id, 0, f.data() - L.offset, size_t(L.total)), "cw_upload (base)");
    };
    up(CW_MUB, b.mub); up(CW_PB, b.pb); up(CW_ALB, b.alb); up(CW_T_INIT, b.t_init); up(CW_QV_BASE, b.qv_base);
    up(CW_PHB, b.phb); up(CW_HT, b.ht); up(CW_MSFTX, b.msftx); up(CW_MSFTY, b.msfty); up(CW_MSFUX, b.msfux);
    up(CW_MSFUY, b.msfuy); up(CW_MSFVX, b.msfvx); up(CW_MSFVY, b.msfvy); up(CW_MSFVX_INV, b.msfvx_inv);
    up(CW_F, b.f); up(CW_E, b.e); up(CW_SINA, b.sina); up(CW_COSA, b.cosa);
    base_loaded_ = true;
  }

  // every State / Tendencies field the step reads or writes, with its C ABI id (State order of the header)
  template <class F>
  void for_fields(dyn::State& s, dyn::Tendencies& t, F fn) const {
    auto one = [&](int id, int n, auto& f) {
      const cppwrf::Layout& L = f.layout();
      fn(id, n, f.data() - L.offset, L);
    };
    one(CW_U_1, 0, s.u_1); one(CW_U_2, 0, s.u_2); one(CW_V_1, 0, s.v_1); one(CW_V_2, 0, s.v_2);
    one(CW_W_1, 0, s.w_1); one(CW_W_2, 0, s.w_2); one(CW_T_1, 0, s.t_1); one(CW_T_2, 0, s.t_2);
    one(CW_PH_1, 0, s.ph_1); one(CW_PH_2, 0, s.ph_2); one(CW_MU_1, 0, s.mu_1); one(CW_MU_2, 0, s.mu_2);
    one(CW_P, 0, s.p); one(CW_AL, 0, s.al); one(CW_ALT, 0, s.alt); one(CW_PHP, 0, s.php); one(CW_WW, 0, s.ww);
    one(CW_MUT, 0, s.mut); one(CW_MUU, 0, s.muu); one(CW_MUV, 0, s.muv); one(CW_MUTS, 0, s.muts);
    one(CW_MUUS, 0, s.muus); one(CW_MUVS, 0, s.muvs); one(CW_RU, 0, s.ru); one(CW_RV, 0, s.rv); one(CW_RW, 0, s.rw);
    one(CW_RU_M, 0, s.ru_m); one(CW_RV_M, 0, s.rv_m); one(CW_WW_M, 0, s.ww_m);
    if (s.n_moist > 0) {
      one(CW_CQU, 0, s.cqu); one(CW_CQV, 0, s.cqv); one(CW_CQW, 0, s.cqw); one(CW_H_DIABATIC, 0, s.h_diabatic);
    }
    one(CW_RU_TEND, 0, t.ru_tend); one(CW_RV_TEND, 0, t.rv_tend); one(CW_RW_TEND, 0, t.rw_tend);
    one(CW_T_TEND, 0, t.t_tend); one(CW_PH_TEND, 0, t.ph_tend); one(CW_MU_TEND, 0, t.mu_tend);
    one(CW_RU_TENDF, 0, t.ru_tendf); one(CW_RV_TENDF, 0, t.rv_tendf); one(CW_RW_TENDF, 0, t.rw_tendf);
    one(CW_T_TENDF, 0, t.t_tendf); one(CW_PH_TENDF, 0, t.ph_tendf);
    for (int n = 0; n < s.n_scalars(); ++n) {
      one(CW_Q_1, n, s.q_1[size_t(n)]);
      one(CW_Q_2, n, s.q_2[size_t(n)]);
      one(CW_Q_TENDF, n, t.q_tendf[size_t(n)]);
    }
  }

  // LateralBC::set / set_scalar's slabs (values and tendencies, (pos, k, b) pos fastest) and dtbc
  void load_boundaries(const dyn::State& s) {
    using LB = dyn::LateralBC;
    for (int var = 0; var < 5; ++var) {
      const LB::Var v = LB::Var(var);
      if (!bc_->has(v)) continue;
      for (int side = 0; side < 4; ++side) {
        const LB::Side sd = LB::Side(side);
        const size_t n = size_t(bc_->slab_npos(v, sd)) * size_t(bc_->slab_nk(v)) * size_t(bc_->width());
        check_h(cw_set_lbc(h_, var, side, bc_->slab(v, sd, false), bc_->slab(v, sd, true), n), "cw_set_lbc");
      }
    }
    for (int q = 0; q < s.n_scalars(); ++q) {
      if (!bc_->has_scalar(q)) continue;
      for (int side = 0; side < 4; ++side) {
        const LB::Side sd = LB::Side(side);
        const int npos = side < 2 ? g_.ny : g_.nx;
        const size_t n = size_t(npos) * size_t(g_.nz) * size_t(bc_->width());
        check_h(cw_set_lbc_scalar(h_, q, side, bc_->scalar_slab(q, sd, false), bc_->scalar_slab(q, sd, true), n),
                "cw_set_lbc_scalar");
      }
    }
    check_h(cw_set_lbc_time(h_, bc_->dtbc), "cw_set_lbc_time");
  }

  cppwrf::Grid g_;
  dyn::LargeStepParams lp_;
  dyn::AcousticParams ap_;
  dyn::ScalarParams sp_;
  int tss_ = 0, n_sound_ = 0;
  int mp_physics_ = 0;
  double mp_tend_lim_ = 10;
  dyn::LateralBC* bc_ = nullptr;
  dyn::DiffusionDriver* dd_ = nullptr;
  cw_handle* h_ = nullptr;
  bool base_loaded_ = false;
};

}  // namespace cppwrf_b200
