// SPDX-License-Identifier: GPL-3.0-or-later
// TEST INFRASTRUCTURE ONLY: drives CPPWRF's own CPU FP64 dynamics step (its sources compiled by
// oracle/Makefile into _ref/) on inputs written by oracle/refdump.py, and writes every field back.
//
//   ref_harness <input.bin> <output.bin | --time>
//   ref_harness --lam nx ny nz dx dt n_sound n_moist p_top hybrid_opt etac seed nsteps <output.bin | --time>
//
// The second form (ref_harness only, built with CW_HARNESS_LAM) makes the input in this process: a limited-area
// case (specified boundaries, terrain, every species moist) from the repository's seeded generator (cw_gen_lam of
// cppwrf_b200/csrc/cw_case.cpp, compiled into this program), serialised exactly as refdump.write_input serialises
// it. The timed step loop is the reference's own RK3::step either way; nothing of the repository's dycore takes
// part. ref_harness_own has no such form: its pow, sin, cos and log are interposed for the whole program, so the
// generator would not compute what the product library's generator computes with glibc's.
//
// Input: the cw_grid and cw_options structs (include/cw_dycore.h), the vertical arrays, the whole
// allocation of every State / Tendencies / BaseState field in CPPWRF's Layout (the same layout as this
// repository's), the boundary slabs, dtbc and the number of steps. Output: the whole allocation of every
// field after the steps, in the same order. The objects are built the way cases::Model::build builds
// them (src/cases/model.cpp:248-449): Grid, BaseState, State + scalars, Tendencies, RK3, DiffusionDriver
// (diff_opt 1 / km_opt 1), LateralBC.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "core/field.hpp"
#include "dyn/diffusion_driver.hpp"
#include "dyn/lateral_bc.hpp"
#include "dyn/rk3.hpp"
#include "dyn/state.hpp"
#include "phys/driver/phy_prep.hpp"
#include "../include/cw_dycore.h"
#ifdef CW_HARNESS_FACADE
// ref_harness_facade: the same driver with the step replaced by the repository's drop-in (RK3B200 over the C ABI,
// on the GPU); everything else -- the reference's State / Tendencies / BaseState / LateralBC / DiffusionDriver
// objects, their set-up and the output -- is unchanged
#include "../cppwrf_b200/facade/rk3_b200.hpp"
using Stepper = cppwrf_b200::RK3B200;
#else
using Stepper = cppwrf::dyn::RK3;
#endif

// The dycore links three symbols of the physics coupling that the dynamics-only configurations never call.
namespace cppwrf::dyn {
void PhysicsCoupling::step(State&, const BaseState&, double) { throw std::runtime_error("physics not linked"); }
}  // namespace cppwrf::dyn
namespace cppwrf::phys::driver {
PhyPrepFields::PhyPrepFields(const cppwrf::Grid&) { throw std::runtime_error("phy_prep not linked"); }
void run_phy_prep(const cppwrf::dyn::State&, const cppwrf::dyn::BaseState&, PhyPrepFields&, const PhyPrepParams&) {
  throw std::runtime_error("phy_prep not linked");
}
}  // namespace cppwrf::phys::driver

using namespace cppwrf;

namespace {
FILE* in_f;
FILE* out_f;
template <class T>
T rd() {
  T v;
  if (std::fread(&v, sizeof v, 1, in_f) != 1) throw std::runtime_error("input truncated");
  return v;
}
std::vector<double> rdv(size_t n) {
  std::vector<double> v(n);
  if (n && std::fread(v.data(), sizeof(double), n, in_f) != n) throw std::runtime_error("input truncated");
  return v;
}
void load(real* base_ptr, const Layout& L) {
  const int64_t n = rd<int64_t>();
  if (n != int64_t(L.total)) throw std::runtime_error("layout mismatch: " + std::to_string(n) + " vs " + std::to_string(L.total));
  std::vector<double> v = rdv(size_t(n));
  std::memcpy(base_ptr, v.data(), size_t(n) * sizeof(double));
}
void save(const real* base_ptr, const Layout& L) {
  const int64_t n = int64_t(L.total);
  std::fwrite(&n, sizeof n, 1, out_f);
  std::fwrite(base_ptr, sizeof(double), size_t(n), out_f);
}

#ifdef CW_HARNESS_LAM
// the input bytes of a limited-area case made by cw_gen_lam, in refdump.write_input's order
struct Bytes {
  std::vector<char> b;
  template <class T>
  void put(const T& v) {
    const char* p = reinterpret_cast<const char*>(&v);
    b.insert(b.end(), p, p + sizeof(T));
  }
  void put_n(const double* p, size_t n) {
    const char* c = reinterpret_cast<const char*>(p);
    b.insert(b.end(), c, c + n * sizeof(double));
  }
};
void check_rc(int rc, const char* what) {
  if (rc != 0) throw std::runtime_error(std::string(what) + " failed");
}
std::vector<char> lam_input(char** a) {
  cw_grid g{};
  g.nx = std::atoi(a[0]); g.ny = std::atoi(a[1]); g.nz = std::atoi(a[2]);
  g.dx = g.dy = std::atof(a[3]); g.dt = std::atof(a[4]); g.ztop = 0.0; g.p_top = std::atof(a[7]);
  g.bc_x = g.bc_y = CW_BC_SPECIFIED;
  cw_options o{};
  check_rc(cw_default_options(&o), "cw_default_options");
  o.flat = 0; o.lbc = 1; o.precision = CW_FP64;
  o.time_step_sound = std::atoi(a[5]);
  o.n_moist = o.n_scalars = std::atoi(a[6]);
  cw_lam_params p{};
  check_rc(cw_default_lam_params(&p), "cw_default_lam_params");
  p.hybrid_opt = std::atoi(a[8]); p.etac = std::atof(a[9]); p.seed = std::strtoull(a[10], nullptr, 10);
  const int nsteps = std::atoi(a[11]);
  cw_case* c = nullptr;
  check_rc(cw_case_create(&g, &o, &c), "cw_case_create");
  std::unique_ptr<cw_case, int (*)(cw_case*)> own(c, cw_case_destroy);
  check_rc(cw_gen_lam(c, &p), "cw_gen_lam");
  check_rc(cw_case_config(c, &g, &o), "cw_case_config");
  cw_vertical v{};
  check_rc(cw_case_vertical(c, &v), "cw_case_vertical");
  g.p_top = v.p_top;  // the generator sets the model top
  Bytes B;
  B.put(g);
  B.put(o);
  const int nz = g.nz;
  const std::vector<double> zeros(size_t(nz) + 1, 0.0);
  auto arr = [&](const double* x, int n) { B.put_n(x ? x : zeros.data(), size_t(n)); };
  for (const double* x : {v.znu, v.dnw, v.rdnw, v.c1h, v.c2h, v.c3h, v.c4h}) arr(x, nz);
  for (const double* x : {v.znw, v.dn, v.rdn, v.fnm, v.fnp, v.c1f, v.c2f, v.c3f, v.c4f}) arr(x, nz + 1);
  for (const double* x : {v.u_base, v.v_base, v.t_base, v.qv_base_1d, v.z_base}) arr(x, nz);
  for (double x : {v.cf1, v.cf2, v.cf3, v.cfn, v.cfn1, v.rdx, v.rdy, v.p_top, v.t0}) B.put(x);
  auto field = [&](int id, int n) {
    double* d = nullptr;
    cw_layout L{};
    check_rc(cw_case_field(c, id, n, &d, &L), "cw_case_field");
    B.put(int64_t(L.total));
    B.put_n(d, size_t(L.total));
  };
  for (int id = 0; id < CW_Q_1; ++id) field(id, 0);
  for (int n = 0; n < o.n_scalars; ++n)
    for (int id : {CW_Q_1, CW_Q_2, CW_Q_TENDF}) field(id, n);
  for (int scalar = 0; scalar < 2; ++scalar)
    for (int var = 0; var < (scalar ? o.n_scalars : 5); ++var)
      for (int side = 0; side < 4; ++side) {
        double *vals = nullptr, *tends = nullptr;
        size_t cnt = 0;
        if (cw_case_lbc(c, scalar, var, side, &vals, &tends, &cnt) != 0) {
          if (!scalar) throw std::runtime_error("cw_case_lbc failed");
          B.put(int64_t(0));
          continue;
        }
        B.put(int64_t(cnt));
        B.put_n(vals, cnt);
        B.put_n(tends, cnt);
      }
  double dtbc = 0;
  check_rc(cw_case_lbc_time(c, &dtbc), "cw_case_lbc_time");
  B.put(dtbc);
  B.put(int32_t(nsteps));
  return std::move(B.b);
}
#else
std::vector<char> lam_input(char**) { throw std::runtime_error("--lam: built without the case generator"); }
#endif
}  // namespace

int main(int argc, char** argv) {
  const bool gen = argc >= 2 && std::strcmp(argv[1], "--lam") == 0;
  if (gen ? argc != 15 : (argc != 3 && argc != 4)) {
    std::fprintf(stderr,
                 "usage: ref_harness input.bin output.bin [--time]\n"
                 "       ref_harness --lam nx ny nz dx dt n_sound n_moist p_top hybrid_opt etac seed nsteps <output.bin|--time>\n");
    return 2;
  }
  // the output path, or timing only (the step loop's wall time, no output)
  const char* out_path = gen ? argv[14] : argv[2];
  const bool time_only = gen ? std::strcmp(argv[14], "--time") == 0 : argc == 4;
  try {
    std::vector<char> generated;
    if (gen) {
      generated = lam_input(argv + 2);
      in_f = fmemopen(generated.data(), generated.size(), "rb");
    } else {
      in_f = std::fopen(argv[1], "rb");
    }
    if (!in_f) throw std::runtime_error("cannot open input");
    const cw_grid cg = rd<cw_grid>();
    const cw_options co = rd<cw_options>();
    Grid g;
    g.nx = cg.nx; g.ny = cg.ny; g.nz = cg.nz; g.dx = cg.dx; g.dy = cg.dy; g.dt = cg.dt; g.ztop = cg.ztop; g.p_top = cg.p_top;
    g.bc_x = BC(cg.bc_x); g.bc_y = BC(cg.bc_y);
    const int nz = g.nz;
    dyn::BaseState b(g, co.flat != 0, co.mapped != 0);
    b.coriolis = co.coriolis != 0;
    // vertical arrays: znu dnw rdnw c1h c2h c3h c4h (nz), znw dn rdn fnm fnp c1f c2f c3f c4f (nz+1),
    // u_base v_base t_base qv_base_1d z_base (nz), then cf1 cf2 cf3 cfn cfn1 rdx rdy p_top t0
    Array1* a_nz[] = {&b.znu, &b.dnw, &b.rdnw, &b.c1h, &b.c2h, &b.c3h, &b.c4h};
    Array1* a_nz1[] = {&b.znw, &b.dn, &b.rdn, &b.fnm, &b.fnp, &b.c1f, &b.c2f, &b.c3f, &b.c4f};
    Array1* a_base[] = {&b.u_base, &b.v_base, &b.t_base, &b.qv_base_1d, &b.z_base};
    for (Array1* a : a_nz) { auto v = rdv(nz); for (int k = 0; k < nz; ++k) (*a)[k] = v[k]; }
    for (Array1* a : a_nz1) { auto v = rdv(nz + 1); for (int k = 0; k <= nz; ++k) (*a)[k] = v[k]; }
    for (Array1* a : a_base) { auto v = rdv(nz); for (int k = 0; k < nz; ++k) (*a)[k] = v[k]; }
    b.cf1 = rd<double>(); b.cf2 = rd<double>(); b.cf3 = rd<double>(); b.cfn = rd<double>(); b.cfn1 = rd<double>();
    b.rdx = rd<double>(); b.rdy = rd<double>(); b.p_top = rd<double>(); b.t0 = rd<double>();
    b.upload_levels();
    dyn::State s(g);
    dyn::Tendencies t(g);
    static const char* moist_names[] = {"qv", "qc", "qr", "qi", "qs", "qg"};
    for (int n = 0; n < co.n_scalars; ++n) {
      const bool moist = n < co.n_moist;
      const std::string name = moist ? moist_names[n] : "tracer" + std::to_string(n);
      s.add_scalar(g, name, moist);
      t.add_scalar(g, name);
    }
    // fields in cw_field order
    auto state3 = [&](int id) -> Field3* {
      switch (id) {
        case CW_U_1: return &s.u_1; case CW_U_2: return &s.u_2; case CW_V_1: return &s.v_1; case CW_V_2: return &s.v_2;
        case CW_W_1: return &s.w_1; case CW_W_2: return &s.w_2; case CW_T_1: return &s.t_1; case CW_T_2: return &s.t_2;
        case CW_PH_1: return &s.ph_1; case CW_PH_2: return &s.ph_2; case CW_P: return &s.p; case CW_AL: return &s.al;
        case CW_ALT: return &s.alt; case CW_PHP: return &s.php; case CW_WW: return &s.ww; case CW_RU: return &s.ru;
        case CW_RV: return &s.rv; case CW_RW: return &s.rw; case CW_RU_M: return &s.ru_m; case CW_RV_M: return &s.rv_m;
        case CW_WW_M: return &s.ww_m; case CW_RU_TEND: return &t.ru_tend; case CW_RV_TEND: return &t.rv_tend;
        case CW_RW_TEND: return &t.rw_tend; case CW_T_TEND: return &t.t_tend; case CW_PH_TEND: return &t.ph_tend;
        case CW_RU_TENDF: return &t.ru_tendf; case CW_RV_TENDF: return &t.rv_tendf; case CW_RW_TENDF: return &t.rw_tendf;
        case CW_T_TENDF: return &t.t_tendf; case CW_PH_TENDF: return &t.ph_tendf;
        case CW_CQU: return co.n_moist ? &s.cqu : nullptr; case CW_CQV: return co.n_moist ? &s.cqv : nullptr;
        case CW_CQW: return co.n_moist ? &s.cqw : nullptr; case CW_H_DIABATIC: return co.n_moist ? &s.h_diabatic : nullptr;
        default: return nullptr;
      }
    };
    auto state2 = [&](int id) -> Field2* {
      switch (id) {
        case CW_MU_1: return &s.mu_1; case CW_MU_2: return &s.mu_2; case CW_MUT: return &s.mut; case CW_MUU: return &s.muu;
        case CW_MUV: return &s.muv; case CW_MUTS: return &s.muts; case CW_MUUS: return &s.muus; case CW_MUVS: return &s.muvs;
        case CW_MU_TEND: return &t.mu_tend;
        default: return nullptr;
      }
    };
    auto base3 = [&](int id) -> BaseField3* {
      switch (id) {
        case CW_PB: return &b.pb; case CW_ALB: return &b.alb; case CW_T_INIT: return &b.t_init;
        case CW_QV_BASE: return &b.qv_base; case CW_PHB: return &b.phb;
        default: return nullptr;
      }
    };
    auto base2 = [&](int id) -> BaseField2* {
      switch (id) {
        case CW_MUB: return &b.mub; case CW_HT: return &b.ht; case CW_MSFTX: return &b.msftx; case CW_MSFTY: return &b.msfty;
        case CW_MSFUX: return &b.msfux; case CW_MSFUY: return &b.msfuy; case CW_MSFVX: return &b.msfvx;
        case CW_MSFVY: return &b.msfvy; case CW_MSFVX_INV: return &b.msfvx_inv; case CW_F: return &b.f; case CW_E: return &b.e;
        case CW_SINA: return &b.sina; case CW_COSA: return &b.cosa;
        default: return nullptr;
      }
    };
    auto each_field = [&](auto&& fn3, auto&& fnb, auto&& missing) {
      for (int id = 0; id < CW_Q_1; ++id) {
        if (Field3* f = state3(id)) fn3(f->data() - f->layout().offset, f->layout());
        else if (Field2* f2 = state2(id)) fn3(f2->data() - f2->layout().offset, f2->layout());
        else if (BaseField3* bf = base3(id)) fnb(bf->data() - bf->layout().offset, bf->layout());
        else if (BaseField2* bf2 = base2(id)) fnb(bf2->data() - bf2->layout().offset, bf2->layout());
        else missing();  // a field the reference allocates only with moisture
      }
      for (int n = 0; n < co.n_scalars; ++n) {
        fn3(s.q_1[n].data() - s.q_1[n].layout().offset, s.q_1[n].layout());
        fn3(s.q_2[n].data() - s.q_2[n].layout().offset, s.q_2[n].layout());
        fn3(t.q_tendf[n].data() - t.q_tendf[n].layout().offset, t.q_tendf[n].layout());
      }
    };
    each_field([&](real* p, const Layout& L) { load(p, L); }, [&](const real* p, const Layout& L) { load(const_cast<real*>(p), L); },
               [&] {
                 const int64_t n = rd<int64_t>();
                 rdv(size_t(n));
               });
    // boundary slabs
    std::unique_ptr<dyn::LateralBC> bc;
    if (co.lbc) {
      bc = std::make_unique<dyn::LateralBC>(g, g.dt);
      for (int var = 0; var < 5; ++var)
        for (int side = 0; side < 4; ++side) {
          const int64_t n = rd<int64_t>();
          auto v = rdv(size_t(n)), tt = rdv(size_t(n));
          bc->set(dyn::LateralBC::Var(var), dyn::LateralBC::Side(side), v, tt);
        }
      for (int q = 0; q < co.n_scalars; ++q)
        for (int side = 0; side < 4; ++side) {
          const int64_t n = rd<int64_t>();
          if (n == 0) continue;
          auto v = rdv(size_t(n)), tt = rdv(size_t(n));
          bc->set_scalar(q, dyn::LateralBC::Side(side), v, tt);
        }
      bc->dtbc = rd<double>();
    }
    const int nsteps = rd<int32_t>();
    std::fclose(in_f);
    dyn::LargeStepParams lp;
    lp.khdif = co.khdif; lp.kvdif = co.kvdif; lp.pr_inv = co.pr_inv; lp.top_lid = co.top_lid != 0;
    lp.h_adv_order = co.h_adv_order; lp.v_adv_order = co.v_adv_order; lp.w_damping = co.w_damping; lp.w_crit_cfl = co.w_crit_cfl;
    dyn::AcousticParams ap;
    ap.epssm = co.epssm; ap.smdiv = co.smdiv; ap.emdiv = co.emdiv; ap.top_lid = co.top_lid != 0; ap.damp_opt = co.damp_opt;
    ap.hypsometric_opt = co.hypsometric_opt; ap.zdamp = co.zdamp; ap.dampcoef = co.dampcoef;
    dyn::ScalarParams sp;
    sp.moist_adv_opt = co.moist_adv_opt; sp.scalar_adv_opt = co.scalar_adv_opt; sp.tke_adv_opt = co.tke_adv_opt;
    sp.h_adv_order = co.h_adv_order; sp.v_adv_order = co.v_adv_order;
    Stepper rk(g, lp, ap, co.time_step_sound, sp);
    std::unique_ptr<dyn::DiffusionDriver> dd;
    if (co.diff_opt == 1 || co.diff_6th_opt != 0 || co.damp_opt == 2) {  // DiffusionConfig::on (model.cpp:439)
      dyn::DiffusionConfig dc;
      dc.diff_opt = co.diff_opt; dc.km_opt = co.km_opt; dc.damp_opt = co.damp_opt; dc.zdamp = co.zdamp; dc.dampcoef = co.dampcoef;
      dc.diff_6th_opt = co.diff_6th_opt; dc.diff_6th_factor = co.diff_6th_factor;
      dc.khdif = co.khdif; dc.kvdif = co.kvdif; dc.prandtl = real(1.0) / co.pr_inv;
      dd = std::make_unique<dyn::DiffusionDriver>(g, dc);
      rk.set_diffusion(dd.get());
    }
    if (bc) rk.set_lateral_bc(bc.get());
    const auto t0 = std::chrono::steady_clock::now();
    for (int n = 0; n < nsteps; ++n) rk.step(s, t, b);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (time_only) {
      std::printf("STEP_SECONDS %.9f\n", secs);
      return 0;
    }
    out_f = std::fopen(out_path, "wb");
    if (!out_f) throw std::runtime_error("cannot open output");
    each_field([&](real* p, const Layout& L) { save(p, L); }, [&](const real* p, const Layout& L) { save(p, L); },
               [&] {
                 const int64_t n = 0;
                 std::fwrite(&n, sizeof n, 1, out_f);
               });
    std::fclose(out_f);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_harness: %s\n", e.what());
    return 1;
  }
  return 0;
}
