// SPDX-License-Identifier: GPL-3.0-or-later
// Acoustic small step, small_step_finish + calc_p_rho_phi, scalar transport, set_w_surface (see
// kernels.cuh for the conventions). Reference: src/dyn/small_step.cpp, scalars.cpp, rk3.cpp of CPPWRF.
#pragma once

#include "kernels.cuh"

namespace cw {

// Edge (small_step.cpp:39-45): the spec zone of specified boundaries
template <class R>
__device__ __forceinline__ bool edge_mass(const Dom<R>& D, int i, int j) {
  return (D.spec_x && (i == 0 || i == D.nx - 1)) || (D.spec_y && (j == 0 || j == D.ny - 1));
}
template <class R>
__device__ __forceinline__ bool edge_uface(const Dom<R>& D, int i, int j) {
  return (D.spec_x && (i <= 0 || i >= D.nx)) || (D.spec_y && (j == 0 || j == D.ny - 1));
}
template <class R>
__device__ __forceinline__ bool edge_vface(const Dom<R>& D, int i, int j) {
  return (D.spec_x && (i == 0 || i == D.nx - 1)) || (D.spec_y && (j <= 0 || j >= D.ny));
}
template <class R>
__device__ __forceinline__ R mh_(const Dom<R>& D, int k, R m) { return R(D.c1h[k]) * m + R(D.c2h[k]); }
template <class R>
__device__ __forceinline__ R mf_(const Dom<R>& D, int k, R m) { return R(D.c1f[k]) * m + R(D.c2f[k]); }

// p_rho_point (small_step.cpp:97-112): calc_p_rho, with smdiv divergence damping when damp.
// The mixed form evaluates it in double (the hydrostatic p'' / al'' relation).
template <class R>
__device__ __forceinline__ void p_rho_point(const Dom<R>& D, int i, int j, int k, bool damp) {
  using A = double;
  const A c1h = D.c1h[k];
  const A m = c1h * A(D.muts(i, j, 0)) + A(D.c2h[k]);
  const A alt = A(D.alt(i, j, k)), mu = A(D.mu2(i, j, 0)), ts = A(D.t_save(i, j, k));
  const A a = -((1. / m) * (alt * (c1h * mu) + A(D.rdnw[k]) * (A(D.ph2(i, j, k + 1)) - A(D.ph2(i, j, k)))));
  D.al(i, j, k) = R(a);
  A pp = A(D.c2a(i, j, k)) * (alt * (A(D.t2(i, j, k)) - c1h * mu * ts) / (m * (k::t0 + ts)) - a);
  if (damp) {
    const A ptmp = pp;
    pp = pp + A(D.smdiv) * (pp - A(D.pm1(i, j, k)));
    D.pm1(i, j, k) = R(ptmp);
  } else {
    D.pm1(i, j, k) = R(pp);
  }
  D.p(i, j, k) = R(pp);
}

// small_step_prep (KPrep :50-93) + calc_p_rho (KPRho :114-119) + calc_coef_w (KCoefW :122-148), per column
template <class R>
__global__ void __launch_bounds__(CX) k_ss_prep(const Dom<R>* __restrict__ doms, BlockMap bm, int rk) {
  const Dom<R>* Dp;
  int i, j, k0;
  if (!thread_index(doms, bm, RG_COLS_STAG, Dp, i, j, k0)) return;
  const Dom<R>& D = *Dp;
  const int nx = D.nx, ny = D.ny, nz = D.nz, nyv = D.nyv;
  const bool first = rk == 1;
  const R mts = D.mub(i, j) + D.mu1(i, j, 0);
  const R mus_u = first ? D.muu(i, j, 0) : R(0.5) * (mts + D.mub(i - 1, j) + D.mu1(i - 1, j, 0));
  const R mus_v = first ? D.muv(i, j, 0) : R(0.5) * (mts + D.mub(i, j - 1) + D.mu1(i, j - 1, 0));
  if (i < nx && j < ny) {
    D.muts(i, j, 0) = mts;
    D.mu_save(i, j, 0) = D.mu2(i, j, 0);
    D.mu2(i, j, 0) = D.mu1(i, j, 0) - D.mu2(i, j, 0);
  }
  if (j < ny) D.muus(i, j, 0) = mus_u;
  if (i < nx && j < nyv) D.muvs(i, j, 0) = mus_v;
  const R mut = (i < nx && j < ny) ? D.mut(i, j, 0) : R(0);
  for (int k = 0; k < nz + 1; ++k) {
    const R c1h = k < nz ? R(D.c1h[k]) : R(0), c2h = k < nz ? R(D.c2h[k]) : R(0);
    if (j < ny && k < nz) {
      const R ui = D.u2(i, j, k);
      D.u_save(i, j, k) = ui;
      D.u2(i, j, k) = ((c1h * mus_u + c2h) * D.u1(i, j, k) - (c1h * D.muu(i, j, 0) + c2h) * ui) / D.msfuy(i, j);
    }
    if (i < nx && j < nyv && k < nz) {
      const R vi = D.v2(i, j, k);
      D.v_save(i, j, k) = vi;
      D.v2(i, j, k) = ((c1h * mus_v + c2h) * D.v1(i, j, k) - (c1h * D.muv(i, j, 0) + c2h) * vi) * D.msfvx_inv(i, j);
    }
    if (i < nx && j < ny) {
      if (k < nz) {
        const R ti = D.t2(i, j, k);
        D.t_save(i, j, k) = ti;
        D.t2(i, j, k) = (c1h * mts + c2h) * D.t1(i, j, k) - (c1h * mut + c2h) * ti;
        D.c2a(i, j, k) = R(k::cpovcv) * (D.pb(i, j, k) + D.p(i, j, k)) / D.alt(i, j, k);
      }
      const R wi = D.w2(i, j, k), phi = D.ph2(i, j, k);
      D.w_save(i, j, k) = wi;
      D.w2(i, j, k) = ((R(D.c1f[k]) * mts + R(D.c2f[k])) * D.w1(i, j, k) - (R(D.c1f[k]) * mut + R(D.c2f[k])) * wi) / D.msfty(i, j);
      D.ph_save(i, j, k) = phi;
      D.ph2(i, j, k) = D.ph1(i, j, k) - phi;
      D.ww1(i, j, k) = (k == 0 || k == nz) ? R(0) : D.ww(i, j, k);
    }
  }
  if (!(i < nx && j < ny)) return;
  for (int k = 0; k < nz; ++k) p_rho_point(D, i, j, k, false);
  // calc_coef_w (the tridiagonal coefficients of advance_w); double in both forms
  {
    using A = double;
    const A dts = D.dt / D.n_sound;
    const A dts_rk = rk == 1 ? D.dt / 3.0 : dts;
    const A cof_h = 0.5 * (rk == 1 ? A(R(dts_rk)) : A(R(dts))) * k::g * (1.0 + A(R(D.epssm)));
    const A cof = A(R(cof_h * cof_h));
    const A lid = D.top_lid ? 0.0 : 1.0;
    const A m = A(mut);
    auto mh = [&](int kk, A mm) { return D.c1h[kk] * mm + D.c2h[kk]; };
    auto mf = [&](int kk, A mm) { return D.c1f[kk] * mm + D.c2f[kk]; };
    auto cq1 = [&](int kk) { return A(R(1) / (R(1) + cqw_(D, i, j, kk))); };
    D.a(i, j, 0) = 0;
    D.alpha(i, j, 0) = 0;
    D.gamma(i, j, 0) = 0;
    D.a(i, j, 1) = 0;
    D.a(i, j, nz) = R(-2. * cof * (D.rdnw[nz - 1] * D.rdnw[nz - 1]) * A(D.c2a(i, j, nz - 1)) * lid / (mh(nz - 1, m) * mf(nz - 1, m)));
    for (int k = 2; k < nz; ++k)
      D.a(i, j, k) = R(-cq1(k) * cof * D.rdn[k] * D.rdnw[k - 1] * A(D.c2a(i, j, k - 1)) / (mh(k - 1, m) * mf(k - 1, m)));
    A gprev = 0;
    for (int k = 1; k < nz; ++k) {
      const A q1 = cq1(k);
      const A b = 1. + q1 * cof * D.rdn[k] *
                           (D.rdnw[k] * A(D.c2a(i, j, k)) / (mh(k, m) * mf(k, m)) +
                            D.rdnw[k - 1] * A(D.c2a(i, j, k - 1)) / (mh(k - 1, m) * mf(k, m)));
      const A cc = -q1 * cof * D.rdn[k] * D.rdnw[k] * A(D.c2a(i, j, k)) / (mh(k, m) * mf(k + 1, m));
      const A al = 1. / (b - A(D.a(i, j, k)) * gprev);
      D.alpha(i, j, k) = R(al);
      gprev = A(R(cc * A(R(al))));
      D.gamma(i, j, k) = R(gprev);
    }
    const A b = 1. + 2. * cof * (D.rdnw[nz - 1] * D.rdnw[nz - 1]) * A(D.c2a(i, j, nz - 1)) / (mh(nz - 1, m) * mf(nz, m));
    D.alpha(i, j, nz) = R(1. / (b - A(D.a(i, j, nz)) * gprev));
    D.gamma(i, j, nz) = 0;
  }
}

// advance_uv (KUV :151-190) over the mass-cell index range (faces i, j of cells i, j)
template <class R, int DI, int DJ>
__device__ __forceinline__ R uv_dpn(const Dom<R>& D, int i, int j, int k) {
  auto ps = [&](int kk) { return D.p(i, j, kk) + D.p(i - DI, j - DJ, kk); };
  const int nz = D.nz;
  if (k == 0) return R(0.5) * (R(D.cf1) * ps(0) + R(D.cf2) * ps(1) + R(D.cf3) * ps(2));
  if (k == nz) return D.top_lid ? R(0.5) * (R(D.cf1) * ps(nz - 1) + R(D.cf2) * ps(nz - 2) + R(D.cf3) * ps(nz - 3)) : R(0);
  return R(0.5) * (R(D.fnm[k]) * ps(k) + R(D.fnp[k]) * ps(k - 1));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R uv_dp(const Dom<R>& D, int i, int j, int k, R mface, R rd, R rm) {
  const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  R d = rm * R(0.5) * rd * (c1h * mface + c2h) *
        (((D.ph2(i, j, k + 1) - D.ph2(i - DI, j - DJ, k + 1)) + (D.ph2(i, j, k) - D.ph2(i - DI, j - DJ, k))) +
         (D.alt(i, j, k) + D.alt(i - DI, j - DJ, k)) * (D.p(i, j, k) - D.p(i - DI, j - DJ, k)) +
         (D.al(i, j, k) + D.al(i - DI, j - DJ, k)) * (D.pb(i, j, k) - D.pb(i - DI, j - DJ, k)));
  d += rm * rd * (D.php(i, j, k) - D.php(i - DI, j - DJ, k)) *
       (R(D.rdnw[k]) * (uv_dpn<R, DI, DJ>(D, i, j, k + 1) - uv_dpn<R, DI, DJ>(D, i, j, k)) -
        R(0.5) * (c1h * D.mu2(i - DI, j - DJ, 0) + c1h * D.mu2(i, j, 0)));
  return d;
}
template <class R>
__global__ void __launch_bounds__(PX) k_uv(const Dom<R>* __restrict__ doms, BlockMap bm, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dts = R(rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound);
  const int ui0 = D.bc_x != CW_BC_PERIODIC ? 1 : 0, ui1 = D.nx;
  const int vj0 = (D.bc_y != CW_BC_PERIODIC && D.do_y) ? 1 : 0, vj1 = D.ny;
  const R emdx = R(D.emdiv) * (R(1.) / R(D.rdx)), emdy = D.do_y ? R(D.emdiv) * (R(1.) / R(D.rdy)) : R(0);
  const R c1h = R(D.c1h[k]);
  if (i >= ui0 && i < ui1 && !edge_uface(D, i, j)) {
    const R mudf_x = -emdx * (D.mudf(i, j, 0) - D.mudf(i - 1, j, 0)) / D.msfuy(i, j);
    D.u2(i, j, k) = D.u2(i, j, k) + dts * D.ru_tend(i, j, k) -
                    dts * cqu_(D, i, j, k) * uv_dp<R, 1, 0>(D, i, j, k, D.muu(i, j, 0), R(D.rdx), D.msfux(i, j) / D.msfuy(i, j)) +
                    c1h * mudf_x;
  }
  if (D.do_y && j >= vj0 && j < vj1 && !edge_vface(D, i, j)) {
    const R mudf_y = -emdy * (D.mudf(i, j, 0) - D.mudf(i, j - 1, 0)) * D.msfvx_inv(i, j);
    D.v2(i, j, k) = D.v2(i, j, k) + dts * D.rv_tend(i, j, k) -
                    dts * cqv_(D, i, j, k) * uv_dp<R, 0, 1>(D, i, j, k, D.muv(i, j, 0), R(D.rdy), D.msfvy(i, j) / D.msfvx(i, j)) +
                    c1h * mudf_y;
  }
}

// KMuTDiv (:194-206): the mass divergence of level k of column (i, j)
template <class R>
__device__ __forceinline__ R mut_dv(const Dom<R>& D, int i, int j, int k) {
  const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  const R fx = (D.u2(i + 1, j, k) + (c1h * D.muu(i + 1, j, 0) + c2h) * D.u_save(i + 1, j, k) / D.msfuy(i + 1, j)) -
               (D.u2(i, j, k) + (c1h * D.muu(i, j, 0) + c2h) * D.u_save(i, j, k) / D.msfuy(i, j));
  R d = R(D.rdx) * fx;
  if (D.do_y)
    d += R(D.rdy) * ((D.v2(i, j + 1, k) + (c1h * D.muv(i, j + 1, 0) + c2h) * D.v_save(i, j + 1, k) * D.msfvx_inv(i, j + 1)) -
                     (D.v2(i, j, k) + (c1h * D.muv(i, j, 0) + c2h) * D.v_save(i, j, k) * D.msfvx_inv(i, j)));
  return D.msftx(i, j) * D.msfty(i, j) * d;
}

// One acoustic substep of a column: advance_mu_t + sumflux (KMuTCol :208-249, KMuTPoint :251-277,
// KSumEdge :281-290) when phase & 1, advance_w (KWRhs / KWExpl / KWSolve :295-408) when phase & 2,
// calc_p_rho with divergence damping (KWPRho :411-416) when phase & 4. The column mass sum, the
// tridiagonal solve and p'' / al'' are evaluated in double in both forms.
template <class R>
__global__ void __launch_bounds__(CX) k_ac(const Dom<R>* __restrict__ doms, BlockMap bm, int rk, int it, int nsteps, int phase) {
  const Dom<R>* Dp;
  int i, j, k0;
  if (!thread_index(doms, bm, RG_COLS_STAG, Dp, i, j, k0)) return;
  const Dom<R>& D = *Dp;
  using A = double;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const R dts = R(rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound);
  const R epssm = R(D.epssm);
  const bool first = it == 1, last = it == nsteps;
  const R rn = R(nsteps);
  const bool mass_col = i < nx && j < ny;
  if (phase & 1) {
    // KSumEdge: east (i = nx) and north (j = ny) faces of specified boundaries
    if (D.spec_x && i == nx && j < ny)
      for (int k = 0; k < nz; ++k) {
        const R su = (first ? R(0) : D.ru_m(i, j, k)) + D.u2(i, j, k);
        const R cpl = (R(D.c1h[k]) * D.muu(i, j, 0) + R(D.c2h[k])) * D.u_save(i, j, k);
        D.ru_m(i, j, k) = last ? su / rn + cpl / D.msfuy(i, j) : su;
      }
    if (D.spec_y && j == ny && i < nx)
      for (int k = 0; k < nz; ++k) {
        const R su = (first ? R(0) : D.rv_m(i, j, k)) + D.v2(i, j, k);
        const R cpl = (R(D.c1h[k]) * D.muv(i, j, 0) + R(D.c2h[k])) * D.v_save(i, j, k);
        D.rv_m(i, j, k) = last ? su / rn + cpl * D.msfvx_inv(i, j) : su;
      }
  }
  if (!mass_col) return;
  const bool spec = edge_mass(D, i, j);
  if (phase & 1) {
    if (spec) {  // spec zone: sumflux of ww only
      for (int k = 0; k <= nz; ++k) {
        const R sw = (first ? R(0) : D.ww_m(i, j, k)) + D.ww(i, j, k);
        D.ww_m(i, j, k) = last ? sw / rn + D.ww1(i, j, k) : sw;
      }
    } else {
      A dmdt = 0;
      for (int k = 0; k < nz; ++k) dmdt += D.dnw[k] * A(mut_dv(D, i, j, k));
      const A mtend = A(D.mu_tend(i, j, 0));
      const A mu_old = A(D.mu2(i, j, 0));
      const A mu_new = mu_old + A(dts) * (dmdt + mtend);
      D.mu2(i, j, 0) = R(mu_new);
      D.mudf(i, j, 0) = R(dmdt + mtend);
      D.muts(i, j, 0) = D.mut(i, j, 0) + R(mu_new);
      D.muave(i, j, 0) = R(0.5) * ((R(1) + epssm) * R(mu_new) + (R(1) - epssm) * R(mu_old));
      A ww_full = 0;
      D.ww(i, j, 0) = 0;
      {
        const R sw = (first ? R(0) : D.ww_m(i, j, 0)) + R(0);
        D.ww_m(i, j, 0) = last ? sw / rn + D.ww1(i, j, 0) : sw;
      }
      const A msfty = A(D.msfty(i, j));
      for (int k = 0; k < nz; ++k) {
        R wpp_hi = 0;
        if (k + 1 < nz) {
          ww_full = ww_full - D.dnw[k] * (D.c1h[k] * dmdt + A(mut_dv(D, i, j, k)) + D.c1h[k] * mtend) / msfty;
          wpp_hi = R(ww_full - A(D.ww1(i, j, k + 1)));
          D.ww(i, j, k + 1) = wpp_hi;
        } else {
          D.ww(i, j, nz) = 0;
        }
        const R sw = (first ? R(0) : D.ww_m(i, j, k + 1)) + wpp_hi;
        D.ww_m(i, j, k + 1) = last ? sw / rn + D.ww1(i, j, k + 1) : sw;
      }
    }
    // KMuTPoint: time sums of ru, rv; theta''
    for (int k = 0; k < nz; ++k) {
      const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
      const R su = (first ? R(0) : D.ru_m(i, j, k)) + D.u2(i, j, k);
      D.ru_m(i, j, k) = last ? su / rn + (c1h * D.muu(i, j, 0) + c2h) * D.u_save(i, j, k) / D.msfuy(i, j) : su;
      if (D.do_y) {
        const R sv = (first ? R(0) : D.rv_m(i, j, k)) + D.v2(i, j, k);
        D.rv_m(i, j, k) = last ? sv / rn + (c1h * D.muv(i, j, 0) + c2h) * D.v_save(i, j, k) * D.msfvx_inv(i, j) : sv;
      }
      const R tk = D.t2(i, j, k);
      D.t_2save(i, j, k) = tk;
      if (spec) continue;
      R hflux = R(0.5) * R(D.rdx) *
                (D.u2(i + 1, j, k) * (D.t_save(i + 1, j, k) + D.t_save(i, j, k)) - D.u2(i, j, k) * (D.t_save(i, j, k) + D.t_save(i - 1, j, k)));
      if (D.do_y)
        hflux += R(0.5) * R(D.rdy) *
                 (D.v2(i, j + 1, k) * (D.t_save(i, j + 1, k) + D.t_save(i, j, k)) - D.v2(i, j, k) * (D.t_save(i, j, k) + D.t_save(i, j - 1, k)));
      const R tn = tk + D.msfty(i, j) * dts * D.t_tend(i, j, k);
      auto wdtn = [&](int kk) -> R {
        if (kk == 0 || kk == nz) return R(0);
        return D.ww(i, j, kk) * (R(D.fnm[kk]) * D.t_save(i, j, kk) + R(D.fnp[kk]) * D.t_save(i, j, kk - 1));
      };
      D.t2(i, j, k) = tn - dts * D.msfty(i, j) * (D.msftx(i, j) * hflux + R(D.rdnw[k]) * (wdtn(k + 1) - wdtn(k)));
    }
  }
  if ((phase & 2) && !spec) {
    const R ope = R(1) + epssm, ome = R(1) - epssm;
    const R mut = D.mut(i, j, 0), muts = D.muts(i, j, 0), mav = D.muave(i, j, 0);
    const R msfty = D.msfty(i, j);
    // KWRhs: R (explicit phi'') at w levels 0..nz, t_2ave at mass levels
    for (int k = 0; k <= nz; ++k) {
      R r;
      if (k == 0 || (D.top_lid && k == nz)) {
        r = 0;
      } else {
        R rr = dts * (D.ph_tend(i, j, k) + R(0.5) * R(k::g) * (R(1) - epssm) * D.w2(i, j, k));
        if (k < nz) {
          auto wdwn = [&](int m) {
            return R(0.5) * (D.ww(i, j, m) + D.ww(i, j, m - 1)) * R(D.rdnw[m - 1]) *
                   (D.ph_save(i, j, m) - D.ph_save(i, j, m - 1) + D.phb(i, j, m) - D.phb(i, j, m - 1));
          };
          rr -= dts * (R(D.fnm[k]) * wdwn(k + 1) + R(D.fnp[k]) * wdwn(k));
        }
        r = D.ph2(i, j, k) + msfty * rr / mf_(D, k, mut);
      }
      D.w_rhs(i, j, k) = r;
      if (k < nz) {
        const R tav = R(0.5) * ((R(1) + epssm) * D.t2(i, j, k) + (R(1) - epssm) * D.t_2save(i, j, k));
        D.t2a(i, j, k) = (tav + R(D.c1h[k]) * mav * R(k::t0)) / (mh_(D, k, muts) * (R(k::t0) + D.t_save(i, j, k)));
      }
    }
    // KWExpl: explicit w'' (the surface from the terrain slope)
    if (!D.flat) {
      R ws = D.msftx(i, j) * R(0.5) * R(D.rdx) *
             ((D.ht(i + 1, j) - D.ht(i, j)) * (R(D.cf1) * D.u2(i + 1, j, 0) + R(D.cf2) * D.u2(i + 1, j, 1) + R(D.cf3) * D.u2(i + 1, j, 2)) +
              (D.ht(i, j) - D.ht(i - 1, j)) * (R(D.cf1) * D.u2(i, j, 0) + R(D.cf2) * D.u2(i, j, 1) + R(D.cf3) * D.u2(i, j, 2)));
      if (D.do_y)
        ws = msfty * R(0.5) * R(D.rdy) *
                 ((D.ht(i, j + 1) - D.ht(i, j)) * (R(D.cf1) * D.v2(i, j + 1, 0) + R(D.cf2) * D.v2(i, j + 1, 1) + R(D.cf3) * D.v2(i, j + 1, 2)) +
                  (D.ht(i, j) - D.ht(i, j - 1)) * (R(D.cf1) * D.v2(i, j, 0) + R(D.cf2) * D.v2(i, j, 1) + R(D.cf3) * D.v2(i, j, 2))) +
             ws;
      D.w2(i, j, 0) = ws;
    } else {
      D.w2(i, j, 0) = 0;
    }
    const R msft_inv = R(1) / msfty;
    for (int k = 1; k <= nz; ++k) {
      const R r_k = D.w_rhs(i, j, k), r_km1 = D.w_rhs(i, j, k - 1), ph_k = D.ph2(i, j, k), ph_km1 = D.ph2(i, j, k - 1);
      if (k < nz) {
        const R r_kp1 = D.w_rhs(i, j, k + 1), ph_kp1 = D.ph2(i, j, k + 1);
        const R cq1 = R(1) / (R(1) + cqw_(D, i, j, k));
        D.w2(i, j, k) = D.w2(i, j, k) + dts * D.rw_tend(i, j, k) +
                        msft_inv * cq1 *
                            (R(0.5) * dts * R(k::g) * R(D.rdn[k]) *
                             (D.c2a(i, j, k) * R(D.rdnw[k]) / mh_(D, k, mut) * (ope * (r_kp1 - r_k) + ome * (ph_kp1 - ph_k)) -
                              D.c2a(i, j, k - 1) * R(D.rdnw[k - 1]) / mh_(D, k - 1, mut) * (ope * (r_k - r_km1) + ome * (ph_k - ph_km1)))) +
                        dts * R(k::g) * msft_inv *
                            (R(D.rdn[k]) * (D.c2a(i, j, k) * D.alt(i, j, k) * D.t2a(i, j, k) - D.c2a(i, j, k - 1) * D.alt(i, j, k - 1) * D.t2a(i, j, k - 1)) -
                             R(D.c1f[k]) * mav);
      } else {
        const int km = nz - 1;
        R wn = D.w2(i, j, k) + dts * D.rw_tend(i, j, k) +
               msft_inv * (-R(0.5) * dts * R(k::g) / mh_(D, km, mut) * (R(D.rdnw[km]) * R(D.rdnw[km])) * R(2) * D.c2a(i, j, km) *
                               (ope * (r_k - r_km1) + ome * (ph_k - ph_km1)) -
                           dts * R(k::g) * (R(2) * R(D.rdnw[km]) * D.c2a(i, j, km) * D.alt(i, j, km) * D.t2a(i, j, km) + R(D.c1f[k]) * mav));
        if (D.top_lid) wn = 0;
        D.w2(i, j, k) = wn;
      }
    }
    // KWSolve: forward and backward sweeps of the tridiagonal system, then phi''
    {
      A wprev = A(D.w2(i, j, 0));
      for (int k = 1; k <= nz; ++k) {
        const A wk = (A(D.w2(i, j, k)) - A(D.a(i, j, k)) * wprev) * A(D.alpha(i, j, k));
        wprev = A(R(wk));
        D.w2(i, j, k) = R(wk);
      }
      A wnext = wprev;
      for (int k = nz - 1; k >= 1; --k) {
        const A wk = A(D.w2(i, j, k)) - A(D.gamma(i, j, k)) * wnext;
        wnext = A(R(wk));
        D.w2(i, j, k) = R(wk);
      }
      for (int k = nz; k >= 1; --k)
        D.ph2(i, j, k) = D.w_rhs(i, j, k) + msfty * R(0.5) * dts * R(k::g) * ope * D.w2(i, j, k) / mf_(D, k, muts);
    }
  }
  if (phase & 4)
    for (int k = 0; k < nz; ++k) p_rho_point(D, i, j, k, true);
}

// KWPRho as a point kernel (runs after the spec-zone update of phi'' when there are lateral boundaries)
template <class R>
__global__ void __launch_bounds__(PX) k_wprho(const Dom<R>* __restrict__ doms, BlockMap bm) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  p_rho_point(*Dp, i, j, k, true);
}

// calc_p_rho_phi, hypsometric_opt 1 (KPRhoPhi :456-477) at (i, j, k); pow = cw_pow
template <class R>
__device__ __forceinline__ void p_rho_phi_point(const Dom<R>& D, int i, int j, int k) {
  const R a = R(-1) / (R(D.c1h[k]) * D.muts(i, j, 0) + R(D.c2h[k])) *
              (D.alb(i, j, k) * (R(D.c1h[k]) * D.mu2(i, j, 0)) + R(D.rdnw[k]) * (D.ph2(i, j, k + 1) - D.ph2(i, j, k)));
  D.al(i, j, k) = a;
  const double base = double(R(k::r_d) * (R(k::t0) + D.t2(i, j, k)) / (R(k::p1000mb) * (a + D.alb(i, j, k))));
  D.p(i, j, k) = R(k::p1000mb * cw_pow(base, k::cpovcv) - double(D.pb(i, j, k)));
}
template <class R>
__global__ void __launch_bounds__(PX) k_p_rho_phi(const Dom<R>* __restrict__ doms, BlockMap bm, int interior) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  if (interior) {  // calc_p_rho_phi_interior (:622-633): spec_zone 1 off each non-periodic side
    const int sz = 1;
    if (D.bc_x != CW_BC_PERIODIC && (i < sz || i >= D.nx - sz)) return;
    if (D.bc_y != CW_BC_PERIODIC && (j < sz || j >= D.ny - sz)) return;
  }
  p_rho_phi_point(D, i, j, k);
}

// small_step_finish (KFinish :419-444, KFinishMu :446-453) + calc_p_rho_phi, per column
template <class R>
__global__ void __launch_bounds__(CX) k_finish(const Dom<R>* __restrict__ doms, BlockMap bm, int rk, int nsmall) {
  const Dom<R>* Dp;
  int i, j, k0;
  if (!thread_index(doms, bm, RG_COLS_STAG, Dp, i, j, k0)) return;
  const Dom<R>& D = *Dp;
  const int nx = D.nx, ny = D.ny, nz = D.nz, nyv = D.nyv;
  const R dts = R(rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound);
  const R hd_dt = (rk == 3 && D.n_moist > 0) ? dts * R(nsmall) : R(0);
  for (int k = 0; k < nz + 1; ++k) {
    if (j < ny && k < nz) {
      const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
      const R mus_u = R(0.5) * (D.muts(i, j, 0) + D.muts(i - 1, j, 0));
      D.u2(i, j, k) = (D.msfuy(i, j) * D.u2(i, j, k) + D.u_save(i, j, k) * (c1h * D.muu(i, j, 0) + c2h)) / (c1h * mus_u + c2h);
    }
    if (i < nx && j < nyv && k < nz) {
      const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
      const R mus_v = R(0.5) * (D.muts(i, j, 0) + D.muts(i, j - 1, 0));
      D.v2(i, j, k) = (D.msfvx(i, j) * D.v2(i, j, k) + D.v_save(i, j, k) * (c1h * D.muv(i, j, 0) + c2h)) / (c1h * mus_v + c2h);
    }
    if (i < nx && j < ny) {
      const R m = D.mut(i, j, 0), mts = D.muts(i, j, 0);
      D.w2(i, j, k) = (D.msfty(i, j) * D.w2(i, j, k) + D.w_save(i, j, k) * (R(D.c1f[k]) * m + R(D.c2f[k]))) / (R(D.c1f[k]) * mts + R(D.c2f[k]));
      D.ph2(i, j, k) = D.ph2(i, j, k) + D.ph_save(i, j, k);
      D.ww(i, j, k) = D.ww(i, j, k) + D.ww1(i, j, k);
      if (k < nz) {
        const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
        D.t2(i, j, k) = (D.t2(i, j, k) - (hd_dt != R(0) ? hd_dt * (c1h * m + c2h) * D.hd(i, j, k) : R(0)) + D.t_save(i, j, k) * (c1h * m + c2h)) /
                        (c1h * mts + c2h);
      }
    }
  }
  if (i < nx && j < ny) D.mu2(i, j, 0) = D.mu2(i, j, 0) + D.mu_save(i, j, 0);
  if (j < ny) D.muus(i, j, 0) = R(0.5) * (D.muts(i, j, 0) + D.muts(i - 1, j, 0));
  if (i < nx && j < nyv) D.muvs(i, j, 0) = R(0.5) * (D.muts(i, j, 0) + D.muts(i, j - 1, 0));
  if (i < nx && j < ny)
    for (int k = 0; k < nz; ++k) p_rho_phi_point(D, i, j, k);
}

// ------------------------------------------------------------------ scalars
// ScalarTransport (src/dyn/scalars.cpp:42-292): q_2 advected with the time-averaged mass fluxes ru_m,
// rv_m, ww_m from q_1, species n of the tables; pd = advect_scalar_pd's statement functions.
template <class R>
__device__ __forceinline__ bool q_is_pd(const Dom<R>& D, int n, int rk) {
  return rk == 3 && (n < D.n_moist ? D.moist_adv_opt : D.scalar_adv_opt) == 1;
}
template <class R>
__device__ __forceinline__ bool spec_cell(const Dom<R>& D, int i, int j) {
  return (D.spec_x && (i == 0 || i == D.nx - 1)) || (D.spec_y && (j == 0 || j == D.ny - 1));
}
template <class R>
__device__ __forceinline__ R m_full(const Dom<R>& D, int k, R mub, R mu) { return R(D.c1h[k]) * (mub + mu) + R(D.c2h[k]); }

// rk 1: q_tendf = 0 + constant-K diffusion (DiffusionDriver::scalar, diffusion_driver.cpp:293-322)
template <class R>
__global__ void __launch_bounds__(PX) k_q_tendf_rk1(const Dom<R>* __restrict__ doms, BlockMap bm) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const bool sp = D.lbc, px = D.bc_x == CW_BC_PERIODIC;
  int is = sp ? 1 : 0, ie = sp ? D.nx - 1 : D.nx;
  const int js = sp ? 1 : 0, je = sp ? D.ny - 1 : D.ny;
  if (px) { is = 0; ie = D.nx; }
  const R khh = R(D.khdif / D.prandtl), kvdq = R(D.kvdif / D.prandtl);
  for (int n = 0; n < D.n_scalars; ++n) {
    R t = 0;
    if (D.diff_on) {
      if (i >= is && i < ie && j >= js && j < je) t += hdiff_m(D, D.q2[n], (const VB<R>*)nullptr, D.muts, khh, i, j, k);
      const bool qv = n == 0 && D.n_moist > 0;
      t += vdiff_m(D, D.q2[n], qv ? &D.qv_base : (const VB<R>*)nullptr, D.muts, kvdq, i, j, k);
    }
    D.qtf[n](i, j, k) = t;
  }
}

// advect_scalar (Fluxes::adv :126-139) of species n at a cell
template <class R>
__device__ R q_adv(const Dom<R>& D, const V3<R>& q, int i, int j, int k) {
  if (spec_cell(D, i, j)) return 0;
  R r = -(D.msftx(i, j) * R(D.rdx)) * (sc_fx(D, q, D.ru_m, i + 1, j, k, false) - sc_fx(D, q, D.ru_m, i, j, k, false));
  if (D.do_y) r -= (D.msftx(i, j) * R(D.rdy)) * (sc_fy(D, q, D.rv_m, i, j + 1, k, false) - sc_fy(D, q, D.rv_m, i, j, k, false));
  return r - R(D.rdnw[k]) * (sc_fz(D, q, D.ww_m, i, j, k + 1, false) - sc_fz(D, q, D.ww_m, i, j, k, false));
}
// KUpdate (:145-156) for the non-PD species of this stage
template <class R>
__global__ void __launch_bounds__(PX) k_q_update(const Dom<R>* __restrict__ doms, BlockMap bm, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt_rk = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const R mub = D.mub(i, j), mu1 = D.mu1(i, j, 0), mu2 = D.mu2(i, j, 0);
  for (int n = 0; n < D.n_scalars; ++n) {
    if (q_is_pd(D, n, rk)) continue;
    R tend = q_adv(D, D.q2[n], i, j, k) * D.msfty(i, j);
    tend += D.qtf[n](i, j, k);
    D.qn[n](i, j, k) = (m_full(D, k, mub, mu1) * D.q1[n](i, j, k) + dt_rk * tend) / m_full(D, k, mub, mu2);
  }
}
// KPreUpdatePD (:174-180)
template <class R>
__global__ void __launch_bounds__(PX) k_q_pre_pd(const Dom<R>* __restrict__ doms, BlockMap bm, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt_rk = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const R m = m_full(D, k, D.mub(i, j), D.mu1(i, j, 0));
  for (int n = 0; n < D.n_scalars; ++n) {
    if (!q_is_pd(D, n, rk)) continue;
    D.q1[n](i, j, k) = (m * D.q1[n](i, j, k) + dt_rk * D.qtf[n](i, j, k)) / m;
  }
}
// advect_scalar_pd face fluxes: lo = first-order upwind (fxl/fyl/fzl :81-99), dh = high-order - lo
template <class R>
__device__ __forceinline__ R pd_mh(const Dom<R>& D, int i, int j, int k) { return R(D.c1h[k]) * D.muts(i, j, 0) + R(D.c2h[k]); }
template <class R>
__device__ void pd_fx(const Dom<R>& D, const V3<R>& q, const V3<R>& qo, R dt, int i, int j, int k, R& dh, R& lo) {
  const R dx = R(2) / (D.msfty(i, j) + D.msfty(i - 1, j)) / R(D.rdx), mu = R(0.5) * (pd_mh(D, i, j, k) + pd_mh(D, i - 1, j, k)),
          vel = D.ru_m(i, j, k);
  const R cr = (D.spec_x && i == 1) ? (vel / mu) * dt / dx : vel * dt / dx / mu;
  lo = mu * (dx / dt) * flux_upwind(qo(i - 1, j, k), qo(i, j, k), cr);
  dh = sc_fx(D, q, D.ru_m, i, j, k, true) - lo;
}
template <class R>
__device__ void pd_fy(const Dom<R>& D, const V3<R>& q, const V3<R>& qo, R dt, int i, int j, int k, R& dh, R& lo) {
  const R dy = R(2) / (D.msftx(i, j) + D.msftx(i, j - 1)) / R(D.rdy), mu = R(0.5) * (pd_mh(D, i, j, k) + pd_mh(D, i, j - 1, k)),
          vel = D.rv_m(i, j, k);
  const R cr = vel * dt / dy / mu;
  lo = mu * (dy / dt) * flux_upwind(qo(i, j - 1, k), qo(i, j, k), cr);
  dh = sc_fy(D, q, D.rv_m, i, j, k, true) - lo;
}
template <class R>
__device__ void pd_fz(const Dom<R>& D, const V3<R>& q, const V3<R>& qo, R dt, int i, int j, int k, R& dh, R& lo) {
  if (k == 0 || k == D.nz) {
    lo = 0;
    dh = R(0) - R(0);
    return;
  }
  const R dz = R(2) / (R(D.rdnw[k]) + R(D.rdnw[k - 1])), mu = pd_mh(D, i, j, k), vel = D.ww_m(i, j, k);
  const R cr = vel * dt / dz / mu;
  lo = mu * (dz / dt) * flux_upwind(qo(i, j, k - 1), qo(i, j, k), cr);
  dh = sc_fz(D, q, D.ww_m, i, j, k, true) - lo;
}
// KScalePD (:215-241)
template <class R>
__global__ void __launch_bounds__(PX) k_q_scale_pd(const Dom<R>* __restrict__ doms, BlockMap bm, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const bool edge = (D.spec_x && (i == 0 || i == D.nx - 1)) || (D.spec_y && (j == 0 || j == D.ny - 1));
  for (int n = 0; n < D.n_scalars; ++n) {
    if (!q_is_pd(D, n, rk)) continue;
    if (edge) {
      D.qscale[n](i, j, k) = 1;
      continue;
    }
    const V3<R>& q = D.q2[n];
    const V3<R>& qo = D.q1[n];
    R dhx0, lox0, dhx1, lox1, dhy0 = 0, loy0 = 0, dhy1 = 0, loy1 = 0, dhz0, loz0, dhz1, loz1;
    pd_fx(D, q, qo, dt, i, j, k, dhx0, lox0);
    pd_fx(D, q, qo, dt, i + 1, j, k, dhx1, lox1);
    if (D.do_y) {
      pd_fy(D, q, qo, dt, i, j, k, dhy0, loy0);
      pd_fy(D, q, qo, dt, i, j + 1, k, dhy1, loy1);
    }
    pd_fz(D, q, qo, dt, i, j, k, dhz0, loz0);
    pd_fz(D, q, qo, dt, i, j, k + 1, dhz1, loz1);
    const R mxy = D.msftx(i, j) * D.msfty(i, j);
    R hlow = R(D.rdx) * (lox1 - lox0);
    if (D.do_y) hlow += R(D.rdy) * (loy1 - loy0);
    const R ph_low = ((R(D.c1h[k]) * D.mub(i, j) + R(D.c2h[k])) + R(D.c1h[k]) * D.mu1(i, j, 0)) * qo(i, j, k) -
                     dt * (mxy * hlow + D.msfty(i, j) * R(D.rdnw[k]) * (loz1 - loz0));
    R hout = R(D.rdx) * ((dhx1 > 0 ? dhx1 : R(0)) - (dhx0 < 0 ? dhx0 : R(0)));
    if (D.do_y) hout += R(D.rdy) * ((dhy1 > 0 ? dhy1 : R(0)) - (dhy0 < 0 ? dhy0 : R(0)));
    const R out = mxy * hout + D.msfty(i, j) * R(D.rdnw[k]) * ((dhz1 < 0 ? dhz1 : R(0)) - (dhz0 > 0 ? dhz0 : R(0)));
    const R flux_out = dt * out;
    R s = 1;
    if (flux_out > ph_low) {
      s = ph_low / (flux_out + R(1e-20));
      if (s < 0) s = 0;
    }
    D.qscale[n](i, j, k) = s;
  }
}
// KUpdatePD (:244-291)
template <class R>
__global__ void __launch_bounds__(PX) k_q_update_pd(const Dom<R>* __restrict__ doms, BlockMap bm, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index(doms, bm, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const R mub = D.mub(i, j), mu1 = D.mu1(i, j, 0), mu2 = D.mu2(i, j, 0);
  for (int n = 0; n < D.n_scalars; ++n) {
    if (!q_is_pd(D, n, rk)) continue;
    const V3<R>& q = D.q2[n];
    const V3<R>& qo = D.q1[n];
    const V3<R>& sc = D.qscale[n];
    if (spec_cell(D, i, j)) {
      D.qn[n](i, j, k) = m_full(D, k, mub, mu1) * qo(i, j, k) / m_full(D, k, mub, mu2);
      continue;
    }
    R dhx0, lox0, dhx1, lox1, dhy0 = 0, loy0 = 0, dhy1 = 0, loy1 = 0, dhz0, loz0, dhz1, loz1;
    pd_fx(D, q, qo, dt, i, j, k, dhx0, lox0);
    pd_fx(D, q, qo, dt, i + 1, j, k, dhx1, lox1);
    if (D.do_y) {
      pd_fy(D, q, qo, dt, i, j, k, dhy0, loy0);
      pd_fy(D, q, qo, dt, i, j + 1, k, dhy1, loy1);
    }
    pd_fz(D, q, qo, dt, i, j, k, dhz0, loz0);
    pd_fz(D, q, qo, dt, i, j, k + 1, dhz1, loz1);
    auto lim = [](R d, R s_up, R s_dn) { return d * (d > 0 ? s_up : (d < 0 ? s_dn : R(1))); };
    const R dx0 = lim(dhx0, sc(i - 1, j, k), sc(i, j, k)), dx1 = lim(dhx1, sc(i, j, k), sc(i + 1, j, k));
    const R dz0 = (k == 0) ? R(0) : lim(dhz0, sc(i, j, k), sc(i, j, k - 1));
    const R dz1 = (k + 1 == D.nz) ? R(0) : lim(dhz1, sc(i, j, k + 1), sc(i, j, k));
    R tend = -R(D.rdnw[k]) * (dz1 - dz0 + loz1 - loz0);
    tend -= D.msftx(i, j) * (R(D.rdx) * (dx1 - dx0 + lox1 - lox0));
    if (D.do_y) {
      const R dy0 = lim(dhy0, sc(i, j - 1, k), sc(i, j, k)), dy1 = lim(dhy1, sc(i, j, k), sc(i, j + 1, k));
      tend -= D.msftx(i, j) * (R(D.rdy) * (dy1 - dy0 + loy1 - loy0));
    }
    D.qn[n](i, j, k) = (m_full(D, k, mub, mu1) * qo(i, j, k) + dt * (tend * D.msfty(i, j))) / m_full(D, k, mub, mu2);
  }
}
// swap(q_2, q_new) of every species (ScalarTransport::update :425)
template <class R>
__global__ void k_q_swap(Dom<R>* doms, int nmembers) {
  const int m = blockIdx.x;
  if (m >= nmembers) return;
  Dom<R>& D = doms[m];
  for (int n = threadIdx.x; n < D.n_scalars; n += blockDim.x) {
    const V3<R> t = D.q2[n];
    D.q2[n] = D.qn[n];
    D.qn[n] = t;
  }
}

// set_w_surface (KSetWSurface, rk3.cpp:173-200), fill = false
template <class R>
__global__ void __launch_bounds__(CX) k_w_surface(const Dom<R>* __restrict__ doms, BlockMap bm) {
  const Dom<R>* Dp;
  int i, j, k0;
  if (!thread_index(doms, bm, RG_COLS_MASS, Dp, i, j, k0)) return;
  const Dom<R>& D = *Dp;
  const R cf1 = R(D.cf1), cf2 = R(D.cf2), cf3 = R(D.cf3);
  const R ws = D.msfty(i, j) * R(0.5) * R(D.rdy) *
                   ((D.ht(i, j + 1) - D.ht(i, j)) * (cf1 * D.v2(i, j + 1, 0) + cf2 * D.v2(i, j + 1, 1) + cf3 * D.v2(i, j + 1, 2)) +
                    (D.ht(i, j) - D.ht(i, j - 1)) * (cf1 * D.v2(i, j, 0) + cf2 * D.v2(i, j, 1) + cf3 * D.v2(i, j, 2))) +
               D.msftx(i, j) * R(0.5) * R(D.rdx) *
                   ((D.ht(i + 1, j) - D.ht(i, j)) * (cf1 * D.u2(i + 1, j, 0) + cf2 * D.u2(i + 1, j, 1) + cf3 * D.u2(i + 1, j, 2)) +
                    (D.ht(i, j) - D.ht(i - 1, j)) * (cf1 * D.u2(i, j, 0) + cf2 * D.u2(i, j, 1) + cf3 * D.u2(i, j, 2)));
  D.w2(i, j, 0) = ws;
}

}  // namespace cw
