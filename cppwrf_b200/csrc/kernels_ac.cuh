// SPDX-License-Identifier: GPL-3.0-or-later
// Acoustic small step, small_step_finish + calc_p_rho_phi, scalar transport, set_w_surface (see
// kernels.cuh for the conventions). Reference: src/dyn/small_step.cpp, scalars.cpp, rk3.cpp of CPPWRF.
#pragma once

#include "kernels.cuh"

namespace cw {

// Edge (small_step.cpp:36-45): the spec zone of specified boundaries (open boundaries have none: every cell is
// advanced)
template <class R>
__device__ __forceinline__ bool edge_mass(const Dom<R>& D, int i, int j) {
  return (D.sx && (i == 0 || i == D.nx - 1)) || (D.sy && (j == 0 || j == D.ny - 1));
}
template <class R>
__device__ __forceinline__ bool edge_uface(const Dom<R>& D, int i, int j) {
  return (D.sx && (i <= 0 || i >= D.nx)) || (D.sy && (j == 0 || j == D.ny - 1));
}
template <class R>
__device__ __forceinline__ bool edge_vface(const Dom<R>& D, int i, int j) {
  return (D.sx && (i == 0 || i == D.nx - 1)) || (D.sy && (j <= 0 || j >= D.ny));
}
template <class R>
__device__ __forceinline__ R mh_(const Dom<R>& D, int k, R m) { return R(D.c1h[k]) * m + R(D.c2h[k]); }
template <class R>
__device__ __forceinline__ R mf_(const Dom<R>& D, int k, R m) { return R(D.c1f[k]) * m + R(D.c2f[k]); }

// p_rho_point (small_step.cpp:97-112): calc_p_rho, with smdiv divergence damping when damp.
// The mixed form evaluates it in double (the hydrostatic p'' / al'' relation).
// RO: alt, t_save and c2a are read-only in the calling kernel (the read-only load path). ph_k, ph_kp: the
// values of phi'' at levels k and k + 1.
template <bool RO, class R>
__device__ __forceinline__ void p_rho_point_ph(const Dom<R>& D, int i, int j, int k, bool damp, R ph_k_in, R ph_kp_in) {
  using A = double;
  // every load before the first store
  const A c1h = D.c1h[k];
  const A muts = A(D.muts(i, j, 0)), alt = A(RO ? D.alt.ld(i, j, k) : D.alt(i, j, k)), mu = A(D.mu2(i, j, 0));
  const A ts = A(RO ? D.t_save.ld(i, j, k) : D.t_save(i, j, k));
  const A ph_kp = A(ph_kp_in), ph_k = A(ph_k_in), t2 = A(D.t2(i, j, k));
  const A c2a = A(RO ? D.c2a.ld(i, j, k) : D.c2a(i, j, k));
  const A pm1 = damp ? A(D.pm1(i, j, k)) : A(0);
  const A m = c1h * muts + A(D.c2h[k]);
  const A a = -((1. / m) * (alt * (c1h * mu) + A(D.rdnw[k]) * (ph_kp - ph_k)));
  A pp = c2a * (alt * (t2 - c1h * mu * ts) / (m * (k::t0 + ts)) - a);
  D.al(i, j, k) = R(a);
  if (damp) {
    const A ptmp = pp;
    pp = pp + A(D.smdiv) * (pp - pm1);
    D.pm1(i, j, k) = R(ptmp);
  } else {
    D.pm1(i, j, k) = R(pp);
  }
  D.p(i, j, k) = R(pp);
}
template <bool RO, class R>
__device__ __forceinline__ void p_rho_point(const Dom<R>& D, int i, int j, int k, bool damp) {
  p_rho_point_ph<RO>(D, i, j, k, damp, D.ph2(i, j, k), D.ph2(i, j, k + 1));
}

// advance_uv (KUV :151-190): the faces i, j of cells i, j
template <class R, int DI, int DJ>
__device__ __forceinline__ R uv_dpn(const Dom<R>& D, int i, int j, int k) {
  auto ps = [&](int kk) { return D.p.ld(i, j, kk) + D.p.ld(i - DI, j - DJ, kk); };
  const int nz = D.nz;
  if (k == 0) return R(0.5) * (R(D.cf1) * ps(0) + R(D.cf2) * ps(1) + R(D.cf3) * ps(2));
  if (k == nz) return D.top_lid ? R(0.5) * (R(D.cf1) * ps(nz - 1) + R(D.cf2) * ps(nz - 2) + R(D.cf3) * ps(nz - 3)) : R(0);
  return R(0.5) * (R(D.fnm[k]) * ps(k) + R(D.fnp[k]) * ps(k - 1));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R uv_dp(const Dom<R>& D, int i, int j, int k, R mface, R rd, R rm) {
  const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  R d = rm * R(0.5) * rd * (c1h * mface + c2h) *
        (((D.ph2.ld(i, j, k + 1) - D.ph2.ld(i - DI, j - DJ, k + 1)) + (D.ph2.ld(i, j, k) - D.ph2.ld(i - DI, j - DJ, k))) +
         (D.alt.ld(i, j, k) + D.alt.ld(i - DI, j - DJ, k)) * (D.p.ld(i, j, k) - D.p.ld(i - DI, j - DJ, k)) +
         (D.al.ld(i, j, k) + D.al.ld(i - DI, j - DJ, k)) * (D.pb(i, j, k) - D.pb(i - DI, j - DJ, k)));
  d += rm * rd * (D.php.ld(i, j, k) - D.php.ld(i - DI, j - DJ, k)) *
       (R(D.rdnw[k]) * (uv_dpn<R, DI, DJ>(D, i, j, k + 1) - uv_dpn<R, DI, DJ>(D, i, j, k)) -
        R(0.5) * (c1h * D.mu2.ld(i - DI, j - DJ, 0) + c1h * D.mu2.ld(i, j, 0)));
  return d;
}
// over the staggered index range; with lateral boundaries the spec zone's faces take
// u += dts ru_tend (LateralBC::update_uv, lateral_bc.cpp:353-361) instead, and so do the faces of open boundaries
// (no pressure gradient or divergence damping on them, :175-184)
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX, 10) k_uv(const __grid_constant__ Pack<R, NM> P, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_STAG, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  if (k >= D.nz) return;
  const R dts = R(rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound);
  // both new values are computed before either store (the stores cannot alias the loads then)
  bool su = false, sv = false;
  R un = 0, vn = 0;
  if (D.lbc) {
    int sl, pos;
    if (spec_at(ring_for(D.nx, D.ny, 'u'), i, j, sl, pos)) {
      un = D.u2(i, j, k) + dts * D.ru_tend.ld(i, j, k);
      su = true;
    }
    if (spec_at(ring_for(D.nx, D.ny, 'v'), i, j, sl, pos)) {
      vn = D.v2(i, j, k) + dts * D.rv_tend.ld(i, j, k);
      sv = true;
    }
  }
  if (D.open_x && (i == 0 || i == D.nx) && j < D.ny) {
    un = D.u2(i, j, k) + dts * D.ru_tend.ld(i, j, k);
    su = true;
  }
  if (D.do_y && D.open_y && (j == 0 || j == D.ny) && i < D.nx) {
    vn = D.v2(i, j, k) + dts * D.rv_tend.ld(i, j, k);
    sv = true;
  }
  if (i < D.nx && j < D.ny) {
    const int ui0 = D.bc_x != CW_BC_PERIODIC ? 1 : 0, ui1 = D.nx;
    const int vj0 = (D.bc_y != CW_BC_PERIODIC && D.do_y) ? 1 : 0, vj1 = D.ny;
    const R emdx = R(D.emdiv) * (R(1.) / R(D.rdx)), emdy = D.do_y ? R(D.emdiv) * (R(1.) / R(D.rdy)) : R(0);
    const R c1h = R(D.c1h[k]);
    if (i >= ui0 && i < ui1 && !edge_uface(D, i, j)) {
      const R mudf_x = div_msf(-emdx * (D.mudf.ld(i, j, 0) - D.mudf.ld(i - 1, j, 0)), D.msfuy(i, j));
      un = D.u2(i, j, k) + dts * D.ru_tend.ld(i, j, k) -
           dts * cqu_(D, i, j, k) * uv_dp<R, 1, 0>(D, i, j, k, D.muu.ld(i, j, 0), R(D.rdx), div_msf(D.msfux(i, j), D.msfuy(i, j))) +
           c1h * mudf_x;
      su = true;
    }
    if (D.do_y && j >= vj0 && j < vj1 && !edge_vface(D, i, j)) {
      const R mudf_y = -emdy * (D.mudf.ld(i, j, 0) - D.mudf.ld(i, j - 1, 0)) * D.msfvx_inv(i, j);
      vn = D.v2(i, j, k) + dts * D.rv_tend.ld(i, j, k) -
           dts * cqv_(D, i, j, k) * uv_dp<R, 0, 1>(D, i, j, k, D.muv.ld(i, j, 0), R(D.rdy), div_msf(D.msfvy(i, j), D.msfvx(i, j))) +
           c1h * mudf_y;
      sv = true;
    }
  }
  if (su) D.u2(i, j, k) = un;
  if (sv) D.v2(i, j, k) = vn;
}

// calc_p_rho_phi (KPRhoPhi :456-477) at (i, j, k); pow and log in double: cw_pow / cw_log in the FP64 form
// (bit-identical with the oracle), CUDA's in the mixed form
template <class R>
__device__ __forceinline__ double eos_pow(double base) {
  if constexpr (sizeof(R) == 4) return ::pow(base, k::cpovcv);
  else return cw_pow(base, k::cpovcv);
}
template <class R>
__device__ __forceinline__ double hypso_log(double x) {
  if constexpr (sizeof(R) == 4) return ::log(x);
  else return cw_log(x);
}
template <class R>
__device__ __forceinline__ void p_rho_phi_point(const Dom<R>& D, int i, int j, int k) {
  R a;
  if (D.hypsometric_opt == 2) {
    // log-linear in pressure: the total inverse density of the layer is its geopotential thickness over
    // p_mid log(p_bottom / p_top), the dry pressures from the hybrid coefficients; in double in both forms (the
    // perturbation is a small difference of totals)
    const double m = double(D.muts(i, j, 0)), ptop = D.p_top;
    const double pfu = D.c3f[k + 1] * m + D.c4f[k + 1] + ptop, pfd = D.c3f[k] * m + D.c4f[k] + ptop;
    const double phm = D.c3h[k] * m + D.c4h[k] + ptop;
    a = R((double(D.ph2(i, j, k + 1)) - double(D.ph2(i, j, k)) + D.phb64(i, j, k + 1) - D.phb64(i, j, k)) /
              phm / hypso_log<R>(pfd / pfu) -
          D.alb64(i, j, k));
  } else {
    a = R(-1) / (R(D.c1h[k]) * D.muts(i, j, 0) + R(D.c2h[k])) *
        (D.alb(i, j, k) * (R(D.c1h[k]) * D.mu2(i, j, 0)) + R(D.rdnw[k]) * (D.ph2(i, j, k + 1) - D.ph2(i, j, k)));
  }
  D.al(i, j, k) = a;
  // the equation of state in double in both forms: p'' is a small difference of totals of ~1e5 Pa (in float the
  // rounding of the total's base, 6e-8, would be ~1e-4 of p'') -- for the FP64 form the same operations
  const double base = k::r_d * (k::t0 + double(D.t2(i, j, k))) / (k::p1000mb * (double(a) + D.alb64(i, j, k)));
  D.p(i, j, k) = R(k::p1000mb * eos_pow<R>(base) - D.pb64(i, j, k));
}
// mode 0: every mass point; 1: calc_p_rho_phi_interior (after spec_bdy_final); 2: after the microphysics, only in
// the members that have it, on the interior where the member has boundary data (rk3.cpp:146-158)
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX) k_p_rho_phi(const __grid_constant__ Pack<R, NM> P, int mode) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  if (mode == 2 && D.mp_physics == 0) return;
  if (mode == 1 && !D.lbc) return;  // calc_p_rho_phi_interior follows spec_bdy_final: members with boundary data only
  if (mode == 1 || (mode == 2 && D.lbc)) {  // calc_p_rho_phi_interior (:622-633): spec_zone 1 off each non-periodic side
    const int sz = 1;
    if (D.bc_x != CW_BC_PERIODIC && (i < sz || i >= D.nx - sz)) return;
    if (D.bc_y != CW_BC_PERIODIC && (j < sz || j >= D.ny - sz)) return;
  }
  p_rho_phi_point(D, i, j, k);
}

// ------------------------------------------------------------------ scalars
// ScalarTransport (src/dyn/scalars.cpp:42-292): q_2 advected with the time-averaged mass fluxes ru_m,
// rv_m, ww_m from q_1, species n of the tables; pd = advect_scalar_pd's statement functions. The species
// are independent: the scalar kernels run one thread per (cell, species), blockIdx.y the species.
template <class R>
__device__ __forceinline__ bool q_is_pd(const Dom<R>& D, int n, int rk) {
  return rk == 3 && (n < D.n_moist ? D.moist_adv_opt : D.scalar_adv_opt) == 1;
}
template <class R>
__device__ __forceinline__ bool spec_cell(const Dom<R>& D, int i, int j) {
  return (D.sx && (i == 0 || i == D.nx - 1)) || (D.sy && (j == 0 || j == D.ny - 1));
}
template <class R>
__device__ __forceinline__ R m_full(const Dom<R>& D, int k, R mub, R mu) { return R(D.c1h[k]) * (mub + mu) + R(D.c2h[k]); }

// rk 1: q_tendf = 0 + constant-K diffusion (DiffusionDriver::scalar, diffusion_driver.cpp:293-322); for the
// species with boundary data the relaxation of rows 1..3 (relax_scalars, lateral_bc.cpp:388-401) and the
// spec zone's boundary tendency (spec_scalars, :403-414; the held tendency is not changed after rk 1, so
// writing it once per step is the same as the reference's once per stage)
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX) k_q_tendf_rk1(const __grid_constant__ Pack<R, NM> P) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const bool sp = D.lbc, px = D.bc_x == CW_BC_PERIODIC, bx = sp || D.open_x, by = sp || D.open_y;
  int is = bx ? 1 : 0, ie = bx ? D.nx - 1 : D.nx;
  const int js = by ? 1 : 0, je = by ? D.ny - 1 : D.ny;
  if (px) { is = 0; ie = D.nx; }
  const R khh = R(D.khdif / D.prandtl), kvdq = R(D.kvdif / D.prandtl);
  const Ring rq = ring_for(D.nx, D.ny, 'q');
  const int n = blockIdx.y;  // the species
  if (n >= D.n_scalars) return;
  R t = 0;
  if (D.diff_on) {
    if (i >= is && i < ie && j >= js && j < je) {
      if (D.xk_field) t += hdiff_m(D, D.q2[n], (const VB<R>*)nullptr, D.muts, XkField<R>{D.xkhh}, i, j, k);
      else t += hdiff_m(D, D.q2[n], (const VB<R>*)nullptr, D.muts, XkConst<R>{khh}, i, j, k);
    }
    const bool qv = n == 0 && D.n_moist > 0;
    t += vdiff_m(D, D.q2[n], qv ? &D.qv_base : (const VB<R>*)nullptr, D.muts, kvdq, i, j, k);
  }
  if (D.diff_6th_opt != 0 && D.diff_6th_factor != 0.0 && d6_in('m', D.nx, D.ny, sp, px, D.open_x, D.open_y, i, j)) {
    R tx, ty;  // DiffusionDriver::scalar (diffusion_driver.cpp:323-326): muts and the stage's dt / 3
    d6_tend(D, 'm', D.q2[n], D.muts, D.c1h, D.c2h, d6_coef(D, R(D.dt / 3.0)), i, j, k, tx, ty);
    t = t + tx + ty;
  }
  if (sp && D.lbc_q[n].have) {
    R fa, fb;
    int sl, pos;
    if (spec_at(rq, i, j, sl, pos)) t = slab_at(D.lbc_q[n], 1, sl, pos, k, 0);
    else if (relax_at<R, false>(D, D.q2[n], D.c1h, D.c2h, D.lbc_q[n], rq, i, j, k, fa, fb)) t = t + fa - fb;
  }
  D.qtf[n](i, j, k) = t;
}

// advect_scalar (Fluxes::adv :126-139) of species n at a cell outside the spec zone, from its horizontal face
// fluxes: the horizontal part (the vertical flux divergence follows in q_adv)
template <class R>
__device__ R q_adv_h(const Dom<R>& D, const V3<R>& q, int i, int j, int k, R fx0, R fx1, R fy0, R fy1) {
  R r;
  const bool ocol = D.open_x && (i == 0 || i == D.nx - 1), orow = D.open_y && (j == 0 || j == D.ny - 1);
  if (ocol || orow) {  // open boundary (:129-134): y flux, x flux, open x, open y (field_old = the scalar), vertical
    r = R(0);
    if (D.do_y && !orow) r = r - (D.msftx(i, j) * R(D.rdy)) * (fy1 - fy0);
    if (!ocol) r = r - (D.msftx(i, j) * R(D.rdx)) * (fx1 - fx0);
    if (ocol) r = r - open_scalar<R, 1>(D, q, q, D.ru_m, i, j, k);
    if (orow) r = r - open_scalar<R, 0>(D, q, q, D.rv_m, i, j, k);
  } else {
    r = -(D.msftx(i, j) * R(D.rdx)) * (fx1 - fx0);
    if (D.do_y) r -= (D.msftx(i, j) * R(D.rdy)) * (fy1 - fy0);
  }
  return r;
}
template <class R>
__device__ R q_adv(const Dom<R>& D, const V3<R>& q, int i, int j, int k, R fx0, R fx1, R fy0, R fy1) {
  if (spec_cell(D, i, j)) return 0;
  const R r = q_adv_h(D, q, i, j, k, fx0, fx1, fy0, fy1);
  return r - R(D.rdnw[k]) * (sc_fz(D, q, D.ww_m, i, j, k + 1, false) - sc_fz(D, q, D.ww_m, i, j, k, false));
}
// KUpdate (:145-156) for the non-PD species of this stage, every species of the point in one thread (the mass
// fluxes, column masses and map factors loaded once for all of them); the horizontal face fluxes of the block's tile
// once per species, in shared memory
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX, 12) k_q_update(const __grid_constant__ Pack<R, NM> P, int rk) {
  constexpr int SX = shape_x(SH), SY = shape_y(SH);
  __shared__ R sfx[SY][SX + 1];
  __shared__ R sfy[SY + 1][SX];
  const Dom<R>* Dp;
  int i, j, k;
  Range r;
  const bool in = thread_index<SH>(P, RG_MASS, Dp, i, j, k, r);
  const Dom<R>& D = *Dp;
  const int tx = int(threadIdx.x) % SX, ty = int(threadIdx.x) / SX;
  const int nx = D.nx, ny = D.ny;
  // the faces of the member's cells (up to the face after its last one), in its rows / columns
  const bool rx = j < r.j1 && j < ny, ry = i < r.i1 && i < nx;
  const bool fx0 = rx && i <= nx && i <= r.i1, fx1 = tx == SX - 1 && rx && i + 1 <= nx && i + 1 <= r.i1;
  const bool fy0 = D.do_y && ry && j <= ny && j <= r.j1, fy1 = D.do_y && ty == SY - 1 && ry && j + 1 <= ny && j + 1 <= r.j1;
  const R dt_rk = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  R mub = 0, mu1 = 0, mu2 = 0, msfty = 0;
  if (in) {
    mub = D.mub(i, j);
    mu1 = D.mu1.ld(i, j, 0);
    mu2 = D.mu2.ld(i, j, 0);
    msfty = D.msfty(i, j);
  }
  for (int n = 0; n < D.n_scalars; ++n) {  // uniform over the block
    if (q_is_pd(D, n, rk)) continue;
    const V3<R> q = D.q2[n];
    if (fx0) sfx[ty][tx] = sc_fx(D, q, D.ru_m, i, j, k, false);
    if (fx1) sfx[ty][SX] = sc_fx(D, q, D.ru_m, i + 1, j, k, false);
    if (fy0) sfy[ty][tx] = sc_fy(D, q, D.rv_m, i, j, k, false);
    if (fy1) sfy[SY][tx] = sc_fy(D, q, D.rv_m, i, j + 1, k, false);
    __syncthreads();
    if (in) {
      R tend = q_adv(D, q, i, j, k, sfx[ty][tx], sfx[ty][tx + 1], sfy[ty][tx], sfy[ty + 1][tx]) * msfty;
      tend += D.qtf[n].ld(i, j, k);
      D.qn[n](i, j, k) = (m_full(D, k, mub, mu1) * D.q1[n].ld(i, j, k) + dt_rk * tend) / m_full(D, k, mub, mu2);
    }
    __syncthreads();  // the next species reuses the face arrays
  }
}
// The same update with the species' planes staged in shared memory by the tensor-memory accelerator: a block takes
// a tile of kQTx x kQTy columns over a chunk of q_chunk(SH) levels, one thread per point of it; for each species one
// copy per plane brings the tile's planes k0 - 2 .. k1 + 1 with a halo of 4 columns (the copy's x start stays
// 16-byte aligned) and 3 rows into a plane slot of its own (slots 128-byte aligned, as a tensor copy's destination
// must be), the next species' planes copied into the other buffer while this one is computed. The block forms every
// x, y and z face flux of the chunk once (shared arrays), then every point its update. Statement for statement the
// arithmetic of k_q_update (the same values are read, from shared memory instead of global memory).
template <class R>
struct QPlanes {  // a species' planes of one tile in shared memory, read with the domain's indices
  const R* s;
  int i0, j0, k0;  // the indices of s[0]
  static constexpr int W = kQTx + 8, H = kQTy + 6;
  static constexpr int PS = int((W * H * sizeof(R) + 127) / 128 * 128 / sizeof(R));  // plane slot, 128-byte multiple
  __device__ __forceinline__ R ld(int i, int j, int k) const { return s[(i - i0) + W * (j - j0) + PS * (k - k0)]; }
};
// the x, y and z face fluxes of a chunk
__host__ __device__ constexpr size_t q_face_elems(int shape) {
  return size_t(q_chunk(shape)) * (kQTy * (kQTx + 1) + (kQTy + 1) * kQTx) + size_t(q_chunk(shape) + 1) * kQTy * kQTx;
}
template <class R>
__host__ __device__ constexpr size_t q_march_smem(int shape) {
  // two plane buffers, then the x, y and z face fluxes of the chunk, and 128 bytes to align the start
  return 2 * size_t(q_chunk(shape) + 4) * QPlanes<R>::PS * sizeof(R) + q_face_elems(shape) * sizeof(R) + 128;
}
__host__ __device__ constexpr int q_march_threads(int shape) { return kQTx * kQTy * q_chunk(shape); }
template <class R, int NM, int SH>
// (1024 threads per SM by the launch bound: at most 64 registers a thread, 32 warps per SM where shared memory allows)
__global__ void __launch_bounds__(q_march_threads(SH), 1024 / q_march_threads(SH))
    k_q_march(const __grid_constant__ Pack<R, NM> P, int rk) {
  constexpr int KC = q_chunk(SH), NP = KC + 4, PL = QPlanes<R>::W * QPlanes<R>::H, PS = QPlanes<R>::PS;
  constexpr int kNX = KC * kQTy * (kQTx + 1), kNY = KC * (kQTy + 1) * kQTx, kNZ = (KC + 1) * kQTy * kQTx;
  extern __shared__ __align__(128) unsigned char q_smem[];
  __shared__ __align__(8) uint64_t bar[2];
  // the plane slots from the first 128-byte boundary of the dynamic shared memory (its size has 128 bytes to spare)
  R* const pbuf = reinterpret_cast<R*>(q_smem + ((128u - (smem_u32(q_smem) & 127u)) & 127u));
  R (*const sfx)[kQTy][kQTx + 1] = reinterpret_cast<R (*)[kQTy][kQTx + 1]>(pbuf + 2 * NP * PS);
  R (*const sfy)[kQTy + 1][kQTx] = reinterpret_cast<R (*)[kQTy + 1][kQTx]>(pbuf + 2 * NP * PS + KC * kQTy * (kQTx + 1));
  R (*const sfz)[kQTy][kQTx] =
      reinterpret_cast<R (*)[kQTy][kQTx]>(pbuf + 2 * NP * PS + KC * (kQTy * (kQTx + 1) + (kQTy + 1) * kQTx));
  const int b = blockIdx.x;
  const int m = member_of(P, RG_TILES, SH, b);
  const Dom<R>& D = P.d[m];
  const Range r = range_of(RG_TILES, D);
  const int bx = cdiv(r.i1 - r.i0, kQTx), by = cdiv(r.j1 - r.j0, kQTy);
  int local = b - P.start(RG_TILES, SH, m);
  const int bi = local % bx;
  local /= bx;
  const int bj = local % by;
  const int c0 = (local / by) * KC, c1 = min(c0 + KC, D.nz);
  const int tx = int(threadIdx.x) % kQTx, ty = (int(threadIdx.x) / kQTx) % kQTy, tk = int(threadIdx.x) / (kQTx * kQTy);
  const int ti0 = r.i0 + bi * kQTx, tj0 = r.j0 + bj * kQTy;
  const int i = ti0 + tx, j = tj0 + ty, k = c0 + tk;
  const int nx = D.nx, ny = D.ny;
  const bool lev = k < c1;  // this thread's point: its update
  const bool col = i < r.i1 && j < r.j1, in = col && lev;
  const R dt_rk = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  R mub = 0, mu1 = 0, mu2 = 0, msfty = 0;
  if (in) {
    mub = D.mub(i, j);
    mu1 = D.mu1.ld(i, j, 0);
    mu2 = D.mu2.ld(i, j, 0);
    msfty = D.msfty(i, j);
  }
  auto next = [&](int n) {  // the next species updated here (not PD at this stage), from n on
    while (n < D.n_scalars && q_is_pd(D, n, rk)) ++n;
    return n;
  };
  int n = next(0);
  if (n >= D.n_scalars) return;  // uniform over the block
  const QMap* const qm = D.qmap;
  // the map coordinates of the tile's first staged element (ti0 - 4, tj0 - 3, c0 - 2); x * sizeof(R) is a
  // multiple of 16 bytes: ti0 - r.i0 is a multiple of kQTx, and the map's x0 puts the domain's i = r.i0 - 4 at
  // a multiple of 4 elements
  const int xs = qm[0].x0 + ti0 - 4, ys = qm[0].y0 + tj0 - 3;
  if ((xs * int(sizeof(R))) % 16 != 0 || (smem_u32(pbuf) & 127u) != 0) {  // never (maps of cw_create, slots above):
    // an unaligned copy would fault
    if (threadIdx.x == 0) atomicOr(D.status, 2u);
    return;
  }
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](int s, int u) {  // thread 0: species s's planes into buffer u
    const CUtensorMap* map = D.q2[s].p == qm[s].pa ? &qm[s].a : &qm[s].b;
    mbar_expect_tx(&bar[u], unsigned(NP * PL * sizeof(R)));
    for (int p = 0; p < NP; ++p) tma_load_3d(pbuf + (u * NP + p) * PS, map, xs, ys, c0 - 2 + p, &bar[u]);
  };
  if (threadIdx.x == 0) issue(n, 0);
  unsigned phase[2] = {0u, 0u};
  for (int u = 0; n < D.n_scalars; u ^= 1) {
    const int nn = next(n + 1);
    const bool ok = mbar_wait(&bar[u], phase[u]);
    phase[u] ^= 1u;
    if (__syncthreads_or(!ok)) {  // the copies did not arrive: report, leave the species untouched
      if (threadIdx.x == 0) atomicOr(D.status, 1u);
      return;
    }
    // every thread has passed the barrier above after the species before: its reads of plane buffer u ^ 1 (the face
    // phase) and of the face arrays (the update phase) are over, so both may be written again
    if (nn < D.n_scalars && threadIdx.x == 0) issue(nn, u ^ 1);
    const QPlanes<R> T{pbuf + u * NP * PS, ti0 - 4, tj0 - 3, c0 - 2};
    // the chunk's faces in one flat list over the block's threads (consecutive threads take neighbouring faces of one
    // kind, so a warp's lanes seldom diverge): the x faces ti0 .. ti0 + 32 of rows in range, the y faces tj0 ..
    // tj0 + 4 of columns in range, the z faces c0 .. c1 of the columns in range; the faces up to nx (ny) and r.i1
    // (r.j1), as k_q_update forms them
    for (int f = int(threadIdx.x); f < kNX + kNY + kNZ; f += q_march_threads(SH)) {
      if (f < kNX) {
        const int fi = f % (kQTx + 1), fj = (f / (kQTx + 1)) % kQTy, fk = f / ((kQTx + 1) * kQTy);
        const int fi_ = ti0 + fi, fj_ = tj0 + fj, fk_ = c0 + fk;
        if (fk_ < c1 && fj_ < r.j1 && fj_ < ny && fi_ <= nx && fi_ <= r.i1)
          sfx[fk][fj][fi] = sc_fx(D, T, D.ru_m, fi_, fj_, fk_, false);
      } else if (f < kNX + kNY) {
        const int g = f - kNX;
        const int fi = g % kQTx, fj = (g / kQTx) % (kQTy + 1), fk = g / (kQTx * (kQTy + 1));
        const int fi_ = ti0 + fi, fj_ = tj0 + fj, fk_ = c0 + fk;
        if (D.do_y && fk_ < c1 && fi_ < r.i1 && fi_ < nx && fj_ <= ny && fj_ <= r.j1)
          sfy[fk][fj][fi] = sc_fy(D, T, D.rv_m, fi_, fj_, fk_, false);
      } else {
        const int g = f - kNX - kNY;
        const int fi = g % kQTx, fj = (g / kQTx) % kQTy, fk = g / (kQTx * kQTy);
        const int fi_ = ti0 + fi, fj_ = tj0 + fj, fk_ = c0 + fk;
        if (fk_ <= c1 && fi_ < r.i1 && fj_ < r.j1) sfz[fk][fj][fi] = sc_fz(D, T, D.ww_m, fi_, fj_, fk_, false);
      }
    }
    __syncthreads();
    if (in) {
      R a = 0;
      if (!spec_cell(D, i, j)) {
        const R h = q_adv_h(D, D.q2[n], i, j, k, sfx[tk][ty][tx], sfx[tk][ty][tx + 1], sfy[tk][ty][tx], sfy[tk][ty + 1][tx]);
        a = h - R(D.rdnw[k]) * (sfz[tk + 1][ty][tx] - sfz[tk][ty][tx]);
      }
      R tend = a * msfty;
      tend += D.qtf[n].ld(i, j, k);
      D.qn[n](i, j, k) = (m_full(D, k, mub, mu1) * D.q1[n].ld(i, j, k) + dt_rk * tend) / m_full(D, k, mub, mu2);
    }
    n = nn;  // no barrier here: the one after the next species' wait orders these reads before its writes
  }
}
// KPreUpdatePD (:174-180)
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX) k_q_pre_pd(const __grid_constant__ Pack<R, NM> P, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt_rk = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const R m = m_full(D, k, D.mub(i, j), D.mu1(i, j, 0));
  const int n = blockIdx.y;  // the species
  if (n >= D.n_scalars) return;
  if (!q_is_pd(D, n, rk)) return;
  D.q1[n](i, j, k) = (m * D.q1[n](i, j, k) + dt_rk * D.qtf[n](i, j, k)) / m;
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
// KFacePDX / KFacePDY / KFacePDZ (:159-171 with the PD statement functions): every face flux of the PD
// species once, dh and lo, into the species' face arrays (x faces 0..nx, y faces 0..ny, z faces 0..nz). One
// thread per face point for all species: the Courant number and the mass factor of a face (the expressions
// of pd_fx / pd_fy / pd_fz) do not depend on the species and are evaluated once.
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX, 10) k_q_face_pd(const __grid_constant__ Pack<R, NM> P, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  // RG_FACES: in a patch, the faces of its cells up to the face after its last one (the cells' updates read both)
  if (!thread_index<SH>(P, RG_FACES, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const R dt = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const bool fx = j < ny && k < nz, fy = D.do_y && i < nx && k < nz, fz = i < nx && j < ny;
  const bool zin = fz && k != 0 && k != nz;
  R crx = 0, facx = 0, cry = 0, facy = 0, crz = 0, facz = 0;
  if (fx) {
    const R dx = R(2) / (D.msfty(i, j) + D.msfty(i - 1, j)) / R(D.rdx), mu = R(0.5) * (pd_mh(D, i, j, k) + pd_mh(D, i - 1, j, k)),
            vel = D.ru_m.ld(i, j, k);
    crx = (D.spec_x && i == 1) ? (vel / mu) * dt / dx : vel * dt / dx / mu;
    facx = mu * (dx / dt);
  }
  if (fy) {
    const R dy = R(2) / (D.msftx(i, j) + D.msftx(i, j - 1)) / R(D.rdy), mu = R(0.5) * (pd_mh(D, i, j, k) + pd_mh(D, i, j - 1, k)),
            vel = D.rv_m.ld(i, j, k);
    cry = vel * dt / dy / mu;
    facy = mu * (dy / dt);
  }
  if (zin) {
    const R dz = R(2) / (R(D.rdnw[k]) + R(D.rdnw[k - 1])), mu = pd_mh(D, i, j, k), vel = D.ww_m.ld(i, j, k);
    crz = vel * dt / dz / mu;
    facz = mu * (dz / dt);
  }
  for (int n = 0; n < D.n_scalars; ++n) {
    if (!q_is_pd(D, n, rk)) continue;
    const V3<R> q = D.q2[n], qo = D.q1[n];
    R dhx = 0, lox = 0, dhy = 0, loy = 0, dhz = 0, loz = 0;
    if (fx) {
      lox = facx * flux_upwind(qo.ld(i - 1, j, k), qo.ld(i, j, k), crx);
      dhx = sc_fx(D, q, D.ru_m, i, j, k, true) - lox;
    }
    if (fy) {
      loy = facy * flux_upwind(qo.ld(i, j - 1, k), qo.ld(i, j, k), cry);
      dhy = sc_fy(D, q, D.rv_m, i, j, k, true) - loy;
    }
    if (zin) {
      loz = facz * flux_upwind(qo.ld(i, j, k - 1), qo.ld(i, j, k), crz);
      dhz = sc_fz(D, q, D.ww_m, i, j, k, true) - loz;
    } else if (fz) {
      loz = 0;
      dhz = R(0) - R(0);
    }
    const V3<R>* f = D.qpd + 6 * n;
    if (fx) {
      f[0](i, j, k) = dhx;
      f[1](i, j, k) = lox;
    }
    if (fy) {
      f[2](i, j, k) = dhy;
      f[3](i, j, k) = loy;
    }
    if (fz) {
      f[4](i, j, k) = dhz;
      f[5](i, j, k) = loz;
    }
  }
}
// KScalePD (:215-241) from the stored face fluxes
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX) k_q_scale_pd(const __grid_constant__ Pack<R, NM> P, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const bool edge = (D.spec_x && (i == 0 || i == D.nx - 1)) || (D.spec_y && (j == 0 || j == D.ny - 1));
  const int n = blockIdx.y;  // the species
  if (n >= D.n_scalars) return;
  if (!q_is_pd(D, n, rk)) return;
  if (edge) {
    D.qscale[n](i, j, k) = 1;
    return;
  }
  const V3<R>& qo = D.q1[n];
  const V3<R>* f = D.qpd + 6 * n;
  const R dhx0 = f[0](i, j, k), lox0 = f[1](i, j, k), dhx1 = f[0](i + 1, j, k), lox1 = f[1](i + 1, j, k);
  R dhy0 = 0, loy0 = 0, dhy1 = 0, loy1 = 0;
  if (D.do_y) {
    dhy0 = f[2](i, j, k);
    loy0 = f[3](i, j, k);
    dhy1 = f[2](i, j + 1, k);
    loy1 = f[3](i, j + 1, k);
  }
  const R dhz0 = f[4](i, j, k), loz0 = f[5](i, j, k), dhz1 = f[4](i, j, k + 1), loz1 = f[5](i, j, k + 1);
  const R mxy = D.msftx(i, j) * D.msfty(i, j);
  R hlow = R(D.rdx) * (lox1 - lox0);
  if (D.do_y) hlow += R(D.rdy) * (loy1 - loy0);
  const R ph_low = ((R(D.c1h[k]) * D.mub(i, j) + R(D.c2h[k])) + R(D.c1h[k]) * D.mu1(i, j, 0)) * qo(i, j, k) -
                   dt * (mxy * hlow + D.msfty(i, j) * R(D.rdnw[k]) * (loz1 - loz0));
  R hout = R(D.rdx) * ((dhx1 > 0 ? dhx1 : R(0)) - (dhx0 < 0 ? dhx0 : R(0)));
  if (D.do_y) hout += R(D.rdy) * ((dhy1 > 0 ? dhy1 : R(0)) - (dhy0 < 0 ? dhy0 : R(0)));
  const R out = mxy * hout + D.msfty(i, j) * R(D.rdnw[k]) * ((dhz1 < 0 ? dhz1 : R(0)) - (dhz0 > 0 ? dhz0 : R(0)));
  const R flux_out = dt * out;
  R sc = 1;
  if (flux_out > ph_low) {
    sc = ph_low / (flux_out + R(1e-20));
    if (sc < 0) sc = 0;
  }
  D.qscale[n](i, j, k) = sc;
}
// KUpdatePD in an outermost cell of an open boundary (:275-281): the open terms (Fluxes::open_terms :110-116,
// field_old = scalar_old), the vertical term, the x term (not in the outer columns), the y term (not in the outer
// rows). Out of line: it runs on the boundary ring only.
template <class R>
__device__ __noinline__ void q_update_pd_open(const Dom<R>& D, int n, R dt, int i, int j, int k) {
  const R mub = D.mub(i, j), mu1 = D.mu1(i, j, 0), mu2 = D.mu2(i, j, 0);
  const V3<R>& qo = D.q1[n];
  const V3<R>& sc = D.qscale[n];
  const bool ocol = D.open_x && (i == 0 || i == D.nx - 1), orow = D.open_y && (j == 0 || j == D.ny - 1);
  const V3<R>* f = D.qpd + 6 * n;
  const R s0 = sc(i, j, k);
  auto lim = [](R d, R s_up, R s_dn) { return d * (d > 0 ? s_up : (d < 0 ? s_dn : R(1))); };
  const R dhz0 = f[4](i, j, k), loz0 = f[5](i, j, k), dhz1 = f[4](i, j, k + 1), loz1 = f[5](i, j, k + 1);
  const R szm = k == 0 ? R(0) : sc(i, j, k - 1), szp = (k + 1 == D.nz) ? R(0) : sc(i, j, k + 1);
  const R dz0 = (k == 0) ? R(0) : lim(dhz0, s0, szm);
  const R dz1 = (k + 1 == D.nz) ? R(0) : lim(dhz1, szp, s0);
  R tend = R(0);
  if (ocol) tend = tend - open_scalar<R, 1>(D, D.q2[n], qo, D.ru_m, i, j, k);
  if (orow) tend = tend - open_scalar<R, 0>(D, D.q2[n], qo, D.rv_m, i, j, k);
  tend = tend - R(D.rdnw[k]) * (dz1 - dz0 + loz1 - loz0);
  if (!ocol) {
    const R dhx0 = f[0](i, j, k), lox0 = f[1](i, j, k), dhx1 = f[0](i + 1, j, k), lox1 = f[1](i + 1, j, k);
    const R dx0 = lim(dhx0, sc(i - 1, j, k), s0), dx1 = lim(dhx1, s0, sc(i + 1, j, k));
    tend -= D.msftx(i, j) * (R(D.rdx) * (dx1 - dx0 + lox1 - lox0));
  }
  if (D.do_y && !orow) {
    const R dhy0 = f[2](i, j, k), loy0 = f[3](i, j, k), dhy1 = f[2](i, j + 1, k), loy1 = f[3](i, j + 1, k);
    const R dy0 = lim(dhy0, sc(i, j - 1, k), s0), dy1 = lim(dhy1, s0, sc(i, j + 1, k));
    tend -= D.msftx(i, j) * (R(D.rdy) * (dy1 - dy0 + loy1 - loy0));
  }
  D.qn[n](i, j, k) = (m_full(D, k, mub, mu1) * qo(i, j, k) + dt * (tend * D.msfty(i, j))) / m_full(D, k, mub, mu2);
}
// KUpdatePD (:244-291) from the stored face fluxes; the launch bound keeps the interior path at 40 registers (the
// boundary ring's out-of-line update spills instead)
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX, 12) k_q_update_pd(const __grid_constant__ Pack<R, NM> P, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const R dt = R(rk == 1 ? D.dt / 3.0 : (rk == 2 ? 0.5 * D.dt : D.dt));
  const R mub = D.mub(i, j), mu1 = D.mu1(i, j, 0), mu2 = D.mu2(i, j, 0);
  const int n = blockIdx.y;  // the species
  if (n >= D.n_scalars) return;
  if (!q_is_pd(D, n, rk)) return;
  const V3<R>& qo = D.q1[n];
  const V3<R>& sc = D.qscale[n];
  if (spec_cell(D, i, j)) {
    D.qn[n](i, j, k) = m_full(D, k, mub, mu1) * qo(i, j, k) / m_full(D, k, mub, mu2);
    return;
  }
  if ((D.open_x && (i == 0 || i == D.nx - 1)) || (D.open_y && (j == 0 || j == D.ny - 1))) {
    q_update_pd_open(D, n, dt, i, j, k);
    return;
  }
  const V3<R>* f = D.qpd + 6 * n;
  const R dhx0 = f[0](i, j, k), lox0 = f[1](i, j, k), dhx1 = f[0](i + 1, j, k), lox1 = f[1](i + 1, j, k);
  const R dhz0 = f[4](i, j, k), loz0 = f[5](i, j, k), dhz1 = f[4](i, j, k + 1), loz1 = f[5](i, j, k + 1);
  const R s0 = sc(i, j, k), sxm = sc(i - 1, j, k), sxp = sc(i + 1, j, k);
  const R szm = k == 0 ? R(0) : sc(i, j, k - 1), szp = (k + 1 == D.nz) ? R(0) : sc(i, j, k + 1);
  auto lim = [](R d, R s_up, R s_dn) { return d * (d > 0 ? s_up : (d < 0 ? s_dn : R(1))); };
  const R dx0 = lim(dhx0, sxm, s0), dx1 = lim(dhx1, s0, sxp);
  const R dz0 = (k == 0) ? R(0) : lim(dhz0, s0, szm);
  const R dz1 = (k + 1 == D.nz) ? R(0) : lim(dhz1, szp, s0);
  R tend = -R(D.rdnw[k]) * (dz1 - dz0 + loz1 - loz0);
  tend -= D.msftx(i, j) * (R(D.rdx) * (dx1 - dx0 + lox1 - lox0));
  if (D.do_y) {
    const R dhy0 = f[2](i, j, k), loy0 = f[3](i, j, k), dhy1 = f[2](i, j + 1, k), loy1 = f[3](i, j + 1, k);
    const R dy0 = lim(dhy0, sc(i, j - 1, k), s0), dy1 = lim(dhy1, s0, sc(i, j + 1, k));
    tend -= D.msftx(i, j) * (R(D.rdy) * (dy1 - dy0 + loy1 - loy0));
  }
  D.qn[n](i, j, k) = (m_full(D, k, mub, mu1) * qo(i, j, k) + dt * (tend * D.msfty(i, j))) / m_full(D, k, mub, mu2);
}
// swap(q_2, q_new) of every species (ScalarTransport::update :425)
template <class R, int NM>
__global__ void k_q_swap(const __grid_constant__ Pack<R, NM> P) {
  const int m = blockIdx.x;
  if (m >= P.n) return;
  const Dom<R>& D = P.d[m];
  for (int n = threadIdx.x; n < D.n_scalars; n += blockDim.x) {
    const V3<R> t = D.q2[n];
    D.q2[n] = D.qn[n];
    D.qn[n] = t;
  }
}

}  // namespace cw
