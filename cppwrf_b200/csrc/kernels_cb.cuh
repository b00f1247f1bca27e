// SPDX-License-Identifier: GPL-3.0-or-later
// Column-block kernels: a CTA holds CX neighbouring columns along i (the lanes, so every global access is
// coalesced along i) and CNW warps. The pointwise work of the levels is split over the warps; the
// vertical recurrences -- column sums, running integrals, the tridiagonal sweeps -- run on warp 0, one lane
// per column, in the reference's order, on per-level terms staged in shared memory. Every value is the
// same expression as the reference's column functor, so the results are bit-identical to it.
#pragma once

#include "kernels_ac.cuh"

namespace cw {

#define CB_LOOP(k, n) for (int k = int(threadIdx.y); k < (n); k += NW)
// the same for a body whose only stores go to shared memory: unrolled, the loads of the next level can be
// issued before the stores of this one (shared stores cannot alias global loads)
#define CB_LOOP_SH(k, n) _Pragma("unroll 2") for (int k = int(threadIdx.y); k < (n); k += NW)
// unrolled by two where that measured faster although the body stores to global memory (its read-only loads of
// the next level can still be issued early)
#define CB_LOOP_U2(k, n) _Pragma("unroll 2") for (int k = int(threadIdx.y); k < (n); k += NW)


// a hint that brings the line of a into L2 (no register, no wait): the column blocks' level loops then meet L2
// instead of DRAM latency
__device__ __forceinline__ void pf_l2(const void* a) { asm volatile("prefetch.global.L2 [%0];" ::"l"(a)); }
// the levels of a loop split over warps 1 .. NW - 1 (warp 0 runs a recurrence meanwhile)
#define CB_LOOP_W1(k, n) for (int k = int(threadIdx.y) - 1; threadIdx.y > 0 && k < (n); k += NW - 1)
// block -> (member, column i of this lane, row j)
// (ilim: the end of the member's column range along i; the lanes at or past it have no column)
template <class R, int NM>
__device__ __forceinline__ const Dom<R>& cb_member(const Pack<R, NM>& P, int kind, int& i, int& j, int& ilim) {
  const int b = blockIdx.x;
  const int m = member_of(P, kind, 0, b);
  const Dom<R>& D = P.d[m];
  const Range r = range_of(kind, D);
  const int bx = cdiv(r.i1 - r.i0, CX);
  const int local = b - P.start(kind, 0, m);
  i = r.i0 + (local % bx) * CX + int(threadIdx.x);
  j = r.j0 + local / bx;
  ilim = r.i1;
  return D;
}
// shared level array a of the block: a[k * CX + lane]
__device__ __forceinline__ double* cb_array(int a, int nz) {
  extern __shared__ double cb_smem[];
  return cb_smem + size_t(a) * (nz + 2) * CX;
}

// rk_step_prep: KMu (large_step.cpp:49-66), KPrep3 (:68-81), KWW (:83-108), KCq (:127-148)
template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW, cb_minblocks(NW)) k_ls_prep(const __grid_constant__ Pack<R, NM> P) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_STAG, i, j, ilim);
  const int nx = D.nx, ny = D.ny, nz = D.nz, nyv = D.nyv;
  const int lane = threadIdx.x;
  const bool col = i < ilim;  // a column of the member (its faces' range)
  const bool w0 = threadIdx.y == 0;
  const int spx = D.spec_x, spy = D.spec_y;
  double* s_div = cb_array(0, nz);
  R muu = 0, muv = 0, mut = 0;
  if (col) {
    if (i < nx && j < ny) mut = D.mu2.ld(i, j, 0) + D.mub(i, j);
    if (j < ny) {
      if (spx && i == 0) muu = R(0.5) * (D.mu2.ld(0, j, 0) + D.mu2.ld(0, j, 0) + D.mub(0, j) + D.mub(0, j));
      else if (spx && i == nx)
        muu = R(0.5) * (D.mu2.ld(nx - 1, j, 0) + D.mu2.ld(nx - 1, j, 0) + D.mub(nx - 1, j) + D.mub(nx - 1, j));
      else muu = R(0.5) * (D.mu2.ld(i, j, 0) + D.mu2.ld(i - 1, j, 0) + D.mub(i, j) + D.mub(i - 1, j));
    }
    if (i < nx && j < nyv) {
      if (spy && j == 0) muv = R(0.5) * (D.mu2.ld(i, 0, 0) + D.mu2.ld(i, 0, 0) + D.mub(i, 0) + D.mub(i, 0));
      else if (spy && j == ny)
        muv = R(0.5) * (D.mu2.ld(i, ny - 1, 0) + D.mu2.ld(i, ny - 1, 0) + D.mub(i, ny - 1) + D.mub(i, ny - 1));
      else muv = R(0.5) * (D.mu2.ld(i, j, 0) + D.mu2.ld(i, j - 1, 0) + D.mub(i, j) + D.mub(i, j - 1));
    }
    if (w0) {
      if (i < nx && j < ny) D.mut(i, j, 0) = mut;
      if (j < ny) D.muu(i, j, 0) = muu;
      if (i < nx && j < nyv) D.muv(i, j, 0) = muv;
    }
    CB_LOOP(k, nz + 1) {  // KPrep3 (every load of a level before its first store)
      const bool has_u = j < ny && k < nz, has_v = i < nx && j < nyv && k < nz, has_w = i < nx && j < ny;
      const bool has_m = has_w && k < nz;
      const R u2 = has_u ? D.u2.ld(i, j, k) : R(0), msfuy = has_u ? D.msfuy(i, j) : R(1);
      const R v2 = has_v ? D.v2.ld(i, j, k) : R(0), mvxi = has_v ? D.msfvx_inv(i, j) : R(0);
      const R w2 = has_w ? D.w2.ld(i, j, k) : R(0), msfty = has_w ? D.msfty(i, j) : R(1);
      R al = 0, alb = 0, phb0 = 0, phb1 = 0, ph0 = 0, ph1 = 0;
      if (has_m) {
        al = D.al.ld(i, j, k);
        alb = D.alb(i, j, k);
        phb0 = D.phb(i, j, k);
        phb1 = D.phb(i, j, k + 1);
        ph0 = D.ph2.ld(i, j, k);
        ph1 = D.ph2.ld(i, j, k + 1);
      }
      if (has_u) D.ru(i, j, k) = div_msf(u2 * (R(D.c1h[k]) * muu + R(D.c2h[k])), msfuy);
      if (has_v) D.rv(i, j, k) = v2 * (R(D.c1h[k]) * muv + R(D.c2h[k])) * mvxi;
      if (has_w) D.rw(i, j, k) = div_msf(w2 * (R(D.c1f[k]) * mut + R(D.c2f[k])), msfty);
      if (has_m) {
        D.alt(i, j, k) = al + alb;
        D.php(i, j, k) = R(0.5) * (phb0 + phb1 + ph0 + ph1);
      }
    }
  }
  const bool mass = col && i < nx && j < ny;
  R mu1 = 0, mu0 = 0, mv1 = 0, mv0 = 0;
  if (mass) {
    mu1 = ww_mu_u(D, i + 1, j);
    mu0 = ww_mu_u(D, i, j);
    mv1 = ww_mu_v(D, i, j + 1);
    mv0 = ww_mu_v(D, i, j);
    CB_LOOP_SH(k, nz) s_div[k * CX + lane] = double(ww_divv(D, i, j, k, mu1, mu0, mv1, mv0));
  }
  __syncthreads();
  if (mass && w0) {  // KWW: the column integral, then the running sum, in the reference's order
    R dmdt = 0;
#pragma unroll 4
    for (int k = 0; k < nz; ++k) dmdt += R(s_div[k * CX + lane]);
    R w = 0;
#pragma unroll 4
    for (int k = 1; k < nz; ++k) {  // ww of level k into the slot of the divergence it consumed
      w = w - R(D.dnw[k - 1]) * R(D.c1h[k - 1]) * dmdt - R(s_div[(k - 1) * CX + lane]);
      s_div[(k - 1) * CX + lane] = double(w);
    }
  }
  __syncthreads();
  if (mass) CB_LOOP(k, nz + 1) D.ww(i, j, k) = (k == 0 || k == nz) ? R(0) : R(s_div[(k - 1) * CX + lane]);
  if (col && D.n_moist > 0) {  // KCq
    CB_LOOP(k, nz) {  // the three sums over species first, then the stores
      const bool has_u = j < ny, has_v = i < nx && j < nyv, has_w = i < nx && j < ny && k >= 1;
      R tu = 0, tv = 0, tw = 0;
      for (int s = 0; s < D.n_moist; ++s) {
        const V3<R> q = D.q2[s];
        const R q0 = q(i, j, k);
        if (has_u) tu = tu + q0 + q(i - 1, j, k);
        if (has_v) tv = tv + q0 + q(i, j - 1, k);
        if (has_w) tw = tw + q0 + q(i, j, k - 1);
      }
      if (has_u) D.cqu(i, j, k) = R(1) / (R(1) + R(0.5) * tu);
      if (has_v) D.cqv(i, j, k) = R(1) / (R(1) + R(0.5) * tv);
      if (has_w) D.cqw(i, j, k) = R(0.5) * tw;
    }
  }
}

// small_step_prep (KPrep small_step.cpp:50-93) + calc_p_rho (KPRho :114-119) + calc_coef_w (KCoefW :122-148)
template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW, cb_minblocks(NW)) k_ss_prep(const __grid_constant__ Pack<R, NM> P, int rk) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_STAG, i, j, ilim);
  const int nx = D.nx, ny = D.ny, nz = D.nz, nyv = D.nyv;
  const int lane = threadIdx.x;
  const bool col = i < ilim;  // a column of the member (its faces' range)
  const bool w0 = threadIdx.y == 0;
  const bool mass = col && i < nx && j < ny;
  const bool first = rk == 1;
  R mts = 0, mus_u = 0, mus_v = 0, mut = 0;
  if (col) {
    mts = D.mub(i, j) + D.mu1.ld(i, j, 0);
    mus_u = first ? D.muu.ld(i, j, 0) : R(0.5) * (mts + D.mub(i - 1, j) + D.mu1.ld(i - 1, j, 0));
    mus_v = first ? D.muv.ld(i, j, 0) : R(0.5) * (mts + D.mub(i, j - 1) + D.mu1.ld(i, j - 1, 0));
    if (mass) mut = D.mut.ld(i, j, 0);
    if (w0) {
      if (mass) {
        D.muts(i, j, 0) = mts;
        D.mu_save(i, j, 0) = D.mu2(i, j, 0);
        D.mu2(i, j, 0) = D.mu1.ld(i, j, 0) - D.mu2(i, j, 0);
      }
      if (j < ny) D.muus(i, j, 0) = mus_u;
      if (i < nx && j < nyv) D.muvs(i, j, 0) = mus_v;
    }
    CB_LOOP_U2(k, nz + 1) {  // KPrep (every load of a level before its first store)
      const R c1h = k < nz ? R(D.c1h[k]) : R(0), c2h = k < nz ? R(D.c2h[k]) : R(0);
      const bool has_u = j < ny && k < nz, has_v = i < nx && j < nyv && k < nz;
      R ui = 0, u1 = 0, muu = 0, msfuy = 1, vi = 0, v1 = 0, muv = 0, mvxi = 0;
      if (has_u) {
        ui = D.u2(i, j, k);
        u1 = D.u1.ld(i, j, k);
        muu = D.muu.ld(i, j, 0);
        msfuy = D.msfuy(i, j);
      }
      if (has_v) {
        vi = D.v2(i, j, k);
        v1 = D.v1.ld(i, j, k);
        muv = D.muv.ld(i, j, 0);
        mvxi = D.msfvx_inv(i, j);
      }
      R ti = 0, t1 = 0, pb = 0, pp = 0, alt = 1, wi = 0, w1 = 0, msfty = 1, phi = 0, ph1 = 0, ww = 0;
      if (mass) {
        if (k < nz) {
          ti = D.t2(i, j, k);
          t1 = D.t1.ld(i, j, k);
          pb = D.pb(i, j, k);
          pp = D.p(i, j, k);
          alt = D.alt.ld(i, j, k);
        }
        wi = D.w2(i, j, k);
        w1 = D.w1.ld(i, j, k);
        msfty = D.msfty(i, j);
        phi = D.ph2(i, j, k);
        ph1 = D.ph1.ld(i, j, k);
        ww = (k == 0 || k == nz) ? R(0) : D.ww.ld(i, j, k);
      }
      if (has_u) {
        D.u_save(i, j, k) = ui;
        D.u2(i, j, k) = div_msf(((c1h * mus_u + c2h) * u1 - (c1h * muu + c2h) * ui), msfuy);
      }
      if (has_v) {
        D.v_save(i, j, k) = vi;
        D.v2(i, j, k) = ((c1h * mus_v + c2h) * v1 - (c1h * muv + c2h) * vi) * mvxi;
      }
      if (mass) {
        if (k < nz) {
          D.t_save(i, j, k) = ti;
          D.t2(i, j, k) = (c1h * mts + c2h) * t1 - (c1h * mut + c2h) * ti;
          D.c2a(i, j, k) = R(k::cpovcv) * (pb + pp) / alt;
        }
        D.w_save(i, j, k) = wi;
        D.w2(i, j, k) = div_msf(((R(D.c1f[k]) * mts + R(D.c2f[k])) * w1 - (R(D.c1f[k]) * mut + R(D.c2f[k])) * wi), msfty);
        D.ph_save(i, j, k) = phi;
        D.ph2(i, j, k) = ph1 - phi;
        D.ww1(i, j, k) = ww;
      }
    }
  }
  __syncthreads();
  using A = double;
  double* s_a = cb_array(0, nz);
  double* s_b = cb_array(1, nz);
  double* s_c = cb_array(2, nz);
  const A dts = rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound;
  const A cof_h = 0.5 * A(R(dts)) * k::g * (1.0 + A(R(D.epssm)));
  const A cof = A(R(cof_h * cof_h));
  const A m = A(mut);
  auto mh = [&](int kk, A mm) { return D.c1h[kk] * mm + D.c2h[kk]; };
  auto mf = [&](int kk, A mm) { return D.c1f[kk] * mm + D.c2f[kk]; };
  auto cq1 = [&](int kk) { return A(R(1) / (R(1) + cqw_(D, i, j, kk))); };
  if (mass) {
    CB_LOOP(k, nz) p_rho_point<false>(D, i, j, k, false);
    // calc_coef_w: the pointwise coefficients a, b, c of each level
    CB_LOOP(k, nz + 1) {
      A a = 0, b = 0, cc = 0;
      if (k == nz) {
        a = -2. * cof * (D.rdnw[nz - 1] * D.rdnw[nz - 1]) * A(D.c2a(i, j, nz - 1)) * (D.top_lid ? 0.0 : 1.0) /
            (mh(nz - 1, m) * mf(nz - 1, m));
        b = 1. + 2. * cof * (D.rdnw[nz - 1] * D.rdnw[nz - 1]) * A(D.c2a(i, j, nz - 1)) / (mh(nz - 1, m) * mf(nz, m));
      } else if (k >= 1) {
        if (k >= 2) a = -cq1(k) * cof * D.rdn[k] * D.rdnw[k - 1] * A(D.c2a(i, j, k - 1)) / (mh(k - 1, m) * mf(k - 1, m));
        const A q1 = cq1(k);
        b = 1. + q1 * cof * D.rdn[k] *
                     (D.rdnw[k] * A(D.c2a(i, j, k)) / (mh(k, m) * mf(k, m)) +
                      D.rdnw[k - 1] * A(D.c2a(i, j, k - 1)) / (mh(k - 1, m) * mf(k, m)));
        cc = -q1 * cof * D.rdn[k] * D.rdnw[k] * A(D.c2a(i, j, k)) / (mh(k, m) * mf(k + 1, m));
      }
      s_a[k * CX + lane] = A(R(a));
      s_b[k * CX + lane] = b;
      s_c[k * CX + lane] = cc;
      D.a(i, j, k) = R(a);
    }
  }
  __syncthreads();
  if (mass && w0) {  // the forward-elimination factors, a recurrence in k
    D.alpha(i, j, 0) = 0;
    D.gamma(i, j, 0) = 0;
    A gprev = 0;
#pragma unroll 4
    for (int k = 1; k < nz; ++k) {
      const A al = 1. / (s_b[k * CX + lane] - s_a[k * CX + lane] * gprev);
      D.alpha(i, j, k) = R(al);
      gprev = A(R(s_c[k * CX + lane] * A(R(al))));
      D.gamma(i, j, k) = R(gprev);
    }
    D.alpha(i, j, nz) = R(1. / (s_b[nz * CX + lane] - s_a[nz * CX + lane] * gprev));
    D.gamma(i, j, nz) = 0;
  }
}

// One acoustic substep of a column block: advance_mu_t + sumflux (KMuTCol :208-249, KMuTPoint :251-277,
// KSumEdge :281-290) (phase 1), advance_w (KWRhs / KWExpl / KWSolve :295-408) (phase 2), calc_p_rho with
// divergence damping (KWPRho :411-416) (phase 3). The column mass sum, the running
// omega integral and the tridiagonal sweeps are evaluated in double in both forms, on terms staged in
// shared memory. With lateral boundaries the spec zone's columns take LateralBC::update_mu_t (phase 1) and
// the phi'' part of update_ph_w (phase 2); the zero-gradient w of that zone needs the neighbours' new w and
// follows in its own launch.
template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW, cb_minblocks(NW)) k_ac(const __grid_constant__ Pack<R, NM> P, int rk, int it,
                                                    int nsteps) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_STAG, i, j, ilim);
  using A = double;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const int lane = threadIdx.x;
  const bool w0 = threadIdx.y == 0;
  const bool col = i < ilim;  // a column of the member (its faces' range)
  const R dts = R(rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound);
  const R epssm = R(D.epssm);
  const bool first = it == 1, last = it == nsteps;
  const R rn = R(nsteps);
  const bool mass = col && i < nx && j < ny;
  const bool spec = mass && edge_mass(D, i, j);
  const bool dyn = mass && !spec;
  double* s0 = cb_array(0, nz);
  double* s1 = cb_array(1, nz);
  double* s2 = cb_array(2, nz);
  double* sc = cb_array(3, nz);  // per-column scalars: sc[n * CX + lane]
  double* s_t2s = cb_array(4, nz);  // theta'' before the substep's update (t_2save), phase 1 to phase 2

  if (mass)  // phase 1's inputs of the block's columns into L2 (a level above nz takes level 0: inside the field)
    CB_LOOP(k, nz + 1) {
      const int kh = k < nz ? k : 0;
      pf_l2(&D.u2(i, j, kh));
      pf_l2(&D.u2(i + 1, j, kh));
      pf_l2(&D.u_save(i, j, kh));
      pf_l2(&D.ru_m(i, j, kh));
      if (D.do_y) {
        pf_l2(&D.v2(i, j, kh));
        pf_l2(&D.v2(i, j + 1, kh));
        pf_l2(&D.v_save(i, j, kh));
        pf_l2(&D.v_save(i, j + 1, kh));
        pf_l2(&D.rv_m(i, j, kh));
      }
      pf_l2(&D.ww1(i, j, k));
      pf_l2(&D.ww_m(i, j, k));
      if (k < nz) {
        pf_l2(&D.t2(i, j, k));
        pf_l2(&D.t_tend(i, j, k));
        pf_l2(&D.t_save(i, j, k));
        if (D.do_y) {
          pf_l2(&D.t_save(i, j - 1, k));
          pf_l2(&D.t_save(i, j + 1, k));
        }
      }
    }
  {  // phase 1
    if (col && D.spec_x && i == nx && j < ny)  // KSumEdge, east face (specified or open x)
      CB_LOOP(k, nz) {
        const R su = (first ? R(0) : D.ru_m(i, j, k)) + D.u2.ld(i, j, k);
        const R cpl = (R(D.c1h[k]) * D.muu.ld(i, j, 0) + R(D.c2h[k])) * D.u_save.ld(i, j, k);
        D.ru_m(i, j, k) = last ? su / rn + div_msf(cpl, D.msfuy(i, j)) : su;
      }
    if (col && D.spec_y && j == ny && i < nx)  // KSumEdge, north face (specified or open y)
      CB_LOOP(k, nz) {
        const R su = (first ? R(0) : D.rv_m(i, j, k)) + D.v2.ld(i, j, k);
        const R cpl = (R(D.c1h[k]) * D.muv.ld(i, j, 0) + R(D.c2h[k])) * D.v_save.ld(i, j, k);
        D.rv_m(i, j, k) = last ? su / rn + cpl * D.msfvx_inv(i, j) : su;
      }
    if (spec) {  // spec zone: sumflux of ww only; mu and mu_ts take dts mu_tend (LateralBC::update_mu_t :363-372)
      CB_LOOP(k, nz + 1) {
        const R sw = (first ? R(0) : D.ww_m(i, j, k)) + D.ww(i, j, k);
        D.ww_m(i, j, k) = last ? sw / rn + D.ww1.ld(i, j, k) : sw;
      }
      if (w0) {
        D.mu2(i, j, 0) += dts * D.mu_tend.ld(i, j, 0);
        D.muts(i, j, 0) += dts * D.mu_tend.ld(i, j, 0);
      }
    }
    if (mass)
      CB_LOOP(k, nz) {  // dv of each level (KMuTDiv), the time sums of ru, rv (KMuTPoint), ww1 staged
        const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
        const R u_k = D.u2.ld(i, j, k), usv = D.u_save.ld(i, j, k), muu = D.muu.ld(i, j, 0), msfuy = D.msfuy(i, j);
        const R rum = first ? R(0) : D.ru_m(i, j, k);
        R v_k = 0, vsv = 0, muv = 0, mvxi = 0, rvm = 0;
        if (D.do_y) {
          v_k = D.v2.ld(i, j, k);
          vsv = D.v_save.ld(i, j, k);
          muv = D.muv.ld(i, j, 0);
          mvxi = D.msfvx_inv(i, j);
          rvm = first ? R(0) : D.rv_m(i, j, k);
        }
        if (dyn) {
          const R u_ip = D.u2.ld(i + 1, j, k), usv_ip = D.u_save.ld(i + 1, j, k), muu_ip = D.muu.ld(i + 1, j, 0);
          const R msfuy_ip = D.msfuy(i + 1, j);
          R v_jp = 0, vsv_jp = 0, muv_jp = 0, mvxi_jp = 0;
          if (D.do_y) {
            v_jp = D.v2.ld(i, j + 1, k);
            vsv_jp = D.v_save.ld(i, j + 1, k);
            muv_jp = D.muv.ld(i, j + 1, 0);
            mvxi_jp = D.msfvx_inv(i, j + 1);
          }
          if (k + 1 < nz) s2[(k + 1) * CX + lane] = A(D.ww1.ld(i, j, k + 1));
          // KMuTDiv (small_step.cpp:194-206), the expression of mut_dv
          const R fx = (u_ip + div_msf((c1h * muu_ip + c2h) * usv_ip, msfuy_ip)) - (u_k + div_msf((c1h * muu + c2h) * usv, msfuy));
          R d = R(D.rdx) * fx;
          if (D.do_y) d += R(D.rdy) * ((v_jp + (c1h * muv_jp + c2h) * vsv_jp * mvxi_jp) - (v_k + (c1h * muv + c2h) * vsv * mvxi));
          const A dv = A(D.msftx(i, j) * D.msfty(i, j) * d);
          s0[k * CX + lane] = dv;
          s1[k * CX + lane] = D.dnw[k] * dv;  // the term of the column sum, for the serial sum below
        }
        const R su = rum + u_k;
        D.ru_m(i, j, k) = last ? su / rn + div_msf((c1h * muu + c2h) * usv, msfuy) : su;
        if (D.do_y) {
          const R sv = rvm + v_k;
          D.rv_m(i, j, k) = last ? sv / rn + (c1h * muv + c2h) * vsv * mvxi : sv;
        }
      }
    __syncthreads();
    if (mass)  // while warp 0 sums the column: phase 2's inputs into L2
      CB_LOOP_W1(k, nz + 1) {
        pf_l2(&D.ph_tend(i, j, k));
        pf_l2(&D.w2(i, j, k));
        pf_l2(&D.ph_save(i, j, k));
        pf_l2(&D.ph2(i, j, k));
        pf_l2(&D.rw_tend(i, j, k));
        pf_l2(&D.a(i, j, k));
        pf_l2(&D.alpha(i, j, k));
        pf_l2(&D.gamma(i, j, k));
        if (!D.flat) pf_l2(D.phb.p + (i * D.phb.si + j * D.phb.sj + k * D.phb.sk));
        if (k < nz) {
          pf_l2(&D.c2a(i, j, k));
          pf_l2(&D.alt(i, j, k));
          pf_l2(&D.pm1(i, j, k));
          if (D.n_moist) pf_l2(&D.cqw(i, j, k));
        }
      }
    if (dyn && w0) {  // the column mass tendency: sum over k in order
      A dmdt = 0;
#pragma unroll 4
      for (int k = 0; k < nz; ++k) dmdt += s1[k * CX + lane];
      const A mtend = A(D.mu_tend.ld(i, j, 0));
      const A mu_old = A(D.mu2(i, j, 0));
      const A mu_new = mu_old + A(dts) * (dmdt + mtend);
      D.mu2(i, j, 0) = R(mu_new);
      D.mudf(i, j, 0) = R(dmdt + mtend);
      D.muts(i, j, 0) = D.mut.ld(i, j, 0) + R(mu_new);
      D.muave(i, j, 0) = R(0.5) * ((R(1) + epssm) * R(mu_new) + (R(1) - epssm) * R(mu_old));
      sc[0 * CX + lane] = dmdt;
      sc[1 * CX + lane] = mtend;
    }
    __syncthreads();
    if (dyn) {  // the decrement of the omega integral at each level
      const A dmdt = sc[0 * CX + lane], mtend = sc[1 * CX + lane];
      const A msfty = A(D.msfty(i, j));
      CB_LOOP_SH(k, nz - 1) s1[k * CX + lane] = div_msf(D.dnw[k] * (D.c1h[k] * dmdt + s0[k * CX + lane] + D.c1h[k] * mtend), msfty);
    }
    __syncthreads();
    if (dyn && w0) {  // ww'' by the running integral (ww1 of level k + 1 staged in s2[k + 1])
      A ww_full = 0;
      s2[0 * CX + lane] = 0;
#pragma unroll 4
      for (int k = 0; k < nz - 1; ++k) {
        ww_full = ww_full - s1[k * CX + lane];
        s2[(k + 1) * CX + lane] = A(R(ww_full - s2[(k + 1) * CX + lane]));
      }
      s2[nz * CX + lane] = 0;
    }
    __syncthreads();
    if (mass) {
      CB_LOOP(k, nz + 1) {  // ww'' and its time sum; theta'' (KMuTPoint), every load before the first store
        R wpp = 0, wwm = 0, ww1 = 0;
        if (dyn) {
          wpp = R(s2[k * CX + lane]);
          wwm = first ? R(0) : D.ww_m(i, j, k);
          ww1 = D.ww1.ld(i, j, k);
        }
        R tk = 0, tnew = 0;
        if (k < nz) {
          tk = D.t2(i, j, k);
          const R ttend = D.t_tend.ld(i, j, k);
          if (spec) {  // theta'' of the spec zone (update_mu_t)
            tnew = tk + dts * ttend;
          } else {
            const R u_k = D.u2.ld(i, j, k), u_ip = D.u2.ld(i + 1, j, k);
            const R ts = D.t_save.ld(i, j, k), ts_ip = D.t_save.ld(i + 1, j, k), ts_im = D.t_save.ld(i - 1, j, k);
            R v_k = 0, v_jp = 0, ts_jp = 0, ts_jm = 0;
            if (D.do_y) {
              v_k = D.v2.ld(i, j, k);
              v_jp = D.v2.ld(i, j + 1, k);
              ts_jp = D.t_save.ld(i, j + 1, k);
              ts_jm = D.t_save.ld(i, j - 1, k);
            }
            const R ts_kp = k + 1 < nz ? D.t_save.ld(i, j, k + 1) : R(0), ts_km = k >= 1 ? D.t_save.ld(i, j, k - 1) : R(0);
            const R msfty = D.msfty(i, j), msftx = D.msftx(i, j);
            R hflux = R(0.5) * R(D.rdx) * (u_ip * (ts_ip + ts) - u_k * (ts + ts_im));
            if (D.do_y) hflux += R(0.5) * R(D.rdy) * (v_jp * (ts_jp + ts) - v_k * (ts + ts_jm));
            const R tn = tk + msfty * dts * ttend;
            const R wd_kp = (k + 1 == nz) ? R(0) : R(s2[(k + 1) * CX + lane]) * (R(D.fnm[k + 1]) * ts_kp + R(D.fnp[k + 1]) * ts);
            const R wd_k = (k == 0) ? R(0) : R(s2[k * CX + lane]) * (R(D.fnm[k]) * ts + R(D.fnp[k]) * ts_km);
            tnew = tn - dts * msfty * (msftx * hflux + R(D.rdnw[k]) * (wd_kp - wd_k));
          }
        }
        if (dyn) {
          const R sw = wwm + (k == 0 ? R(0) : wpp);
          D.ww(i, j, k) = wpp;
          D.ww_m(i, j, k) = last ? sw / rn + ww1 : sw;
        }
        if (k < nz) {
          s_t2s[k * CX + lane] = double(tk);  // t_2save: kept in shared memory for advance_w
          D.t2(i, j, k) = tnew;
        }
      }
    }
    __syncthreads();
  }
  {  // phase 2
    // advance_w in double in both forms (the mixed form's fields are float; the explicit phi'' and w'' right-hand
    // sides are differences of nearly equal pressure-gradient and buoyancy terms, kept in double). For the FP64
    // form every conversion below is the identity and the operations are the reference's, in its order.
    const A dtsA = rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound, eps = D.epssm;
    const A ope = 1.0 + eps, ome = 1.0 - eps;
    auto mhA = [&](int kk, A m) { return D.c1h[kk] * m + D.c2h[kk]; };
    auto mfA = [&](int kk, A m) { return D.c1f[kk] * m + D.c2f[kk]; };
    A mut = 0, muts = 0, mav = 0, msfty = 1;
    double* s_a = cb_array(3, nz);
    double* s_al = cb_array(4, nz);
    double* s_ga = cb_array(5, nz);
    if (spec) {  // phi'' of the spec zone (LateralBC::update_ph_w, KUpdatePh :374-386)
      const R mts = D.muts(i, j, 0), mold = mts - dts * D.mu_tend.ld(i, j, 0);
      CB_LOOP(k, nz + 1) {
        const R m_old = R(D.c1f[k]) * mold + R(D.c2f[k]), m_new = R(D.c1f[k]) * mts + R(D.c2f[k]);
        D.ph2(i, j, k) = D.ph2(i, j, k) * m_old / m_new + dts * D.ph_tend.ld(i, j, k) / m_new + D.ph_save.ld(i, j, k) * (m_old / m_new - R(1));
      }
    }
    if (dyn) {
      mut = A(D.mut.ld(i, j, 0));
      muts = A(D.muts(i, j, 0));
      mav = A(D.muave(i, j, 0));
      msfty = A(D.msfty(i, j));
      CB_LOOP_SH(k, nz + 1) {  // KWRhs: R (explicit phi'') and t_2ave
        A r;
        if (k == 0 || (D.top_lid && k == nz)) {
          r = 0;
        } else {
          A rr = dtsA * (A(D.ph_tend.ld(i, j, k)) + 0.5 * k::g * (1.0 - eps) * A(D.w2(i, j, k)));
          if (k < nz) {
            auto wdwn = [&](int mm) {
              return 0.5 * (A(D.ww(i, j, mm)) + A(D.ww(i, j, mm - 1))) * D.rdnw[mm - 1] *
                     (A(D.ph_save.ld(i, j, mm)) - A(D.ph_save.ld(i, j, mm - 1)) + A(D.phb64(i, j, mm)) - A(D.phb64(i, j, mm - 1)));
            };
            rr -= dtsA * (D.fnm[k] * wdwn(k + 1) + D.fnp[k] * wdwn(k));
          }
          r = A(D.ph2(i, j, k)) + msfty * rr / mfA(k, mut);
        }
        s0[k * CX + lane] = r;
        if (k < nz) {
          const A tav = 0.5 * ((1.0 + eps) * A(D.t2(i, j, k)) + (1.0 - eps) * s_t2s[k * CX + lane]);
          s1[k * CX + lane] = (tav + D.c1h[k] * mav * k::t0) / (mhA(k, muts) * (k::t0 + A(D.t_save.ld(i, j, k))));
        }
      }
    }
    __syncthreads();
    if (dyn) {
      const A msft_inv = div_msf(1.0, msfty);
      CB_LOOP_SH(k, nz + 1) {  // KWExpl: explicit w''
        A wn;
        if (k == 0) {
          if (!D.flat) {
            const A cf1 = D.cf1, cf2 = D.cf2, cf3 = D.cf3;
            auto U = [&](int ii, int kk) { return A(D.u2.ld(ii, j, kk)); };
            auto V = [&](int jj, int kk) { return A(D.v2.ld(i, jj, kk)); };
            auto H = [&](int ii, int jj) { return A(D.ht(ii, jj)); };
            A ws = A(D.msftx(i, j)) * 0.5 * D.rdx *
                   ((H(i + 1, j) - H(i, j)) * (cf1 * U(i + 1, 0) + cf2 * U(i + 1, 1) + cf3 * U(i + 1, 2)) +
                    (H(i, j) - H(i - 1, j)) * (cf1 * U(i, 0) + cf2 * U(i, 1) + cf3 * U(i, 2)));
            if (D.do_y)
              ws = msfty * 0.5 * D.rdy *
                       ((H(i, j + 1) - H(i, j)) * (cf1 * V(j + 1, 0) + cf2 * V(j + 1, 1) + cf3 * V(j + 1, 2)) +
                        (H(i, j) - H(i, j - 1)) * (cf1 * V(j, 0) + cf2 * V(j, 1) + cf3 * V(j, 2))) +
                   ws;
            wn = ws;
          } else {
            wn = 0;
          }
        } else {
          const A r_k = s0[k * CX + lane], r_km1 = s0[(k - 1) * CX + lane];
          const A ph_k = A(D.ph2(i, j, k)), ph_km1 = A(D.ph2(i, j, k - 1));
          const A c2a_k1 = A(D.c2a.ld(i, j, k - 1)), alt_k1 = A(D.alt.ld(i, j, k - 1));
          if (k < nz) {
            const A r_kp1 = s0[(k + 1) * CX + lane], ph_kp1 = A(D.ph2(i, j, k + 1));
            const A cq1 = 1.0 / (1.0 + A(cqw_(D, i, j, k)));
            const A c2a_k = A(D.c2a.ld(i, j, k)), alt_k = A(D.alt.ld(i, j, k));
            wn = A(D.w2(i, j, k)) + dtsA * A(D.rw_tend.ld(i, j, k)) +
                 msft_inv * cq1 *
                     (0.5 * dtsA * k::g * D.rdn[k] *
                      (c2a_k * D.rdnw[k] / mhA(k, mut) * (ope * (r_kp1 - r_k) + ome * (ph_kp1 - ph_k)) -
                       c2a_k1 * D.rdnw[k - 1] / mhA(k - 1, mut) * (ope * (r_k - r_km1) + ome * (ph_k - ph_km1)))) +
                 dtsA * k::g * msft_inv *
                     (D.rdn[k] * (c2a_k * alt_k * s1[k * CX + lane] - c2a_k1 * alt_k1 * s1[(k - 1) * CX + lane]) -
                      D.c1f[k] * mav);
          } else {
            const int km = nz - 1;
            wn = A(D.w2(i, j, k)) + dtsA * A(D.rw_tend.ld(i, j, k)) +
                 msft_inv * (-0.5 * dtsA * k::g / mhA(km, mut) * (D.rdnw[km] * D.rdnw[km]) * 2.0 * c2a_k1 *
                                 (ope * (r_k - r_km1) + ome * (ph_k - ph_km1)) -
                             dtsA * k::g * (2.0 * D.rdnw[km] * c2a_k1 * alt_k1 * s1[km * CX + lane] + D.c1f[k] * mav));
            if (D.top_lid) wn = 0;
          }
        }
        s2[k * CX + lane] = wn;
        s_a[k * CX + lane] = A(D.a.ld(i, j, k));
        s_al[k * CX + lane] = A(D.alpha.ld(i, j, k));
        s_ga[k * CX + lane] = A(D.gamma.ld(i, j, k));
      }
    }
    __syncthreads();
    if (dyn && w0) {  // KWSolve: forward and backward sweeps
      A wprev = s2[0 * CX + lane];
#pragma unroll 4
      for (int k = 1; k <= nz; ++k) {
        wprev = (s2[k * CX + lane] - s_a[k * CX + lane] * wprev) * s_al[k * CX + lane];
        s2[k * CX + lane] = wprev;
      }
      A wnext = wprev;
#pragma unroll 4
      for (int k = nz - 1; k >= 1; --k) {
        wnext = s2[k * CX + lane] - s_ga[k * CX + lane] * wnext;
        s2[k * CX + lane] = wnext;
      }
    }
    __syncthreads();
    if (D.damp_opt == 3) {  // damp_opt 3: implicit Rayleigh damping of w toward 0 near the top (KWSolve :393-404)
      if (dyn) {
        const R dampmag = dts * R(D.dampcoef), hdepth = R(D.zdamp), pi = R(0x1.921fb54442d18p+1);  // 4 atan(1)
        const R htop = (D.ph_save.ld(i, j, nz) + D.phb(i, j, nz)) / R(k::g), hbot = htop - hdepth;
        CB_LOOP_SH(k, nz + 1) {
          if (k >= 1) {
            const R hk = (D.ph_save.ld(i, j, k) + D.phb(i, j, k)) / R(k::g);
            R dampwt = 0;
            if (hk >= hbot) {
              const R sn = R(cw_sin(double(R(0.5) * pi * (hk - hbot) / hdepth)));
              dampwt = dampmag * sn * sn;
            }
            s2[k * CX + lane] = A(R((R(s2[k * CX + lane]) - dampwt * mf_(D, k, R(mut)) * D.w_save.ld(i, j, k)) / (R(1) + dampwt)));
          }
        }
      }
      __syncthreads();  // the member's option: uniform over the block
    }
    // w'' and phi'' (dyn columns), then calc_p_rho of the level (every mass column, phase 3) from the new
    // phi'' of levels k and k + 1: recomputed from the shared terms here (the same expression as the store),
    // read back for the spec zone (written before the last barriers) and for the unchanged level 0
    auto ph_new = [&](int m) { return R(s0[m * CX + lane] + msfty * 0.5 * dtsA * k::g * ope * s2[m * CX + lane] / mfA(m, muts)); };
    if (mass)
      CB_LOOP(k, nz + 1) {
        R wk = 0, phk = 0, phkp = 0;
        if (dyn) {
          wk = R(s2[k * CX + lane]);
          phk = k >= 1 ? ph_new(k) : D.ph2(i, j, 0);
          if (k < nz) phkp = ph_new(k + 1);
        } else if (k < nz) {
          phk = D.ph2(i, j, k);
          phkp = D.ph2(i, j, k + 1);
        }
        if (dyn) {
          D.w2(i, j, k) = wk;
          if (k >= 1) D.ph2(i, j, k) = phk;
        }
        if (k < nz) p_rho_point_ph<true>(D, i, j, k, true, phk, phkp);
      }
  }
}

// small_step_finish (KFinish :419-444, KFinishMu :446-453) + calc_p_rho_phi (KPRhoPhi :456-477)
template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW, cb_minblocks(NW)) k_finish(const __grid_constant__ Pack<R, NM> P, int rk, int nsmall) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_STAG, i, j, ilim);
  const int nx = D.nx, ny = D.ny, nz = D.nz, nyv = D.nyv;
  const bool col = i < ilim;  // a column of the member (its faces' range)
  const bool mass = col && i < nx && j < ny;
  const R dts = R(rk == 1 ? D.dt / 3.0 : D.dt / D.n_sound);
  const R hd_dt = (rk == 3 && D.n_moist > 0) ? dts * R(nsmall) : R(0);
  if (col) {
    CB_LOOP(k, nz + 1) {  // every load of a level before its first store
      const bool has_u = j < ny && k < nz, has_v = i < nx && j < nyv && k < nz;
      const R c1h = k < nz ? R(D.c1h[k]) : R(0), c2h = k < nz ? R(D.c2h[k]) : R(0);
      R u2 = 0, usv = 0, msfuy = 0, muu = 0, mts_u0 = 0, mts_u1 = 0;
      if (has_u) {
        u2 = D.u2(i, j, k);
        usv = D.u_save.ld(i, j, k);
        msfuy = D.msfuy(i, j);
        muu = D.muu.ld(i, j, 0);
        mts_u0 = D.muts.ld(i, j, 0);
        mts_u1 = D.muts.ld(i - 1, j, 0);
      }
      R v2 = 0, vsv = 0, msfvx = 0, muv = 0, mts_v0 = 0, mts_v1 = 0;
      if (has_v) {
        v2 = D.v2(i, j, k);
        vsv = D.v_save.ld(i, j, k);
        msfvx = D.msfvx(i, j);
        muv = D.muv.ld(i, j, 0);
        mts_v0 = D.muts.ld(i, j, 0);
        mts_v1 = D.muts.ld(i, j - 1, 0);
      }
      R m = 0, mts = 0, w2 = 0, wsv = 0, msfty = 0, ph2 = 0, phsv = 0, ww = 0, ww1 = 0, t2 = 0, tsv = 0, hd = 0;
      if (mass) {
        m = D.mut.ld(i, j, 0);
        mts = D.muts.ld(i, j, 0);
        w2 = D.w2(i, j, k);
        wsv = D.w_save.ld(i, j, k);
        msfty = D.msfty(i, j);
        ph2 = D.ph2(i, j, k);
        phsv = D.ph_save.ld(i, j, k);
        ww = D.ww(i, j, k);
        ww1 = D.ww1.ld(i, j, k);
        if (k < nz) {
          t2 = D.t2(i, j, k);
          tsv = D.t_save.ld(i, j, k);
          if (hd_dt != R(0)) hd = D.hd.ld(i, j, k);
        }
      }
      if (has_u) {
        const R mus_u = R(0.5) * (mts_u0 + mts_u1);
        D.u2(i, j, k) = (msfuy * u2 + usv * (c1h * muu + c2h)) / (c1h * mus_u + c2h);
      }
      if (has_v) {
        const R mus_v = R(0.5) * (mts_v0 + mts_v1);
        D.v2(i, j, k) = (msfvx * v2 + vsv * (c1h * muv + c2h)) / (c1h * mus_v + c2h);
      }
      if (mass) {
        D.w2(i, j, k) = (msfty * w2 + wsv * (R(D.c1f[k]) * m + R(D.c2f[k]))) / (R(D.c1f[k]) * mts + R(D.c2f[k]));
        D.ph2(i, j, k) = ph2 + phsv;
        D.ww(i, j, k) = ww + ww1;
        if (k < nz)
          D.t2(i, j, k) = (t2 - (hd_dt != R(0) ? hd_dt * (c1h * m + c2h) * hd : R(0)) + tsv * (c1h * m + c2h)) / (c1h * mts + c2h);
      }
    }
    if (threadIdx.y == 0) {
      if (mass) D.mu2(i, j, 0) = D.mu2(i, j, 0) + D.mu_save(i, j, 0);
      if (j < ny) D.muus(i, j, 0) = R(0.5) * (D.muts.ld(i, j, 0) + D.muts.ld(i - 1, j, 0));
      if (i < nx && j < nyv) D.muvs(i, j, 0) = R(0.5) * (D.muts.ld(i, j, 0) + D.muts.ld(i, j - 1, 0));
    }
  }
  __syncthreads();
  if (mass) CB_LOOP(k, nz) p_rho_phi_point(D, i, j, k);
}

// DiffusionDriver::prepare with damp_opt 1 (diffusion_driver.cpp:114-130): the horizontal eddy viscosities start at
// khdif and khdif / prandtl (KIsotropicKm, km_kh.hpp:35-45); cal_dampkm (km_kh.hpp:485-567) raises them in the columns
// inside spec_bdy_width - 1 rows of specified boundaries to dampcoef cos^2(pi/2 min(depth / zdamp, 1)) ds^2 / dt,
// the depth below the top summed from the diffusion metrics 1 / rdz and 1 / rdzw of ph_2 + phb
// (compute_diff_metrics, diff_metrics.hpp:11-33), level by level from the top. The vertical viscosities it also
// raises are not read by constant-K diffusion. One thread per column (warp 0); cos: cw_cos in the FP64 form (the
// reference's CPU build takes glibc's cos, libmvec's on the lanes of its column loop), CUDA's in the mixed form.
template <class R>
__device__ __forceinline__ double damp_cos(double x) {
  if constexpr (sizeof(R) == 4) return ::cos(x);
  else return cw_cos(x);
}
template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW) k_dampkm(const __grid_constant__ Pack<R, NM> P) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_MASS, i, j, ilim);
  if (D.damp_opt != 1 || !D.diff_on) return;  // uniform over the block
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  if (threadIdx.y != 0 || i >= ilim || j >= ny) return;
  const R khm = R(D.khdif), khh = R(D.khdif / D.prandtl);
  int i0 = 0, i1 = nx, j0 = 0, j1 = ny;
  if (D.lbc) {  // specified boundaries: spec_bdy_width (5) - 1 rows keep the constants
    const int w = 5;
    i0 = i0 > w - 1 ? i0 : w - 1;
    i1 = i1 < nx - w + 1 ? i1 : nx - w + 1;
    j0 = j0 > w - 1 ? j0 : w - 1;
    j1 = j1 < ny - w + 1 ? j1 : ny - w + 1;
  }
  const bool km4 = D.km_opt == 4;  // raise k_smag's viscosities instead of the constants
  if (!(i >= i0 && i < i1 && j >= j0 && j < j1)) {
    if (!km4)
      for (int k = 0; k < nz; ++k) {
        D.xkmh(i, j, k) = khm;
        D.xkhh(i, j, k) = khh;
      }
    return;
  }
  const double piconst = 3.1415926535897932384626433, degrad = piconst / 180.0, degrad90 = degrad * 90.0;
  auto zw = [&](int k) { return (double(D.ph2.ld(i, j, k)) + D.phb64(i, j, k)) / k::g; };
  const double dx_m = D.dx / double(D.msftx(i, j)), dy_m = D.dy / double(D.msfty(i, j));
  const double ds = dx_m < dy_m ? dx_m : dy_m;
  const double kmmax = ds * ds / D.dt;
  double zkp = zw(nz), zk = zw(nz - 1), deltaz = 0.0;  // zw at levels k + 1 and k
  for (int k = nz - 1; k >= 0; --k) {
    const double zkm = k > 0 ? zw(k - 1) : 0.0;
    const double rdzw = 1.0 / (zkp - zk);
    if (k == nz - 1) {
      deltaz = 0.5 * (1.0 / rdzw);
    } else {
      const double rdz = k == 0 ? 2.0 / (zkp - zk) : 2.0 / (zkp - zkm);
      deltaz = deltaz + 1.0 / rdz;
    }
    const double ratio = deltaz / D.zdamp;
    const double tmp = ratio < 1.0 ? ratio : 1.0;
    const double c = damp_cos<R>(degrad90 * tmp);
    const R dampk = R(c * c * kmmax * D.dampcoef);
    const R bm = km4 ? D.xkmh(i, j, k) : khm, bh = km4 ? D.xkhh(i, j, k) : khh;
    D.xkmh(i, j, k) = dampk > bm ? dampk : bm;
    D.xkhh(i, j, k) = dampk > bh ? dampk : bh;
    zkp = zk;
    zk = zkm;
  }
}

// set_w_surface (KSetWSurface, rk3.cpp:173-200), fill = false
template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW) k_w_surface(const __grid_constant__ Pack<R, NM> P) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_MASS, i, j, ilim);
  if (threadIdx.y != 0 || i >= ilim) return;
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
