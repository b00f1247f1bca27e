// SPDX-License-Identifier: GPL-3.0-or-later
// Microphysics after the RK3 loop, mp_physics = 1 (PhysicsCoupling::step, src/dyn/physics_coupling.cpp:262-456):
// moist_physics_prep_em (KPrep :42-60), the Kessler warm-rain scheme (src/phys/mp_kessler/kessler.hpp:47-159) on
// the columns outside the spec zone, and moist_physics_finish_em (KFinish :63-76), fused into one column-block
// kernel. Species 0, 1, 2 are qv, qc, qr.
//
// Phase 1 (all warps, levels split): the terms of the rain sedimentation per level -- qr, rho, the terminal
// velocity and its density factor, 1/dz at w and mass levels -- staged in shared memory. Phase 2 (warp 0, one lane
// per column): the sedimentation, in the reference's order (its time splitting depends on the column's Courant
// number), accumulating the surface rain. Phase 3 (all warps, levels split): production, evaporation and the
// finish (new theta_m and the heating rate h_diabatic) of each level, which are pointwise.
//
// pow and exp: cw_pow / cw_exp in the FP64 form (the reference's CPU build takes glibc's, libmvec's on the lanes
// of its vectorised loops), CUDA's in the mixed form. Both forms compute in double.
#pragma once

#include "kernels_cb.cuh"

namespace cw {

// the sedimentation's time splitting stops after this many sub-steps in a column (a Courant number of ~50000;
// physical columns take a few): a bound for columns holding non-finite or absurd values
constexpr int kMaxFall = 1 << 16;

template <class R>
__device__ __forceinline__ double mp_pow(double a, double b) {
  if constexpr (sizeof(R) == 4) return ::pow(a, b);
  else return cw_pow(a, b);
}
template <class R>
__device__ __forceinline__ double mp_exp(double a) {
  if constexpr (sizeof(R) == 4) return ::exp(a);
  else return cw_exp(a);
}
__device__ __forceinline__ double mp_max(double a, double b) { return a < b ? b : a; }  // std::max
__device__ __forceinline__ double mp_min(double a, double b) { return b < a ? b : a; }  // std::min
// nfall = max(1, int(round(0.5 + crmax / 0.75))) with the x86 conversion of the reference's CPU build (NaN and
// values beyond the int range convert to INT_MIN, so nfall = 1)
__device__ __forceinline__ int mp_fall(double crmax) {
  const double r = round(0.5 + crmax / 0.75);
  const int n = (r == r && r < 2147483648.0) ? int(r) : -2147483647 - 1;
  return 1 < n ? n : 1;
}

template <class R, int NM, int NW = CNW>
__global__ void __launch_bounds__(CX * NW) k_kessler(const __grid_constant__ Pack<R, NM> P) {
  int i, j, ilim;
  const Dom<R>& D = cb_member(P, RG_COLS_MASS, i, j, ilim);
  if (D.mp_physics != 1) return;  // uniform over the block
  const int nx = D.nx, ny = D.ny, nz = D.nz, lane = threadIdx.x;
  const bool col = i < ilim && j < ny;
  const int sx = D.bc_x == CW_BC_SPECIFIED ? 1 : 0, sy = D.bc_y == CW_BC_SPECIFIED ? 1 : 0;
  const bool mp = col && i >= sx && i < nx - sx && j >= sy && j < ny - sy;
  constexpr double t0 = 300.0, g = 9.81, rvrd = 461.6 / 287.0, rcp = 287.0 / (7.0 * 287.0 / 2.0);
  constexpr double xlv = 2.5e6, cp = 7.0 * 287.0 / 2.0, ep2 = 287.0 / 461.6, svp1 = 0.6112, svp2 = 17.67,
                   svp3 = 29.65, svpt0 = 273.15, rhowater = 1000.0;
  const double dt = D.dt;
  const V3<R> qv = D.q2[0], qc = D.q2[1], qr = D.q2[2];
  double* s_prodk = cb_array(0, nz);
  double* s_rho = cb_array(1, nz);
  double* s_vt = cb_array(2, nz);
  double* s_vtden = cb_array(3, nz);
  double* s_rdzw = cb_array(4, nz);
  double* s_rdzk = cb_array(5, nz);
  auto zw = [&](int k) { return (double(D.ph2(i, j, k)) + D.phb64(i, j, k)) / g; };
  auto rho_at = [&](int k) { return 1.0 / (double(D.al(i, j, k)) + D.alb64(i, j, k)); };
  if (mp) {
    const double rho0 = rho_at(0);
    CB_LOOP(k, nz) {  // kessler.hpp:103-117
      const double q = double(qr(i, j, k)), rho = rho_at(k);
      const double z0 = zw(k), z1 = zw(k + 1);
      const double qrr = mp_max(0.0, q * 0.001 * rho);
      const double vtden = sqrt(rho0 / rho);
      s_prodk[k * CX + lane] = q;
      s_rho[k * CX + lane] = rho;
      s_vtden[k * CX + lane] = vtden;
      s_vt[k * CX + lane] = 36.34 * mp_pow<R>(qrr, 0.1364) * vtden;
      s_rdzw[k * CX + lane] = 1.0 / (z1 - z0);
      // 1 / (z(k+1) - z(k)) of the mass-level heights z = (zw(k) + zw(k+1)) / 2; the top level repeats the last
      if (k < nz - 1) s_rdzk[k * CX + lane] = 1.0 / (0.5 * (z1 + zw(k + 2)) - 0.5 * (z0 + z1));
      else s_rdzk[k * CX + lane] = 1.0 / (0.5 * (z0 + z1) - 0.5 * (zw(nz - 2) + z0));
    }
  }
  __syncthreads();
  if (mp && threadIdx.y == 0) {  // sedimentation (kessler.hpp:118-165), serial in k
    auto A = [&](const double* a, int k) -> double& { return const_cast<double*>(a)[k * CX + lane]; };
    double crmax = 0;
    for (int k = 0; k < nz; ++k) crmax = mp_max(A(s_vt, k) * dt * A(s_rdzw, k), crmax);
    int nfall = mp_fall(crmax);
    double dtfall = dt / nfall, time_sediment = dt;
    for (int n = 0; nfall > 0 && n < kMaxFall; ++n) {
      time_sediment = time_sediment - dtfall;
      const double ppt = A(s_rho, 0) * A(s_prodk, 0) * A(s_vt, 0) * dtfall / rhowater;
      D.rainncv(i, j, 0) = R(ppt * 1000.0);
      D.rainnc(i, j, 0) = R(double(D.rainnc(i, j, 0)) + ppt * 1000.0);
      for (int k = 0; k < nz - 1; ++k) {
        const double factor = dtfall * A(s_rdzk, k) / A(s_rho, k);
        A(s_prodk, k) = A(s_prodk, k) - factor * (A(s_rho, k) * A(s_prodk, k) * A(s_vt, k) -
                                                  A(s_rho, k + 1) * A(s_prodk, k + 1) * A(s_vt, k + 1));
      }
      const double factor_top = dtfall * A(s_rdzk, nz - 1);
      A(s_prodk, nz - 1) = A(s_prodk, nz - 1) - factor_top * A(s_prodk, nz - 1) * A(s_vt, nz - 1);
      if (nfall > 1) {
        nfall = nfall - 1;
        crmax = 0;
        for (int k = 0; k < nz; ++k) {
          const double qrr = mp_max(0.0, A(s_prodk, k) * 0.001 * A(s_rho, k));
          A(s_vt, k) = 36.34 * mp_pow<R>(qrr, 0.1364) * A(s_vtden, k);
          crmax = mp_max(A(s_vt, k) * time_sediment * A(s_rdzw, k), crmax);
        }
        const int nfall_new = mp_fall(crmax);
        if (nfall_new != nfall) {
          nfall = nfall_new;
          dtfall = time_sediment / nfall;
        }
      } else {
        nfall = 0;  // prod = prodk: read from s_prodk below
      }
    }
  }
  __syncthreads();
  if (!col) return;
  const double f5 = svp2 * (svpt0 - svp3) * xlv / cp;
  const double lim = D.mp_tend_lim;
  CB_LOOP(k, nz) {
    // KPrep: dry theta (th_phy, also the old value kept in h_diabatic) and the old qv
    const double q_old = double(qv(i, j, k));
    const double th_old = (double(D.t2(i, j, k)) + t0) / (1.0 + rvrd * q_old);
    double th = th_old, q = q_old;
    if (mp) {  // production of rain, condensation, evaporation (kessler.hpp:168-197)
      const double c1 = 0.001, c2 = 0.001, c3 = 2.2, c4 = 0.875;
      const double pii = mp_pow<R>((double(D.p(i, j, k)) + D.pb64(i, j, k)) / 100000.0, rcp);
      double qck = double(qc(i, j, k)), qrk = double(qr(i, j, k));
      const double prodk = s_prodk[k * CX + lane];
      const double factorn = 1.0 / (1.0 + c3 * dt * mp_pow<R>(mp_max(0.0, qrk), c4));
      const double qrprod = qck * (1.0 - factorn) + factorn * c1 * dt * mp_max(qck - c2, 0.0);
      const double rcgs = 0.001 * s_rho[k * CX + lane];
      qck = mp_max(qck - qrprod, 0.0);
      qrk = (qrk + prodk - qrk);
      qrk = mp_max(qrk + qrprod, 0.0);
      const double temp = pii * th;
      const double pressure = 1.000e+05 * mp_pow<R>(pii, 1004.0 / 287.0);
      const double gam = 2.5e+06 / (1004.0 * pii);
      const double es = 1000.0 * svp1 * mp_exp<R>(svp2 * (temp - svpt0) / (temp - svp3));
      const double qvs = ep2 * es / (pressure - es);
      const double prod = (q - qvs) / (1.0 + pressure / (pressure - es) * qvs * f5 / ((temp - svp3) * (temp - svp3)));
      const double dim_qvs_qv = mp_max(0.0, qvs - q);
      const double rq = rcgs * qrk;
      const double ern_num = (1.6 + 124.9 * mp_pow<R>(rq, 0.2046)) * mp_pow<R>(rq, 0.525);
      const double ern_den = 2.55e8 / (pressure * qvs) + 5.4e5;
      const double ern_term1 = dt * (ern_num / ern_den) * (dim_qvs_qv / (rcgs * qvs));
      const double ern_term2 = mp_max(-prod - qck, 0.0);
      const double ern = mp_min(ern_term1, mp_min(ern_term2, qrk));
      const double product = mp_max(prod, -qck);
      th = th + gam * (product - ern);
      q = mp_max(q - product + ern, 0.0);
      qck = qck + product;
      qrk = qrk - ern;
      qv(i, j, k) = R(q);
      qc(i, j, k) = R(qck);
      qr(i, j, k) = R(qrk);
    }
    // KFinish: the new theta_m - t0 and the heating rate, mp_tend_lim bounding the change
    double mpten = th - th_old;
    mpten = mpten < lim * dt ? mpten : lim * dt;
    mpten = mpten > -lim * dt ? mpten : -lim * dt;
    const double qvten = q - q_old;
    D.t2(i, j, k) = R(th_old * (1.0 + rvrd * q_old) + mpten * (1.0 + rvrd * q) + rvrd * qvten * th - t0);
    D.hd(i, j, k) = R((mpten * (1.0 + rvrd * q) + rvrd * qvten * th) / dt);
  }
}

}  // namespace cw
