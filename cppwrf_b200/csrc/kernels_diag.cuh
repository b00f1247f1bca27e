// SPDX-License-Identifier: GPL-3.0-or-later
// Domain diagnostics on the device: the diag.csv row of dyn::Diagnostics::compute
// (src/dyn/diagnostics.cpp:56-80, functors :18-51).
//
// The sums are reduced in the reference CPU build's order (Reducer::run, src/core/backend.hpp:836-860): per
// level k one running sum from 0.0 over j (outer) and i (inner), the levels then folded in order on the host,
// so the FP64 result is the CPU build's to the bit. One block per (level, quantity): its threads evaluate a
// chunk of the level's points into shared memory and thread 0 adds the chunk in index order. The maxima do not
// depend on the order (no NaN reaches them: absnan maps NaN and Inf to +Inf) and are reduced across the block.
#pragma once

#include "dycore.cuh"

namespace cw {

constexpr int kDiagThreads = 256;
constexpr int kDiagChunk = 4 * kDiagThreads;
// per-level partials: maxima, then sums; part[q * (nz + 1) + k]
enum { DG_MAX_U, DG_MAX_V, DG_MAX_W, DG_MAX_THP, DG_MAX_THM, DG_MAX_Q, DG_NMAX };
enum { DG_SUM_THETA = DG_NMAX, DG_SUM_ENERGY, DG_SUM_MASS, DG_NPART };

struct DiagConst {  // src/core/constants.hpp:5-14, folded on the host
  double rvovrd, rcp, cv;
};

__device__ __forceinline__ double dg_inf() { return __longlong_as_double(0x7ff0000000000000LL); }
// NaN / Inf -> +Inf so that the maximum exposes it (diagnostics.cpp:20-22)
__device__ __forceinline__ double dg_absnan(double v) { return (v != v || v - v != 0.0) ? dg_inf() : (v < 0 ? -v : v); }

// FThp (diagnostics.cpp:24-32): dry theta' (theta = theta_m / (1 + rvovrd qv) with moist species)
template <class R>
__device__ __forceinline__ double dg_thp(const Dom<R>& D, const DiagConst& c, int i, int j, int k, double sign) {
  double th = double(D.t2.ld(i, j, k));
  if (D.n_moist > 0) th = (th + 300.0) / (1.0 + c.rvovrd * double(D.q2[0].ld(i, j, k))) - 300.0;
  const double v = th - double(D.t_init(i, j, k));
  return v != v ? dg_inf() : sign * v;
}

// FThetaMass (diagnostics.cpp:34-40)
template <class R>
__device__ __forceinline__ double dg_theta_mass(const Dom<R>& D, int i, int j, int k) {
  const double m = D.c1h[k] * (double(D.mu2.ld(i, j, 0)) + double(D.mub(i, j))) + D.c2h[k];
  return -D.dnw[k] * m * (double(D.t2.ld(i, j, k)) + 300.0);
}

// FEnergy (diagnostics.cpp:41-51): kinetic + c_v T + geopotential of the dry air column mass
template <class R>
__device__ __forceinline__ double dg_energy(const Dom<R>& D, const DiagConst& c, int i, int j, int k) {
  const double m = D.c1h[k] * (double(D.mu2.ld(i, j, 0)) + double(D.mub(i, j))) + D.c2h[k];
  const double uc = 0.5 * (double(D.u2.ld(i, j, k)) + double(D.u2.ld(i + 1, j, k)));
  const double vc = 0.5 * (double(D.v2.ld(i, j, k)) + double(D.v2.ld(i, j + 1, k)));
  const double wc = 0.5 * (double(D.w2.ld(i, j, k)) + double(D.w2.ld(i, j, k + 1)));
  const double T = (double(D.t2.ld(i, j, k)) + 300.0) * cw_pow((double(D.p.ld(i, j, k)) + D.pb64(i, j, k)) / 100000.0, c.rcp);
  const double phm = 0.5 * (double(D.ph2.ld(i, j, k)) + double(D.ph2.ld(i, j, k + 1)) + D.phb64(i, j, k) +
                            D.phb64(i, j, k + 1));
  return -D.dnw[k] * m * (0.5 * (uc * uc + vc * vc + wc * wc) + c.cv * T + phm);
}

__device__ __forceinline__ double dg_warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// grid (nz + 1, 4): blockIdx.y = 0 the maxima of level k, 1 the theta-mass sum, 2 the energy sum, 3 the dry
// mass (level 0 only)
template <class R>
__global__ void __launch_bounds__(kDiagThreads) k_diag(const __grid_constant__ Dom<R> D, const DiagConst c,
                                                       double* __restrict__ part) {
  const int k = blockIdx.x, task = blockIdx.y, t = threadIdx.x;
  const int nx = D.nx, ny = D.ny, nz = D.nz, K1 = nz + 1;
  if (task == 0) {
    double acc[DG_NMAX];
    for (int q = 0; q < DG_NMAX; ++q) acc[q] = -1e308;
    auto upd = [](double& a, double v) { a = v > a ? v : a; };
    if (k < nz) {
      for (int p = t; p < (nx + 1) * ny; p += kDiagThreads) upd(acc[DG_MAX_U], dg_absnan(double(D.u2.ld(p % (nx + 1), p / (nx + 1), k))));
      for (int p = t; p < nx * D.nyv; p += kDiagThreads) upd(acc[DG_MAX_V], dg_absnan(double(D.v2.ld(p % nx, p / nx, k))));
      for (int p = t; p < nx * ny; p += kDiagThreads) {
        const int i = p % nx, j = p / nx;
        upd(acc[DG_MAX_THP], dg_thp(D, c, i, j, k, 1.0));
        upd(acc[DG_MAX_THM], dg_thp(D, c, i, j, k, -1.0));
      }
      for (int n = 0; n < D.n_scalars; ++n) {
        const V3<R> q = D.q2[n];
        for (int p = t; p < nx * ny; p += kDiagThreads) upd(acc[DG_MAX_Q], dg_absnan(double(q.ld(p % nx, p / nx, k))));
      }
    }
    for (int p = t; p < nx * ny; p += kDiagThreads) upd(acc[DG_MAX_W], dg_absnan(double(D.w2.ld(p % nx, p / nx, k))));
    __shared__ double red[kDiagThreads / 32][DG_NMAX];
    for (int q = 0; q < DG_NMAX; ++q) {
      const double v = dg_warp_max(acc[q]);
      if ((t & 31) == 0) red[t >> 5][q] = v;
    }
    __syncthreads();
    if (t < DG_NMAX) {
      double v = -1e308;
      for (int w = 0; w < kDiagThreads / 32; ++w) upd(v, red[w][t]);
      part[t * K1 + k] = v;
    }
    return;
  }
  const int q = task == 1 ? DG_SUM_THETA : (task == 2 ? DG_SUM_ENERGY : DG_SUM_MASS);
  if ((task < 3 && k >= nz) || (task == 3 && k > 0)) {
    if (t == 0) part[q * K1 + k] = 0.0;
    return;
  }
  __shared__ double buf[kDiagChunk];
  const int n = nx * ny;
  double acc = 0.0;
  for (int base = 0; base < n; base += kDiagChunk) {
    for (int r = 0; r < kDiagChunk / kDiagThreads; ++r) {
      const int l = r * kDiagThreads + t, p = base + l;
      if (p < n) {
        const int i = p % nx, j = p / nx;
        buf[l] = task == 1 ? dg_theta_mass(D, i, j, k)
                           : (task == 2 ? dg_energy(D, c, i, j, k) : double(D.mu2.ld(i, j, 0)) + double(D.mub(i, j)));
      }
    }
    __syncthreads();
    if (t == 0) {
      const int m = n - base < kDiagChunk ? n - base : kDiagChunk;
      for (int l = 0; l < m; ++l) acc = acc + buf[l];
    }
    __syncthreads();
  }
  if (t == 0) part[q * K1 + k] = acc;
}

}  // namespace cw
