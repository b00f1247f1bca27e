// SPDX-License-Identifier: GPL-3.0-or-later
// Device-side data model of the dycore: one Dom per domain (a member of a batch), views in CPPWRF's
// field layout, the launch geometry shared by every kernel, and the WRF flux statement functions.
//
// Every kernel takes a Pack of members: block b of a launch belongs to member m = the last index with
// start[m] <= b, so one launch covers all members of a pack whatever their sizes (a single domain is a
// pack of one).
#pragma once

#include <cstdint>

#include "cw_pow.h"
#include "tma.cuh"

namespace cw {

constexpr int kMaxMembers = 256;
constexpr int kMaxScalars = 64;
constexpr int kQTab = 11;  // views per species in a member's scalar table: q1 q2 qn qtf qscale + 6 PD faces

template <class T>
struct V3 {  // View3 of CPPWRF (src/core/field.hpp:19-23): element (0,0,0), 32-bit strides
  T* p;
  int sj, sk;
  __device__ __forceinline__ T& operator()(int i, int j, int k) const { return p[i + j * sj + k * sk]; }
  // a load through the read-only path: only for a field no thread of the kernel writes (the compiler may
  // then move it ahead of the kernel's stores)
  __device__ __forceinline__ T ld(int i, int j, int k) const { return __ldg(p + (i + j * sj + k * sk)); }
};
template <class T>
struct VB {  // BView3 / BView2 (field.hpp:35-44): si = sj = 0 for horizontally uniform storage
  const T* p;
  int si, sj, sk;
  __device__ __forceinline__ T operator()(int i, int j, int k) const { return __ldg(p + (i * si + j * sj + k * sk)); }
  __device__ __forceinline__ T operator()(int i, int j) const { return __ldg(p + (i * si + j * sj)); }
};

// Lateral boundary slabs of one variable: 4 sides of values then 4 of tendencies, (pos, k, b) pos fastest
template <class T>
struct Slabs {
  const T* v[4];
  const T* t[4];
  int npos[4];
  int nk;
  int have;
};

template <class T>
struct Dom {
  // grid and options
  int nx, ny, nz, nyv, two_d, do_y;
  // the mass points this member computes, pi0 <= i < pi1, pj0 <= j < pj1, in the domain's indices: the whole domain,
  // or a patch of a domain decomposed over several members (cw_decomp_create), whose fields are allocated for the
  // patch and a halo of 3 and indexed with the domain's indices; the edge patches also own the faces nx / ny
  int pi0, pi1, pj0, pj1;
  int bc_x, bc_y, spec_x, spec_y;  // spec_*: specified or open in that direction (degraded orders)
  int sx, sy;                      // specified in that direction (spec zone, upstream boundary velocity)
  int open_x, open_y;              // open (radiation) in that direction; open_y is 0 in 2-D
  int lbc, flat, n_moist, n_scalars, diff_on, top_lid, w_damping, n_sound, moist_adv_opt, scalar_adv_opt;
  int dd_on;     // a DiffusionDriver is attached (diff_opt 1 or the sixth-order filter): the tendf enter the tendencies
  int diff_6th_opt;
  double diff_6th_factor;
  int damp_opt;  // 1: eddy viscosities raised near the top (xkmh, xkhh); 2: Rayleigh toward the base state; 3: implicit w
  double zdamp, dampcoef;
  int mp_physics;  // 1: Kessler after the RK3 loop (species 0, 1, 2 = qv, qc, qr)
  double mp_tend_lim;
  double dt, epssm, smdiv, emdiv, khdif, kvdif, prandtl, hup, vup, w_crit_cfl;
  double dx, dy;  // grid spacing (cal_dampkm's horizontal limit)
  double* dtbc;  // device scalar: time since the boundary data (LateralBC::dtbc), advanced on the device
  unsigned long long* cfl;  // per RK stage: the vertical and horizontal CFL maxima (bits of positive doubles)
  double rdx, rdy, cf1, cf2, cf3, cfn, cfn1;
  const double *znu, *znw, *dnw, *dn, *rdnw, *rdn, *fnm, *fnp, *c1h, *c2h, *c1f, *c2f, *u_base, *v_base;
  const double *fcx, *gcx;  // relaxation weights per row (LateralBC::set_dt)
  const double *t_base, *z_base;  // BaseState 1-D profiles (damp_opt 2's base state)
  const double *c3h, *c4h, *c3f, *c4f;  // hybrid coefficients of the dry pressure (hypsometric_opt 2)
  int hypsometric_opt;  // calc_p_rho_phi: 1 linear in the column mass, 2 log-linear in pressure
  double p_top;
  // State
  V3<T> rainnc, rainncv;  // accumulated / last-step grid-scale rain [mm] (2-D)
  V3<T> u1, u2, v1, v2, w1, w2, t1, t2, ph1, ph2, mu1, mu2, p, al, alt, php, ww, mut, muu, muv, muts, muus, muvs,
      ru, rv, rw, ru_m, rv_m, ww_m, cqu, cqv, cqw, hd;
  // Tendencies
  V3<T> ru_tend, rv_tend, rw_tend, t_tend, ph_tend, mu_tend, ru_tendf, rv_tendf, rw_tendf, t_tendf, ph_tendf;
  // BaseState
  VB<T> mub, pb, alb, t_init, qv_base, phb, ht, msftx, msfty, msfux, msfuy, msfvx, msfvy, msfvx_inv;
  VB<T> f, e, sina, cosa;  // Coriolis parameters and grid rotation
  // pb, alb, phb in double for the double parts of both forms (the FP64 form: the same arrays; the mixed form:
  // double copies, so that the equation of state's p'' = p(alpha, theta) - pb does not carry pb's float rounding)
  VB<double> pb64, alb64, phb64;
  int cor;                 // MapC::cor = BaseState::mapped || coriolis: the Coriolis terms of the u, v, w tendencies
  int mapped;              // BaseState::mapped: map factors vary; the curvature terms of u, v use their gradients
  // acoustic-step work fields (SmallStep, src/dyn/small_step.hpp:45-49)
  V3<T> u_save, v_save, w_save, t_save, ph_save, ww1, c2a, pm1, t_2save, a, alpha, gamma, mu_save, mudf, muave,
      w_rhs, t2a;
  V3<T> xkmh, xkhh;  // damp_opt 1 / km_opt 4: the horizontal eddy viscosities of momentum and heat per mass point
  int km_opt;        // 1: constant K; 4: 2-D Smagorinsky (horizontal)
  int xk_field;      // the horizontal diffusion reads xkmh / xkhh (else the constants)
  // scalars: device tables of views (q2 and q_new swap roles after each update)
  V3<T>* q1;
  V3<T>* q2;
  V3<T>* qn;
  V3<T>* qtf;
  V3<T>* qscale;
  V3<T>* qpd;  // PD face fluxes of species n: qpd[6 n + f], f = dh_x, lo_x, dh_y, lo_y, dh_z, lo_z
  // boundary slabs: U V T PH MU, then scalars (n_scalars entries)
  Slabs<T> lbc_var[5];
  Slabs<T>* lbc_q;
  // the TMA-staged scalar update: each species' tensor maps (device memory; nullptr where it does not run)
  const QMap* qmap;
  unsigned* status;  // device word of the handle: bit 0 set when a kernel's bounded wait gave up (cw_sync reports it)
};

// The kernels' view of the members. A single domain (NM = 1): its descriptor passed by value as a
// __grid_constant__ parameter, so the field descriptors are read from the constant bank (operands of the address
// arithmetic) and no store of a kernel can alias them. A batch (NM = 0, any number of members): the members'
// descriptors and block prefix sums in device memory, so one launch of each kernel covers the whole batch.
// start(kind, shape, m) is member m's first block of a launch over the index range `kind` in block shape `shape`.
constexpr int kNumKinds = 8;
constexpr int kNumShapes = 3;  // point-kernel block shapes (autotuned per kernel): 128 x 1, 64 x 2, 32 x 4
template <class R, int NM>
struct Pack {
  Dom<R> d[NM];
  int n;
  int start_[kNumKinds][kNumShapes][NM + 1];
  __device__ __forceinline__ int start(int kind, int shape, int m) const { return start_[kind][shape][m]; }
};
template <class R>
struct Pack<R, 0> {
  const Dom<R>* __restrict__ d;  // n descriptors (device memory, written before the launch)
  int n;
  // the block starts in the parameter (the constant bank: a block's binary search over them is uniform and
  // needs no global load), 24.1 KB for the largest batch, within the 32 KB parameter limit
  int start_[kNumKinds][kNumShapes][kMaxMembers + 1];
  __device__ __forceinline__ int start(int kind, int shape, int m) const { return start_[kind][shape][m]; }
};
template <class R, int NM>
__device__ __forceinline__ int member_of(const Pack<R, NM>& P, int kind, int shape, int b) {
  if constexpr (NM == 1) {
    return 0;
  } else {
    int lo = 0, hi = P.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.start(kind, shape, mid) <= b) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
}

// x / m for a map factor m. In IEEE arithmetic x / 1 is x exactly, so the division is skipped when m == 1 with the
// same bits as its result: an unmapped domain's map factors are all 1, and its divisions by them cost a compare.
template <class X>
__device__ __forceinline__ X div_msf(X x, X m) {
  return m == X(1) ? x : x / m;
}

// Block geometry of the two launch shapes. Point kernels: PX threads along i, blockIdx over (i-tiles, j, k)
// of a member. Column kernels ("column blocks"): CX columns along i (the lanes of a warp, coalesced) x CNW
// warps; the pointwise work of the columns' levels is split over the warps, the vertical recurrences run
// on warp 0 (one lane per column) through shared memory. blockIdx over (i-tiles, j).
constexpr int PX = 128, PY = 1;
// point-kernel shape s: shape_x(s) points along i times shape_y(s) rows along j in one block of PX threads
__host__ __device__ constexpr int shape_x(int s) { return s == 0 ? PX : (s == 1 ? PX / 2 : PX / 4); }
__host__ __device__ constexpr int shape_y(int s) { return PX / shape_x(s); }
constexpr int CX = 32, CNW = 8;
// the column kernels' warp counts the autotuner chooses from (shape s: cb_warps(s) warps; the fewest blocks per SM
// their launch bound asks for keeps 3 x 256, 2 x 512 and 6 x 128 threads resident)
__host__ __device__ constexpr int cb_warps(int s) { return s == 0 ? CNW : (s == 1 ? 2 * CNW : CNW / 2); }
__host__ __device__ constexpr int cb_minblocks(int nw) { return nw == CNW ? 3 : (nw > CNW ? 2 : 6); }
constexpr int kCbArrays = 6;  // shared-memory level arrays of the acoustic column block: kCbArrays x (nz + 2) x CX doubles
__host__ __device__ __forceinline__ int cdiv(int a, int b) { return (a + b - 1) / b; }

// ---- WRF flux statement functions (src/dyn/kernels_common.hpp:11-105) ----
template <class R>
__device__ __forceinline__ R sgn1(R a) {
  return a >= R(0) ? R(1) : R(-1);
}
// x / C for the statement functions' constants C = 60, 12: in the FP64 form the correctly rounded quotient without a
// division (cw_div_const: one multiply and two FMAs, bit-identical to the IEEE division); in the mixed form the
// IEEE float division
template <int C>
__device__ __forceinline__ double div_c(double x) {
  return cw_div_const(x, double(C), 1.0 / double(C));
}
template <int C>
__device__ __forceinline__ float div_c(float x) {
  return x / float(C);
}
template <class R>
__device__ __forceinline__ R flux5(R qm3, R qm2, R qm1, R q0, R qp1, R qp2, R ua, R up) {
  return div_c<60>(R(37) * (q0 + qm1) - R(8) * (qp1 + qm2) + (qp2 + qm3)) -
         div_c<60>(up * sgn1(ua) * ((qp2 - qm3) - R(5) * (qp1 - qm2) + R(10) * (q0 - qm1)));
}
template <class R>
__device__ __forceinline__ R flux3(R qm2, R qm1, R q0, R qp1, R ua, R up) {
  return div_c<12>(R(7) * (q0 + qm1) - (qp1 + qm2)) + div_c<12>(up * sgn1(ua) * ((qp1 - qm2) - R(3) * (q0 - qm1)));
}
template <class R>
__device__ __forceinline__ R flux5_pd(R qm3, R qm2, R qm1, R q0, R qp1, R qp2, R ua, R up) {
  const R f6 = (R(37.) / R(60.)) * (q0 + qm1) - (R(2.) / R(15.)) * (qp1 + qm2) + (R(1.) / R(60.)) * (qp2 + qm3);
  return f6 - up * sgn1(ua) * (R(1.) / R(60.)) * ((qp2 - qm3) - R(5.) * (qp1 - qm2) + R(10.) * (q0 - qm1));
}
template <class R>
__device__ __forceinline__ R flux3_pd(R qm2, R qm1, R q0, R qp1, R ua, R up) {
  const R f4 = (R(7.) / R(12.)) * (q0 + qm1) - (R(1.) / R(12.)) * (qp1 + qm2);
  return f4 + up * sgn1(ua) * (R(1.) / R(12.)) * ((qp1 - qm2) - R(3.) * (q0 - qm1));
}
__device__ __forceinline__ int ord_face(int f, int n, int on) {
  if (!on) return 5;
  if (f <= 1 || f >= n - 1) return 2;
  if (f == 2 || f == n - 2) return 3;
  return 5;
}
__device__ __forceinline__ int ord_mass(int f, int n, int on) {
  if (!on) return 5;
  if (f <= 1 || f >= n) return 2;
  if (f == 2 || f == n - 1) return 3;
  return 5;
}
template <class R>
__device__ __forceinline__ R flux_upwind(R qm1, R q0, R cr) {
  const R a = cr < R(0) ? -cr : cr;
  const R lo = cr + a, hi = cr - a;
  return R(0.5) * (lo < R(1) ? lo : R(1)) * qm1 + R(0.5) * (hi > R(-1) ? hi : R(-1)) * q0;
}

// physical constants (src/core/constants.hpp:4-18)
namespace k {
constexpr double g = 9.81;
constexpr double r_d = 287.0;
constexpr double cp = 7.0 * r_d / 2.0;
constexpr double cpovcv = cp / (cp - r_d);
constexpr double p1000mb = 100000.0;
constexpr double t0 = 300.0;
constexpr double reradius = 1. / 6370.0e03;
constexpr double cb = 25.;  // phase speed of the open (radiative) lateral boundaries
}  // namespace k

// ---- halo fill descriptors (HaloLine, src/core/halo.cpp:52-88) ----
// One descriptor per field of a fill point; a launch covers every field of every member. Each thread
// writes one halo cell with its final value, composed from interior sources (x then y, as fill_impl
// orders the passes). The only in-place update, the wall face of an OddFace field (muu on symmetric
// x walls), is done by a second launch (pass 1) after every y cell has read the unflipped face.
struct HaloField {
  void* p;       // element (0,0,0) (double or float)
  void* ind;     // non-null: a device V3 whose .p is read at run time (scalars that swap buffers)
  int sj, sk;
  int lnx, lny, nk;  // logical extents (staggered) and levels
  int wi0, wi1, wj0, wj1;
  int gnx, gny;      // the member's mass-point extents
  unsigned char periodic_x, periodic_y, flat_x, flat_y, two_d, face_x, face_y, odd_x, odd_y, oddface_x, is_float,
      pad;
  int xj0, xj1;              // the x pass's rows: the window's rows inside the domain
  long long ncell_x, ncell;  // x-pass cells, all cells
};
// A decomposed domain's exchange (the halo exchange of core/halo.cpp:120-129 / tiles.hpp:6-12): the rectangle
// i0 <= i < i1, j0 <= j < j1 (all nk levels) of a field that a patch holds in its halo and another patch owns,
// copied from the owner's allocation into the patch's at the same domain indices. src / dst: element (0, 0, 0),
// or the start of a packed buffer with soff / doff the index of element (0, 0, 0) in it; src_ind / dst_ind (scalars
// whose buffers swap): a device V3 whose .p is read at run time instead.
struct XchgBox {
  const void* src;
  const void* src_ind;
  void* dst;
  const void* dst_ind;
  int ssj, ssk, dsj, dsk;
  long long soff, doff;  // element offsets added to the source / destination index (a packed buffer's box)
  int i0, i1, j0, j1, nk;
  int is_float;
  long long ncell;
};
// The fields of one launch, passed by value as a __grid_constant__ parameter (no descriptor is read from
// global memory). Two capacities: a fill point of a single domain fits the small one; a batch's fill point
// uses the large one (160 x 88 B of descriptors, inside the 32 KB parameter limit), in chunks when larger.
constexpr int kHaloSmall = 16, kHaloLarge = 160;
template <int NF>
struct HaloChunk {
  HaloField f[NF];
  unsigned start[NF + 1];  // prefix sums of the fields' cell counts
  int nf;
  int has_oddface;
};

}  // namespace cw
