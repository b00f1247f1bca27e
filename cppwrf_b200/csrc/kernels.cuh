// SPDX-License-Identifier: GPL-3.0-or-later
// The dycore's kernels, templated on the arithmetic type R (double: the plain FP64 form, compiled with
// --fmad=false so every expression rounds exactly as the reference's CPU build; float: the bulk of the
// mixed form, whose column sums, tridiagonal solve and p'' integration stay in double).
//
// Each point formula restates the reference functor named beside it (src/dyn/*.cpp of CPPWRF) with the
// same statement and summation order. The launch structure is this library's own: per RK stage one
// column kernel for rk_step_prep, one point kernel for all five rk_tendency fields, one column kernel
// for small_step_prep + calc_p_rho + calc_coef_w; per acoustic substep one point kernel (advance_uv)
// and one column kernel (advance_mu_t + sumflux + advance_w + calc_p_rho); one column kernel for
// small_step_finish + calc_p_rho_phi; halo refreshes at the reference's refresh points, batched.
#pragma once

#include "dycore.cuh"

namespace cw {

// ------------------------------------------------------------------ launch geometry
enum RangeKind {
  RG_STAG = 0,    // (i, j, k) in [0, nx+1) x [0, nyv) x [0, nz+1)
  RG_MASS = 1,    // [0, nx) x [0, ny) x [0, nz)
  RG_COLS_STAG,   // columns [0, nx+1) x [0, nyv)
  RG_COLS_MASS,   // columns [0, nx) x [0, ny)
  RG_RING,        // boundary ring b = 0: pos in [0, max(nx, ny)+1), k in [0, nz+1), 4 sides
  RG_MASS_W,      // [0, nx) x [0, ny) x [0, nz+1)
  RG_FACES,       // as RG_STAG; in a patch, the faces of its cells up to the face after its last cell
  RG_TILES,       // as RG_MASS, in blocks of kQTx x kQTy columns and q_chunk(shape) levels (the TMA-staged scalars)
};
// The TMA-staged scalar update's block: a tile of kQTx x kQTy columns and a chunk of levels, one thread per point
constexpr int kQTx = 32, kQTy = 4;
__host__ __device__ constexpr int q_chunk(int shape) { return shape == 0 ? 2 : (shape == 1 ? 1 : 4); }
struct Range {
  int i0, i1, j0, j1, k0, k1;
};
// A member's points of an index range. The whole domain: the range as above. A patch (pi0 <= i < pi1,
// pj0 <= j < pj1 of the domain's mass points): the points it owns -- its cells, the faces between them and, at the
// domain's east / north edge, the faces nx / ny -- except RG_FACES, which also takes the face after its last cell
// (owned by the next patch; a kernel of face fluxes computes it again from the values around it). The ring is not
// clipped: its kernel keeps the points the member owns.
__host__ __device__ __forceinline__ Range range_of(int kind, int nx, int ny, int nz, int nyv, int pi0, int pi1, int pj0,
                                                   int pj1) {
  const int iu = pi1 == nx ? nx + 1 : pi1, jv = pj1 == ny ? nyv : pj1;  // owned faces end
  const int jf = nyv > ny ? pj1 + 1 : pj1;                               // RG_FACES: one face more (3-D)
  switch (kind) {
    case RG_STAG: return {pi0, iu, pj0, jv, 0, nz + 1};
    case RG_MASS: return {pi0, pi1, pj0, pj1, 0, nz};
    case RG_COLS_STAG: return {pi0, iu, pj0, jv, 0, 1};
    case RG_COLS_MASS: return {pi0, pi1, pj0, pj1, 0, 1};
    case RG_RING: return {0, (nx > ny ? nx : ny) + 1, 0, nz + 1, 0, 4};
    case RG_FACES: return {pi0, pi1 + 1, pj0, jf, 0, nz + 1};
    case RG_TILES: return {pi0, pi1, pj0, pj1, 0, nz};
    default: return {pi0, pi1, pj0, pj1, 0, nz + 1};
  }
}
template <class R>
__host__ __device__ __forceinline__ Range range_of(int kind, const Dom<R>& D) {
  return range_of(kind, D.nx, D.ny, D.nz, D.nyv, D.pi0, D.pi1, D.pj0, D.pj1);
}
__host__ __device__ __forceinline__ bool is_column(int kind) { return kind == RG_COLS_STAG || kind == RG_COLS_MASS; }
__host__ __device__ __forceinline__ int blocks_of(const Range& r, int kind, int shape = 0) {
  if (is_column(kind)) return cdiv(r.i1 - r.i0, CX) * (r.j1 - r.j0) * (r.k1 - r.k0);
  if (kind == RG_TILES) return cdiv(r.i1 - r.i0, kQTx) * cdiv(r.j1 - r.j0, kQTy) * cdiv(r.k1 - r.k0, q_chunk(shape));
  return cdiv(r.i1 - r.i0, shape_x(shape)) * cdiv(r.j1 - r.j0, shape_y(shape)) * (r.k1 - r.k0);
}
// thread -> (member, i, j, k) of a point kernel launched with block shape SH; false past the range (the range in rg)
template <int SH, class R, int NM>
__device__ __forceinline__ bool thread_index(const Pack<R, NM>& P, int kind, const Dom<R>*& Dp, int& i, int& j, int& k,
                                             Range& r) {
  constexpr int sx = shape_x(SH), sy = shape_y(SH);
  const int b = blockIdx.x;
  const int m = member_of(P, kind, SH, b);
  const Dom<R>& D = P.d[m];
  Dp = &D;
  r = range_of(kind, D);
  const int bx = cdiv(r.i1 - r.i0, sx), by = cdiv(r.j1 - r.j0, sy);
  int local = b - P.start(kind, SH, m);
  const int bi = local % bx;
  local /= bx;
  const int bj = local % by;
  k = r.k0 + local / by;
  i = r.i0 + bi * sx + int(threadIdx.x) % sx;
  j = r.j0 + bj * sy + int(threadIdx.x) / sx;
  return i < r.i1 && j < r.j1;
}
template <int SH, class R, int NM>
__device__ __forceinline__ bool thread_index(const Pack<R, NM>& P, int kind, const Dom<R>*& Dp, int& i, int& j, int& k) {
  Range r;
  return thread_index<SH>(P, kind, Dp, i, j, k, r);
}

// ------------------------------------------------------------------ copies and halos
struct CopyDesc {
  void* dst;
  const void* src;               // nullptr (and src_ind nullptr): write zeros
  const void* const* src_ind;    // non-null: the source is *src_ind - ind_offset elements (a swapped buffer)
  long long n;                   // elements
  int is_float;
  long long ind_offset;
};
static __global__ void k_copy(const CopyDesc* __restrict__ d, int nd, const long long* __restrict__ start) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= start[nd]) return;
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const long long e = t - start[lo];
  const CopyDesc& c = d[lo];
  if (c.is_float) {
    const float* src = c.src_ind ? static_cast<const float*>(*c.src_ind) - c.ind_offset : static_cast<const float*>(c.src);
    static_cast<float*>(c.dst)[e] = src ? src[e] : 0.0f;
  } else {
    const double* src = c.src_ind ? static_cast<const double*>(*c.src_ind) - c.ind_offset : static_cast<const double*>(c.src);
    static_cast<double*>(c.dst)[e] = src ? src[e] : 0.0;
  }
}

// HaloLine's source index of halo position i along a direction of n mass points (-1: keep in place)
__device__ __forceinline__ int halo_src(int i, int n, int face, int periodic, int flat) {
  if (flat) {
    const int last = face ? n : n - 1;
    return i < 0 ? 0 : (i > last ? last : i);
  }
  if (periodic) return ((i % n) + n) % n;
  if (face) return i <= 0 ? -i : 2 * n - i;
  return i < 0 ? -1 - i : 2 * n - 1 - i;
}
// the slot positions of HaloLine: face fields 0,-1,-2,-3 and n..n+3; others -1,-2,-3 and n..n+2
__device__ __forceinline__ int halo_pos(int a, int n, int face) {
  const int nl = face ? 4 : 3;
  return a < nl ? (face ? -a : -1 - a) : n + (a - nl);
}
__device__ __forceinline__ bool is_xslot(int i, int n, int face) { return face ? (i <= 0 || i >= n) : (i < 0 || i >= n); }

template <class T>
__device__ __forceinline__ T halo_xval(const HaloField& f, T* p, int i, int j, int k) {
  // the value of (i, j) after the x pass (j an interior row)
  if (!is_xslot(i, f.gnx, f.face_x) || i < f.wi0 || i >= f.wi1) return p[i + j * f.sj + k * f.sk];
  const int src = halo_src(i, f.gnx, f.face_x, f.periodic_x, f.flat_x);
  const T v = p[src + j * f.sj + k * f.sk];
  if (!f.periodic_x && !f.flat_x && src == i) return f.oddface_x ? T(-v) : v;
  return (!f.periodic_x && !f.flat_x && f.odd_x) ? T(-v) : v;
}

template <class T>
__device__ __forceinline__ void halo_cell(const HaloField& f, unsigned c, int pass) {
  T* p = static_cast<T*>(f.ind ? static_cast<V3<T>*>(f.ind)->p : f.p);
  if (c < unsigned(f.ncell_x)) {  // x pass: (k, row j, slot a)
    const unsigned na = f.face_x ? 8 : 6;
    const int a = int(c % na);
    const unsigned r = c / na;
    const unsigned nr = unsigned(f.xj1 - f.xj0);
    const int j = f.xj0 + int(r % nr), k = int(r / nr);
    const int i = halo_pos(a, f.gnx, f.face_x);
    if (i < f.wi0 || i >= f.wi1) return;
    // the last face row of a periodic y-staggered field is a y-pass slot (a copy of row 0): its x halo is the y
    // pass's value (the reference fills x, then y); writing the stale row here too would race with that pass
    if (f.face_y && f.periodic_y && !f.two_d && j == f.gny) return;
    const int src = halo_src(i, f.gnx, f.face_x, f.periodic_x, f.flat_x);
    if (!f.periodic_x && !f.flat_x && src == i) {  // wall face: kept, or flipped by pass 1 (OddFace)
      if (pass == 1 && f.oddface_x) p[i + j * f.sj + k * f.sk] = -p[i + j * f.sj + k * f.sk];
      return;
    }
    if (pass == 1) return;
    T v = p[src + j * f.sj + k * f.sk];
    if (!f.periodic_x && !f.flat_x && f.odd_x) v = -v;
    p[i + j * f.sj + k * f.sk] = v;
    return;
  }
  if (pass == 1) return;
  // y pass: (k, slot b, column i over the full x extent)
  const unsigned cy = c - unsigned(f.ncell_x);
  const unsigned wiw = unsigned(f.wi1 - f.wi0);
  const unsigned na = f.face_y ? 8 : 6;
  const int i = f.wi0 + int(cy % wiw);
  const unsigned r = cy / wiw;
  const int b = int(r % na), k = int(r / na);
  const int jh = halo_pos(b, f.gny, f.face_y);
  if (jh < f.wj0 || jh >= f.wj1) return;
  const int src = halo_src(jh, f.gny, f.face_y, f.periodic_y, f.flat_y);
  if (!f.periodic_y && !f.flat_y && src == jh) return;  // kept (no OddFace in y)
  T v = halo_xval<T>(f, p, i, src, k);
  if (!f.periodic_y && !f.flat_y && f.odd_y) v = -v;
  p[i + jh * f.sj + k * f.sk] = v;
}

// one thread per halo cell of the chunk (the host keeps a chunk's cell count below 2^31)
template <int NF>
__global__ void k_halo(const __grid_constant__ HaloChunk<NF> s, int pass) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.start[s.nf]) return;
  int lo = 0, hi = s.nf - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s.start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const HaloField& f = s.f[lo];
  const unsigned c = t - s.start[lo];
  if (f.is_float) halo_cell<float>(f, c, pass);
  else halo_cell<double>(f, c, pass);
}

// the same over a fill point's fields held in device memory (a batch: every member's fields in one launch)
static __global__ void k_halo_tab(const HaloField* __restrict__ fs, const unsigned* __restrict__ start, int nf, int pass) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= __ldg(start + nf)) return;
  int lo = 0, hi = nf - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  const HaloField f = fs[lo];
  const unsigned c = t - __ldg(start + lo);
  if (f.is_float) halo_cell<float>(f, c, pass);
  else halo_cell<double>(f, c, pass);
}

// a decomposed domain's exchange: one thread per received point of every box of the table (a box between two patches
// of this process, or between a patch and the packed buffer of an exchange with another rank)
static __global__ void k_exchange(const XchgBox* __restrict__ bs, const unsigned* __restrict__ start, int nb) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= __ldg(start + nb)) return;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  const XchgBox b = bs[lo];
  const unsigned c = t - __ldg(start + lo);
  const unsigned wi = unsigned(b.i1 - b.i0), wj = unsigned(b.j1 - b.j0);
  const int i = b.i0 + int(c % wi), j = b.j0 + int((c / wi) % wj), k = int(c / (wi * wj));
  const long long s = b.soff + i + (long long)j * b.ssj + (long long)k * b.ssk;
  const long long d = b.doff + i + (long long)j * b.dsj + (long long)k * b.dsk;
  if (b.is_float) {
    const float* src = b.src_ind ? static_cast<const V3<float>*>(b.src_ind)->p : static_cast<const float*>(b.src);
    float* dst = b.dst_ind ? static_cast<const V3<float>*>(b.dst_ind)->p : static_cast<float*>(b.dst);
    dst[d] = src[s];
  } else {
    const double* src = b.src_ind ? static_cast<const V3<double>*>(b.src_ind)->p : static_cast<const double*>(b.src);
    double* dst = b.dst_ind ? static_cast<const V3<double>*>(b.dst_ind)->p : static_cast<double*>(b.dst);
    dst[d] = src[s];
  }
}

// ------------------------------------------------------------------ rk_step_prep
// KMu (large_step.cpp:49-66), KPrep3 (:68-81), KWW (:83-108), KCq (:127-148), per column (i, j) of
// [0, nx] x [0, nyv): every value a column thread writes depends only on its own column and on halo
// values that the preceding refresh made current.
template <class R>
// (k_ls_prep: mu, u and v are read-only there)
__device__ __forceinline__ R ww_mu_u(const Dom<R>& D, int i, int j) {
  return R(0.5) * (D.mu2.ld(i, j, 0) + D.mub(i, j) + D.mu2.ld(i - 1, j, 0) + D.mub(i - 1, j));
}
template <class R>
__device__ __forceinline__ R ww_mu_v(const Dom<R>& D, int i, int j) {
  return R(0.5) * (D.mu2.ld(i, j, 0) + D.mub(i, j) + D.mu2.ld(i, j - 1, 0) + D.mub(i, j - 1));
}
template <class R>
__device__ __forceinline__ R ww_divv(const Dom<R>& D, int i, int j, int k, R mu1, R mu0, R mv1, R mv0) {
  const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  return D.msftx(i, j) * R(D.dnw[k]) *
         (R(D.rdx) * (div_msf((c1h * mu1 + c2h) * D.u2.ld(i + 1, j, k), D.msfuy(i + 1, j)) - div_msf((c1h * mu0 + c2h) * D.u2.ld(i, j, k), D.msfuy(i, j))) +
          R(D.rdy) * ((c1h * mv1 + c2h) * D.v2.ld(i, j + 1, k) * D.msfvx_inv(i, j + 1) -
                      (c1h * mv0 + c2h) * D.v2.ld(i, j, k) * D.msfvx_inv(i, j)));
}

// ------------------------------------------------------------------ rk_tendency
template <class R>
__device__ __forceinline__ R cqu_(const Dom<R>& D, int i, int j, int k) { return D.n_moist > 0 ? D.cqu.ld(i, j, k) : R(1); }
template <class R>
__device__ __forceinline__ R cqv_(const Dom<R>& D, int i, int j, int k) { return D.n_moist > 0 ? D.cqv.ld(i, j, k) : R(1); }
template <class R>
__device__ __forceinline__ R cqw_(const Dom<R>& D, int i, int j, int k) { return D.n_moist > 0 ? D.cqw.ld(i, j, k) : R(0); }
// (cqu, cqv, cqw are written only by k_ls_prep, which does not read them). The tendency, flux and diffusion
// functions below read only fields that no thread of their kernels writes: the read-only load path (.ld).

// MapC::vxgm (large_step.cpp:121-124): the curvature factor at mass point (i, j, k) from u, v and the map factors
template <class R>
__device__ __forceinline__ R vxgm(const Dom<R>& D, int i, int j, int k) {
  return R(0.5) * (D.u2.ld(i, j, k) + D.u2.ld(i + 1, j, k)) * (D.msfvx(i, j + 1) - D.msfvx(i, j)) * R(D.rdy) -
         R(0.5) * (D.v2.ld(i, j, k) + D.v2.ld(i, j + 1, k)) * (D.msfuy(i + 1, j) - D.msfuy(i, j)) * R(D.rdx);
}
// KTendU (large_step.cpp:152-264)
template <class R>
__device__ R tu_fx(const Dom<R>& D, int i, int j, int k) {
  const int o = ord_mass(i, D.nx, D.spec_x);
  if (o == 2) {
    if (i <= 1) {
      const R ub = (D.sx && D.u2.ld(i, j, k) < R(0)) ? D.u2.ld(i, j, k) : D.u2.ld(i - 1, j, k);
      return R(0.25) * (D.ru.ld(i, j, k) + D.ru.ld(i - 1, j, k)) * (D.u2.ld(i, j, k) + ub);
    }
    const R ub = (D.sx && D.u2.ld(i - 1, j, k) > R(0)) ? D.u2.ld(i - 1, j, k) : D.u2.ld(i, j, k);
    return R(0.25) * (D.ru.ld(i, j, k) + D.ru.ld(i - 1, j, k)) * (D.u2.ld(i - 1, j, k) + ub);
  }
  const R vel = R(0.5) * (D.ru.ld(i, j, k) + D.ru.ld(i - 1, j, k));
  if (o == 3) return vel * flux3(D.u2.ld(i - 2, j, k), D.u2.ld(i - 1, j, k), D.u2.ld(i, j, k), D.u2.ld(i + 1, j, k), vel, R(D.hup));
  return vel * flux5(D.u2.ld(i - 3, j, k), D.u2.ld(i - 2, j, k), D.u2.ld(i - 1, j, k), D.u2.ld(i, j, k), D.u2.ld(i + 1, j, k),
                     D.u2.ld(i + 2, j, k), vel, R(D.hup));
}
template <class R>
__device__ R tu_fy(const Dom<R>& D, int i, int j, int k) {
  const int o = ord_face(j, D.ny, D.spec_y);
  if (o == 2) return R(0.25) * (D.rv.ld(i, j, k) + D.rv.ld(i - 1, j, k)) * (D.u2.ld(i, j, k) + D.u2.ld(i, j - 1, k));
  const R vel = R(0.5) * (D.rv.ld(i, j, k) + D.rv.ld(i - 1, j, k));
  if (o == 3) return vel * flux3(D.u2.ld(i, j - 2, k), D.u2.ld(i, j - 1, k), D.u2.ld(i, j, k), D.u2.ld(i, j + 1, k), vel, R(D.hup));
  return vel * flux5(D.u2.ld(i, j - 3, k), D.u2.ld(i, j - 2, k), D.u2.ld(i, j - 1, k), D.u2.ld(i, j, k), D.u2.ld(i, j + 1, k),
                     D.u2.ld(i, j + 2, k), vel, R(D.hup));
}
template <class R>
__device__ R tu_fz(const Dom<R>& D, int i, int j, int k) {
  if (k == 0 || k == D.nz) return 0;
  const R vel = R(0.5) * (D.ww.ld(i - 1, j, k) + D.ww.ld(i, j, k));
  if (k == 1 || k == D.nz - 1) return vel * (R(D.fnm[k]) * D.u2.ld(i, j, k) + R(D.fnp[k]) * D.u2.ld(i, j, k - 1));
  return vel * flux3(D.u2.ld(i, j, k - 2), D.u2.ld(i, j, k - 1), D.u2.ld(i, j, k), D.u2.ld(i, j, k + 1), -vel, R(D.vup));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R pgf_dpn(const Dom<R>& D, int i, int j, int k) {  // p' at w level k, face column
  auto ps = [&](int kk) { return D.p.ld(i - DI, j - DJ, kk) + D.p.ld(i, j, kk); };
  const int nz = D.nz;
  if (k == 0) return R(0.5) * (R(D.cf1) * ps(0) + R(D.cf2) * ps(1) + R(D.cf3) * ps(2));
  if (k == nz) return D.top_lid ? R(0.5) * (R(D.cfn) * ps(nz - 1) + R(D.cfn1) * ps(nz - 2)) : R(0);
  return R(0.5) * (R(D.fnm[k]) * ps(k) + R(D.fnp[k]) * ps(k - 1));
}
// advect_u open_ys / open_ye (KTendU::open_y_term, :193-208): the v-flux terms of the outermost rows
template <class R>
__device__ R tu_open_y(const Dom<R>& D, int i, int j, int k) {
  const int imin = 0, imax = D.nx - 1;
  const int ip = i < imax ? i : imax, im = i - 1 > imin ? i - 1 : imin;
  const R mrdy = D.msfux(i, j) * R(D.rdy);
  if (j == 0) {
    const R vw = R(0.5) * (D.rv.ld(ip, 0, k) + D.rv.ld(im, 0, k));
    const R vb = vw < R(0) ? vw : R(0);
    const R dvm = D.rv.ld(ip, 1, k) - D.rv.ld(ip, 0, k), dvp = D.rv.ld(im, 1, k) - D.rv.ld(im, 0, k);
    return mrdy * (vb * (D.u2.ld(i, 1, k) - D.u2.ld(i, 0, k)) + R(0.5) * D.u2.ld(i, 0, k) * (dvm + dvp));
  }
  const int je = D.ny;
  const R vw = R(0.5) * (D.rv.ld(ip, je, k) + D.rv.ld(im, je, k));
  const R vb = vw > R(0) ? vw : R(0);
  const R dvm = D.rv.ld(ip, je, k) - D.rv.ld(ip, je - 1, k), dvp = D.rv.ld(im, je, k) - D.rv.ld(im, je - 1, k);
  return mrdy * (vb * (D.u2.ld(i, je - 1, k) - D.u2.ld(i, je - 2, k)) + R(0.5) * D.u2.ld(i, je - 1, k) * (dvm + dvp));
}
// an open x boundary face of u (:210-227): the radiation condition with phase speed cb, the vertical advection
// unless y is open too, and the held tendency
template <class R>
__device__ R tend_u_open_face(const Dom<R>& D, int i, int j, int k, bool use_tendf) {
  const R rdx = R(D.rdx), c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  R t;
  if (i == 0) {
    R ub = D.ru.ld(0, j, k) - R(k::cb) * (c1h * D.mut.ld(0, j, 0) + c2h);
    ub = ub < R(0) ? ub : R(0);
    t = R(0) - rdx * ub * (D.u2.ld(1, j, k) - D.u2.ld(0, j, k));
  } else {
    R ub = D.ru.ld(i, j, k) + R(k::cb) * (c1h * D.mut.ld(i - 1, j, 0) + c2h);
    ub = ub > R(0) ? ub : R(0);
    t = R(0) - rdx * ub * (D.u2.ld(i, j, k) - D.u2.ld(i - 1, j, k));
  }
  if (!D.open_y) t -= R(D.rdnw[k]) * (tu_fz(D, i, j, k + 1) - tu_fz(D, i, j, k));
  if (use_tendf) t += div_msf(D.ru_tendf.ld(i, j, k), D.msfuy(i, j));
  return t;
}
// OP: the kernel variant for packs with an open boundary (the checks compile away in the other)
template <bool OP, class R>
__device__ R tend_u(const Dom<R>& D, int i, int j, int k, bool use_tendf, R fx0, R fx1, R fy0, R fy1) {
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  R t = -(D.msfux(i, j) * rdx) * (fx1 - fx0);
  if (D.do_y) {  // open_ys / ye: the outermost rows take the open terms instead of the y flux divergence
    if (!(OP && D.open_y && (j == 0 || j == D.ny - 1))) t -= (D.msfux(i, j) * rdy) * (fy1 - fy0);
    else t -= tu_open_y(D, i, j, k);
  }
  if (!(OP && D.open_y && D.spec_x && (i == 0 || i == D.nx))) t -= R(D.rdnw[k]) * (tu_fz(D, i, j, k + 1) - tu_fz(D, i, j, k));
  const R rm = div_msf(D.msfux(i, j), D.msfuy(i, j));
  R dpx = rm * R(0.5) * rdx * (c1h * D.muu.ld(i, j, 0) + c2h) *
          ((D.ph2.ld(i, j, k + 1) - D.ph2.ld(i - 1, j, k + 1) + D.ph2.ld(i, j, k) - D.ph2.ld(i - 1, j, k)) +
           (D.alt.ld(i, j, k) + D.alt.ld(i - 1, j, k)) * (D.p.ld(i, j, k) - D.p.ld(i - 1, j, k)) +
           (D.al.ld(i, j, k) + D.al.ld(i - 1, j, k)) * (D.pb(i, j, k) - D.pb(i - 1, j, k)));
  dpx += rm * rdx * (D.php.ld(i, j, k) - D.php.ld(i - 1, j, k)) *
         (R(D.rdnw[k]) * (pgf_dpn<R, 1, 0>(D, i, j, k + 1) - pgf_dpn<R, 1, 0>(D, i, j, k)) -
          R(0.5) * (c1h * D.mu2.ld(i - 1, j, 0) + c1h * D.mu2.ld(i, j, 0)));
  t -= cqu_(D, i, j, k) * dpx;
  const R rw4 = R(0.25) * (D.rw.ld(i - 1, j, k + 1) + D.rw.ld(i - 1, j, k) + D.rw.ld(i, j, k + 1) + D.rw.ld(i, j, k));
  if (D.cor) {  // Coriolis (:249-253), and the curvature from the map factors' gradients (:255-257)
    const R rv4 = R(0.25) * (D.rv.ld(i - 1, j + 1, k) + D.rv.ld(i, j + 1, k) + D.rv.ld(i - 1, j, k) + D.rv.ld(i, j, k));
    t = t + rm * R(0.5) * (D.f(i, j) + D.f(i - 1, j)) * rv4 -
        R(0.5) * (D.e(i, j) + D.e(i - 1, j)) * R(0.5) * (D.cosa(i, j) + D.cosa(i - 1, j)) * rw4;
    if (D.mapped) t = t + R(0.5) * (vxgm(D, i, j, k) + vxgm(D, i - 1, j, k)) * rv4 - D.u2.ld(i, j, k) * R(k::reradius) * rw4;
    else t = t - D.u2.ld(i, j, k) * R(k::reradius) * rw4;
  } else {
    t = t - D.u2.ld(i, j, k) * R(k::reradius) * rw4;
  }
  if (use_tendf) t += div_msf(D.ru_tendf.ld(i, j, k), D.msfuy(i, j));
  return t;
}

// KTendV (:267-376)
template <class R>
__device__ R tv_fx(const Dom<R>& D, int i, int j, int k) {
  const int o = ord_face(i, D.nx, D.spec_x);
  if (o == 2) return R(0.25) * (D.ru.ld(i, j, k) + D.ru.ld(i, j - 1, k)) * (D.v2.ld(i, j, k) + D.v2.ld(i - 1, j, k));
  const R vel = R(0.5) * (D.ru.ld(i, j, k) + D.ru.ld(i, j - 1, k));
  if (o == 3) return vel * flux3(D.v2.ld(i - 2, j, k), D.v2.ld(i - 1, j, k), D.v2.ld(i, j, k), D.v2.ld(i + 1, j, k), vel, R(D.hup));
  return vel * flux5(D.v2.ld(i - 3, j, k), D.v2.ld(i - 2, j, k), D.v2.ld(i - 1, j, k), D.v2.ld(i, j, k), D.v2.ld(i + 1, j, k),
                     D.v2.ld(i + 2, j, k), vel, R(D.hup));
}
template <class R>
__device__ R tv_fy(const Dom<R>& D, int i, int j, int k) {
  const int o = ord_mass(j, D.ny, D.spec_y);
  if (o == 2) {
    if (j <= 1) {
      const R vb = (D.sy && D.v2.ld(i, j, k) < R(0)) ? D.v2.ld(i, j, k) : D.v2.ld(i, j - 1, k);
      return R(0.25) * (D.rv.ld(i, j, k) + D.rv.ld(i, j - 1, k)) * (D.v2.ld(i, j, k) + vb);
    }
    const R vb = (D.sy && D.v2.ld(i, j - 1, k) > R(0)) ? D.v2.ld(i, j - 1, k) : D.v2.ld(i, j, k);
    return R(0.25) * (D.rv.ld(i, j, k) + D.rv.ld(i, j - 1, k)) * (vb + D.v2.ld(i, j - 1, k));
  }
  const R vel = R(0.5) * (D.rv.ld(i, j, k) + D.rv.ld(i, j - 1, k));
  if (o == 3) return vel * flux3(D.v2.ld(i, j - 2, k), D.v2.ld(i, j - 1, k), D.v2.ld(i, j, k), D.v2.ld(i, j + 1, k), vel, R(D.hup));
  return vel * flux5(D.v2.ld(i, j - 3, k), D.v2.ld(i, j - 2, k), D.v2.ld(i, j - 1, k), D.v2.ld(i, j, k), D.v2.ld(i, j + 1, k),
                     D.v2.ld(i, j + 2, k), vel, R(D.hup));
}
template <class R>
__device__ R tv_fz(const Dom<R>& D, int i, int j, int k) {
  if (k == 0 || k == D.nz) return 0;
  const R vel = R(0.5) * (D.ww.ld(i, j - 1, k) + D.ww.ld(i, j, k));
  if (k == 1 || k == D.nz - 1) return vel * (R(D.fnm[k]) * D.v2.ld(i, j, k) + R(D.fnp[k]) * D.v2.ld(i, j, k - 1));
  return vel * flux3(D.v2.ld(i, j, k - 2), D.v2.ld(i, j, k - 1), D.v2.ld(i, j, k), D.v2.ld(i, j, k + 1), -vel, R(D.vup));
}
// advect_v open_xs / open_xe (KTendV::open_x_term, :307-323): the u-flux terms of the outermost columns
template <class R>
__device__ R tv_open_x(const Dom<R>& D, int i, int j, int k) {
  const int jmin = 0, jmax = D.ny - 1;
  const int jp = j < jmax ? j : jmax, jm = j - 1 > jmin ? j - 1 : jmin;
  if (i == 0) {
    const R mrdx = D.msfvy(0, j) * R(D.rdx);
    const R uw = R(0.5) * (D.ru.ld(0, jp, k) + D.ru.ld(0, jm, k));
    const R ub = uw < R(0) ? uw : R(0);
    const R dup = D.ru.ld(1, jp, k) - D.ru.ld(0, jp, k), dum = D.ru.ld(1, jm, k) - D.ru.ld(0, jm, k);
    return mrdx * (ub * (D.v2.ld(1, j, k) - D.v2.ld(0, j, k)) + R(0.5) * D.v2.ld(0, j, k) * (dup + dum));
  }
  const int ie = D.nx;
  const R mrdx = D.msfvy(ie - 1, j) * R(D.rdx);
  const R uw = R(0.5) * (D.ru.ld(ie, jp, k) + D.ru.ld(ie, jm, k));
  const R ub = uw > R(0) ? uw : R(0);
  const R dup = D.ru.ld(ie, jp, k) - D.ru.ld(ie - 1, jp, k), dum = D.ru.ld(ie, jm, k) - D.ru.ld(ie - 1, jm, k);
  return mrdx * (ub * (D.v2.ld(ie - 1, j, k) - D.v2.ld(ie - 2, j, k)) + R(0.5) * D.v2.ld(ie - 1, j, k) * (dup + dum));
}
// an open y boundary face of v (:327-340): the radiation condition only, and the held tendency
template <class R>
__device__ R tend_v_open_face(const Dom<R>& D, int i, int j, int k, bool use_tendf) {
  const R rdy = R(D.rdy), c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  R t;
  if (j == 0) {
    R vb = D.rv.ld(i, 0, k) - R(k::cb) * (c1h * D.mut.ld(i, 0, 0) + c2h);
    vb = vb < R(0) ? vb : R(0);
    t = R(0) - rdy * vb * (D.v2.ld(i, 1, k) - D.v2.ld(i, 0, k));
  } else {
    R vb = D.rv.ld(i, j, k) + R(k::cb) * (c1h * D.mut.ld(i, j - 1, 0) + c2h);
    vb = vb > R(0) ? vb : R(0);
    t = R(0) - rdy * vb * (D.v2.ld(i, j, k) - D.v2.ld(i, j - 1, k));
  }
  if (use_tendf) t += D.rv_tendf.ld(i, j, k) * D.msfvx_inv(i, j);
  return t;
}
template <bool OP, class R>
__device__ R tend_v(const Dom<R>& D, int i, int j, int k, bool use_tendf, R fx0, R fx1, R fy0, R fy1) {
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  const R c1h = R(D.c1h[k]), c2h = R(D.c2h[k]);
  const R rm = div_msf(D.msfvy(i, j), D.msfvx(i, j));
  R t;
  if (OP && D.open_x && (i == 0 || i == D.nx - 1)) {  // open x: the y flux, then the open term instead of the x flux
    t = -(D.msfvy(i, j) * rdy) * (fy1 - fy0);
    t -= tv_open_x(D, i, j, k);
  } else {
    t = -(D.msfvy(i, j) * rdx) * (fx1 - fx0);
    t -= (D.msfvy(i, j) * rdy) * (fy1 - fy0);
  }
  t -= rm * R(D.rdnw[k]) * (tv_fz(D, i, j, k + 1) - tv_fz(D, i, j, k));
  R dpy = rm * R(0.5) * rdy * (c1h * D.muv.ld(i, j, 0) + c2h) *
          ((D.ph2.ld(i, j, k + 1) - D.ph2.ld(i, j - 1, k + 1) + D.ph2.ld(i, j, k) - D.ph2.ld(i, j - 1, k)) +
           (D.alt.ld(i, j, k) + D.alt.ld(i, j - 1, k)) * (D.p.ld(i, j, k) - D.p.ld(i, j - 1, k)) +
           (D.al.ld(i, j, k) + D.al.ld(i, j - 1, k)) * (D.pb(i, j, k) - D.pb(i, j - 1, k)));
  dpy += rm * rdy * (D.php.ld(i, j, k) - D.php.ld(i, j - 1, k)) *
         (R(D.rdnw[k]) * (pgf_dpn<R, 0, 1>(D, i, j, k + 1) - pgf_dpn<R, 0, 1>(D, i, j, k)) -
          R(0.5) * (c1h * D.mu2.ld(i, j - 1, 0) + c1h * D.mu2.ld(i, j, 0)));
  t -= cqv_(D, i, j, k) * dpy;
  const R rw4 = R(0.25) * (D.rw.ld(i, j - 1, k + 1) + D.rw.ld(i, j - 1, k) + D.rw.ld(i, j, k + 1) + D.rw.ld(i, j, k));
  if (D.cor) {  // Coriolis (:362-365), and the curvature from the map factors' gradients (:367-369)
    const R ru4 = R(0.25) * (D.ru.ld(i, j, k) + D.ru.ld(i + 1, j, k) + D.ru.ld(i, j - 1, k) + D.ru.ld(i + 1, j - 1, k));
    t = t - rm * R(0.5) * (D.f(i, j) + D.f(i, j - 1)) * ru4 +
        rm * R(0.5) * (D.e(i, j) + D.e(i, j - 1)) * R(0.5) * (D.sina(i, j) + D.sina(i, j - 1)) * rw4;
    if (D.mapped) t = t - R(0.5) * (vxgm(D, i, j, k) + vxgm(D, i, j - 1, k)) * ru4 - rm * D.v2.ld(i, j, k) * R(k::reradius) * rw4;
    else t = t - rm * D.v2.ld(i, j, k) * R(k::reradius) * rw4;
  } else {
    t = t - rm * D.v2.ld(i, j, k) * R(k::reradius) * rw4;
  }
  if (use_tendf) t += D.rv_tendf.ld(i, j, k) * D.msfvx_inv(i, j);
  return t;
}

// KTendW (:379-499)
template <class R>
__device__ __forceinline__ R tw_rux(const Dom<R>& D, int i, int j, int k) {
  const int nz = D.nz;
  if (k < nz) return R(D.fnm[k]) * D.ru.ld(i, j, k) + R(D.fnp[k]) * D.ru.ld(i, j, k - 1);
  return (R(2) - R(D.fnm[nz - 1])) * D.ru.ld(i, j, nz - 1) - R(D.fnp[nz - 1]) * D.ru.ld(i, j, nz - 2);
}
template <class R>
__device__ __forceinline__ R tw_rvy(const Dom<R>& D, int i, int j, int k) {
  const int nz = D.nz;
  if (k < nz) return R(D.fnm[k]) * D.rv.ld(i, j, k) + R(D.fnp[k]) * D.rv.ld(i, j, k - 1);
  return (R(2) - R(D.fnm[nz - 1])) * D.rv.ld(i, j, nz - 1) - R(D.fnp[nz - 1]) * D.rv.ld(i, j, nz - 2);
}
template <class R>
__device__ R tw_fx(const Dom<R>& D, int i, int j, int k) {
  const R vel = tw_rux(D, i, j, k);
  const int o = ord_face(i, D.nx, D.spec_x);
  if (o == 2) return R(0.5) * vel * (D.w2.ld(i, j, k) + D.w2.ld(i - 1, j, k));
  if (o == 3) return vel * flux3(D.w2.ld(i - 2, j, k), D.w2.ld(i - 1, j, k), D.w2.ld(i, j, k), D.w2.ld(i + 1, j, k), vel, R(D.hup));
  return vel * flux5(D.w2.ld(i - 3, j, k), D.w2.ld(i - 2, j, k), D.w2.ld(i - 1, j, k), D.w2.ld(i, j, k), D.w2.ld(i + 1, j, k),
                     D.w2.ld(i + 2, j, k), vel, R(D.hup));
}
template <class R>
__device__ R tw_fy(const Dom<R>& D, int i, int j, int k) {
  const R vel = tw_rvy(D, i, j, k);
  const int o = ord_face(j, D.ny, D.spec_y);
  if (o == 2) return R(0.5) * vel * (D.w2.ld(i, j, k) + D.w2.ld(i, j - 1, k));
  if (o == 3) return vel * flux3(D.w2.ld(i, j - 2, k), D.w2.ld(i, j - 1, k), D.w2.ld(i, j, k), D.w2.ld(i, j + 1, k), vel, R(D.hup));
  return vel * flux5(D.w2.ld(i, j - 3, k), D.w2.ld(i, j - 2, k), D.w2.ld(i, j - 1, k), D.w2.ld(i, j, k), D.w2.ld(i, j + 1, k),
                     D.w2.ld(i, j + 2, k), vel, R(D.hup));
}
template <class R>
__device__ R tw_fz(const Dom<R>& D, int i, int j, int m) {
  if (m == 0 || m == D.nz - 1)
    return R(0.25) * (D.ww.ld(i, j, m + 1) + D.ww.ld(i, j, m)) * (D.w2.ld(i, j, m + 1) + D.w2.ld(i, j, m));
  const R vel = R(0.5) * (D.ww.ld(i, j, m + 1) + D.ww.ld(i, j, m));
  return vel * flux3(D.w2.ld(i, j, m - 1), D.w2.ld(i, j, m), D.w2.ld(i, j, m + 1), D.w2.ld(i, j, m + 2), -vel, R(D.vup));
}
// advect_w open_xs/xe (open_ys/ye) terms of the outermost columns (rows) (KTendW::open_x_term / open_y_term,
// :416-453): DI = 1 for x, 0 for y; the normal mass flux fnm/fnp-interpolated to the w level, extrapolated at the lid
template <class R, int DI>
__device__ R tw_open(const Dom<R>& D, int i, int j, int k) {
  const int nz = D.nz;
  const int c = DI ? i : j, n = DI ? D.nx : D.ny;
  const int a = c == 0 ? 0 : n - 1, b = c == 0 ? 1 : n;  // faces: outer side a, inner side b
  const V3<R>& rf = DI ? D.ru : D.rv;
  auto RF = [&](int f, int kk) { return DI ? rf.ld(f, j, kk) : rf.ld(i, f, kk); };
  auto Wv = [&](int f) { return DI ? D.w2.ld(f, j, k) : D.w2.ld(i, f, k); };
  R uw, dru;
  if (k < nz) {
    const R fnm = R(D.fnm[k]), fnp = R(D.fnp[k]);
    uw = R(0.5) * (fnm * (RF(a, k) + RF(b, k)) + fnp * (RF(a, k - 1) + RF(b, k - 1)));
    dru = fnm * (RF(b, k) - RF(a, k)) + fnp * (RF(b, k - 1) - RF(a, k - 1));
  } else {
    const R fm = R(2) - R(D.fnm[nz - 1]), fp = R(D.fnp[nz - 1]);
    uw = R(0.5) * (fm * (RF(a, nz - 1) + RF(b, nz - 1)) - fp * (RF(a, nz - 2) + RF(b, nz - 2)));
    dru = fm * (RF(b, nz - 1) - RF(a, nz - 1)) - fp * (RF(b, nz - 2) - RF(a, nz - 2));
  }
  const R rd = DI ? R(D.rdx) : R(D.rdy);
  if (c == 0) {
    const R ub = uw < R(0) ? uw : R(0);
    return rd * (ub * (Wv(1) - Wv(0)) + Wv(0) * dru);
  }
  const R ub = uw > R(0) ? uw : R(0);
  return rd * (ub * (Wv(c) - Wv(c - 1)) + Wv(c) * dru);
}
template <bool OP, class R>
__device__ R tend_w(const Dom<R>& D, int i, int j, int k, bool use_tendf, R fx0, R fx1, R fy0, R fy1) {
  const int nz = D.nz;
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  R t;
  const bool ocol = OP && D.open_x && (i == 0 || i == D.nx - 1), orow = OP && D.open_y && (j == 0 || j == D.ny - 1);
  if (ocol || orow) {  // the reference's order: y flux, x flux, open x terms, open y terms
    t = R(0);
    if (D.do_y && !orow) t = t - (D.msftx(i, j) * rdy) * (fy1 - fy0);
    if (!ocol) t = t - (D.msftx(i, j) * rdx) * (fx1 - fx0);
    if (ocol) t = t - tw_open<R, 1>(D, i, j, k);
    if (orow) t = t - tw_open<R, 0>(D, i, j, k);
  } else {
    t = -(D.msftx(i, j) * rdx) * (fx1 - fx0);
    if (D.do_y) t -= (D.msftx(i, j) * rdy) * (fy1 - fy0);
  }
  const R rmsft = div_msf(R(1), D.msfty(i, j));
  if (k < nz) {
    t -= R(D.rdn[k]) * (tw_fz(D, i, j, k) - tw_fz(D, i, j, k - 1));
    const R cqw = cqw_(D, i, j, k), cq1 = R(1) / (R(1) + cqw), cq2 = cqw * cq1;
    t += rmsft * R(k::g) *
         (cq1 * R(D.rdn[k]) * (D.p.ld(i, j, k) - D.p.ld(i, j, k - 1)) - R(D.c1f[k]) * D.mu2.ld(i, j, 0) -
          cq2 * (R(D.c1f[k]) * D.mub(i, j) + R(D.c2f[k])));
    if (D.w_damping) {  // w_damp, wd_dt = dt
      const R wd_dt = R(D.dt);
      const R muf = R(D.c1f[k]) * D.mut.ld(i, j, 0) + R(D.c2f[k]);
      R cfl = D.ww.ld(i, j, k) / muf * R(D.rdnw[k]) * wd_dt;
      cfl = cfl < R(0) ? -cfl : cfl;
      if (cfl > R(1)) t = t - (D.w2.ld(i, j, k) < R(0) ? R(-1) : R(1)) * R(0.3) * (cfl - R(D.w_crit_cfl)) * muf;
    }
    const R fnm = R(D.fnm[k]), fnp = R(D.fnp[k]);
    const R ruw = R(0.5) * (fnm * (D.ru.ld(i, j, k) + D.ru.ld(i + 1, j, k)) + fnp * (D.ru.ld(i, j, k - 1) + D.ru.ld(i + 1, j, k - 1)));
    const R rvw = R(0.5) * (fnm * (D.rv.ld(i, j, k) + D.rv.ld(i, j + 1, k)) + fnp * (D.rv.ld(i, j, k - 1) + D.rv.ld(i, j + 1, k - 1)));
    const R rmt = div_msf(D.msftx(i, j), D.msfty(i, j));
    if (D.cor) t = t + D.e(i, j) * (D.cosa(i, j) * ruw - rmt * D.sina(i, j) * rvw);  // Coriolis (:484)
    const R uw = R(0.5) * (fnm * (D.u2.ld(i, j, k) + D.u2.ld(i + 1, j, k)) + fnp * (D.u2.ld(i, j, k - 1) + D.u2.ld(i + 1, j, k - 1)));
    const R vw = R(0.5) * (fnm * (D.v2.ld(i, j, k) + D.v2.ld(i, j + 1, k)) + fnp * (D.v2.ld(i, j, k - 1) + D.v2.ld(i, j + 1, k - 1)));
    t = t + R(k::reradius) * (ruw * uw + rmt * rvw * vw);
  } else {
    t += R(2) * R(D.rdn[nz - 1]) * tw_fz(D, i, j, nz - 1);
    const R cqw = cqw_(D, i, j, nz - 1), cq1 = R(1) / (R(1) + cqw), cq2 = cqw * cq1;
    t += rmsft * R(k::g) *
         (cq1 * R(2) * R(D.rdnw[nz - 1]) * (-D.p.ld(i, j, nz - 1)) - R(D.c1f[nz]) * D.mu2.ld(i, j, 0) -
          cq2 * (R(D.c1f[nz]) * D.mub(i, j) + R(D.c2f[nz])));
  }
  if (use_tendf) t += div_msf(D.rw_tendf.ld(i, j, k), D.msfty(i, j));
  return t;
}

// KTendT (:502-565) / advect_scalar face fluxes of any mass field q with mass fluxes (ufx, vfy, wfz); q is a view of
// the field in global memory (V3) or of a tile of its planes in shared memory (QPlanes), read with the domain's indices
template <class R, class QV>
__device__ R sc_fx(const Dom<R>& D, const QV& q, const V3<R>& ruf, int i, int j, int k, bool pd) {
  const R vel = ruf.ld(i, j, k);
  const int o = ord_face(i, D.nx, D.spec_x);
  if (o == 2) return R(0.5) * vel * (q.ld(i, j, k) + q.ld(i - 1, j, k));
  if (o == 3) {
    if (pd) return vel * flux3_pd(q.ld(i - 2, j, k), q.ld(i - 1, j, k), q.ld(i, j, k), q.ld(i + 1, j, k), vel, R(D.hup));
    return vel * flux3(q.ld(i - 2, j, k), q.ld(i - 1, j, k), q.ld(i, j, k), q.ld(i + 1, j, k), vel, R(D.hup));
  }
  if (pd)
    return vel * flux5_pd(q.ld(i - 3, j, k), q.ld(i - 2, j, k), q.ld(i - 1, j, k), q.ld(i, j, k), q.ld(i + 1, j, k), q.ld(i + 2, j, k), vel, R(D.hup));
  return vel * flux5(q.ld(i - 3, j, k), q.ld(i - 2, j, k), q.ld(i - 1, j, k), q.ld(i, j, k), q.ld(i + 1, j, k), q.ld(i + 2, j, k), vel, R(D.hup));
}
template <class R, class QV>
__device__ R sc_fy(const Dom<R>& D, const QV& q, const V3<R>& rvf, int i, int j, int k, bool pd) {
  const R vel = rvf.ld(i, j, k);
  const int o = ord_face(j, D.ny, D.spec_y);
  if (o == 2) return R(0.5) * vel * (q.ld(i, j, k) + q.ld(i, j - 1, k));
  if (o == 3) {
    if (pd) return vel * flux3_pd(q.ld(i, j - 2, k), q.ld(i, j - 1, k), q.ld(i, j, k), q.ld(i, j + 1, k), vel, R(D.hup));
    return vel * flux3(q.ld(i, j - 2, k), q.ld(i, j - 1, k), q.ld(i, j, k), q.ld(i, j + 1, k), vel, R(D.hup));
  }
  if (pd)
    return vel * flux5_pd(q.ld(i, j - 3, k), q.ld(i, j - 2, k), q.ld(i, j - 1, k), q.ld(i, j, k), q.ld(i, j + 1, k), q.ld(i, j + 2, k), vel, R(D.hup));
  return vel * flux5(q.ld(i, j - 3, k), q.ld(i, j - 2, k), q.ld(i, j - 1, k), q.ld(i, j, k), q.ld(i, j + 1, k), q.ld(i, j + 2, k), vel, R(D.hup));
}
template <class R, class QV>
__device__ R sc_fz(const Dom<R>& D, const QV& q, const V3<R>& wwf, int i, int j, int k, bool pd) {
  if (k == 0 || k == D.nz) return 0;
  const R vel = wwf.ld(i, j, k);
  if (k == 1 || k == D.nz - 1) return vel * (R(D.fnm[k]) * q.ld(i, j, k) + R(D.fnp[k]) * q.ld(i, j, k - 1));
  if (pd) return vel * flux3_pd(q.ld(i, j, k - 2), q.ld(i, j, k - 1), q.ld(i, j, k), q.ld(i, j, k + 1), -vel, R(D.vup));
  return vel * flux3(q.ld(i, j, k - 2), q.ld(i, j, k - 1), q.ld(i, j, k), q.ld(i, j, k + 1), -vel, R(D.vup));
}
// open boundaries of advect_scalar / advect_scalar_pd (kern::open_x_scalar / open_y_scalar, kernels_common.hpp:61-84):
// the outermost column (row) takes rd (ub (qo(inner) - qo(outer)) + q (f(b) - f(a))) with the inflow mean normal
// mass flux ub of the cell (returned without sign); DI = 1 for x, 0 for y
template <class R, int DI>
__device__ R open_scalar(const Dom<R>& D, const V3<R>& q, const V3<R>& qo, const V3<R>& mf, int i, int j, int k) {
  auto M = [&](int f) { return DI ? mf.ld(f, j, k) : mf.ld(i, f, k); };
  auto Q = [&](const V3<R>& a, int f) { return DI ? a.ld(f, j, k) : a.ld(i, f, k); };
  const int c = DI ? i : j, n = DI ? D.nx : D.ny;
  const R rd = DI ? R(D.rdx) : R(D.rdy);
  if (c == 0) {
    R ub = R(0.5) * (M(0) + M(1));
    ub = ub < R(0) ? ub : R(0);
    return rd * (ub * (Q(qo, 1) - Q(qo, 0)) + Q(q, 0) * (M(1) - M(0)));
  }
  R ub = R(0.5) * (M(n - 1) + M(n));
  ub = ub > R(0) ? ub : R(0);
  return rd * (ub * (Q(qo, n - 1) - Q(qo, n - 2)) + Q(q, n - 1) * (M(n) - M(n - 1)));
}
template <bool OP, class R>
__device__ R tend_t(const Dom<R>& D, int i, int j, int k, bool use_tendf, bool use_hd, R fx0, R fx1, R fy0, R fy1) {
  R r;
  const bool ocol = OP && D.open_x && (i == 0 || i == D.nx - 1), orow = OP && D.open_y && (j == 0 || j == D.ny - 1);
  if (ocol || orow) {  // open boundary (:535-541): y flux, x flux, open x terms, open y terms, then the vertical
    r = R(0);
    if (D.do_y && !orow) r = r - (D.msftx(i, j) * R(D.rdy)) * (fy1 - fy0);
    if (!ocol) r = r - (D.msftx(i, j) * R(D.rdx)) * (fx1 - fx0);
    if (ocol) r = r - open_scalar<R, 1>(D, D.t2, D.t2, D.ru, i, j, k);
    if (orow) r = r - open_scalar<R, 0>(D, D.t2, D.t2, D.rv, i, j, k);
  } else {
    r = -(D.msftx(i, j) * R(D.rdx)) * (fx1 - fx0);
    if (D.do_y) r -= (D.msftx(i, j) * R(D.rdy)) * (fy1 - fy0);
  }
  r -= R(D.rdnw[k]) * (sc_fz(D, D.t2, D.ww, i, j, k + 1, false) - sc_fz(D, D.t2, D.ww, i, j, k, false));
  if (use_tendf) r += div_msf(D.t_tendf.ld(i, j, k), D.msfty(i, j));
  if (use_hd) r += div_msf((R(D.c1h[k]) * D.mut.ld(i, j, 0) + R(D.c2h[k])) * D.hd.ld(i, j, k), D.msfty(i, j));
  return r;
}

// KTendPh (:570-668)
template <class R>
__device__ __forceinline__ R tph_wdwn(const Dom<R>& D, int i, int j, int m) {
  return R(0.5) * (D.ww.ld(i, j, m + 1) + D.ww.ld(i, j, m)) * R(D.rdnw[m]) *
         (D.ph2.ld(i, j, m + 1) - D.ph2.ld(i, j, m) + D.phb(i, j, m + 1) - D.phb(i, j, m));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R grad6(const Dom<R>& D, int i, int j, int k) {
  return R(45) * (D.ph2.ld(i + DI, j + DJ, k) - D.ph2.ld(i - DI, j - DJ, k)) -
         R(9) * (D.ph2.ld(i + 2 * DI, j + 2 * DJ, k) - D.ph2.ld(i - 2 * DI, j - 2 * DJ, k)) +
         (D.ph2.ld(i + 3 * DI, j + 3 * DJ, k) - D.ph2.ld(i - 3 * DI, j - 3 * DJ, k)) +
         R(45) * (D.phb(i + DI, j + DJ, k) - D.phb(i - DI, j - DJ, k)) -
         R(9) * (D.phb(i + 2 * DI, j + 2 * DJ, k) - D.phb(i - 2 * DI, j - 2 * DJ, k)) +
         (D.phb(i + 3 * DI, j + 3 * DJ, k) - D.phb(i - 3 * DI, j - 3 * DJ, k));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R grad4(const Dom<R>& D, int i, int j, int k) {
  return R(8) * (D.ph2.ld(i + DI, j + DJ, k) - D.ph2.ld(i - DI, j - DJ, k)) -
         (D.ph2.ld(i + 2 * DI, j + 2 * DJ, k) - D.ph2.ld(i - 2 * DI, j - 2 * DJ, k)) +
         R(8) * (D.phb(i + DI, j + DJ, k) - D.phb(i - DI, j - DJ, k)) -
         (D.phb(i + 2 * DI, j + 2 * DJ, k) - D.phb(i - 2 * DI, j - 2 * DJ, k));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R dfwd(const Dom<R>& D, int i, int j, int k) {
  return D.phb(i + DI, j + DJ, k) - D.phb(i, j, k) + D.ph2.ld(i + DI, j + DJ, k) - D.ph2.ld(i, j, k);
}
__device__ __forceinline__ int ph_horder(int i, int n, int on, int is_x, int open_x) {
  if (!on) return 6;
  if (i <= 0 || i >= n - 1) return 0;
  if (i == 1 || i == n - 2) return 2;
  if (i == 2 || i == n - 3) return (is_x && !open_x) ? 0 : 4;  // open x: 4th order (open_xs/xe only)
  return 6;
}
template <bool OP, class R>
__device__ R tend_ph(const Dom<R>& D, int i, int j, int k, bool use_tendf) {
  const int nz = D.nz;
  const R c1f = R(D.c1f[k]), c2f = R(D.c2f[k]);
  R t = 0;
  if (k < nz) t = t - (R(D.fnm[k]) * tph_wdwn(D, i, j, k) + R(D.fnp[k]) * tph_wdwn(D, i, j, k - 1));
  t = t + div_msf((c1f * D.mut.ld(i, j, 0) + c2f) * R(k::g) * D.w2.ld(i, j, k), D.msfty(i, j));
  const R r60 = R(1) / R(60), r12 = R(1) / R(12);
  if (D.do_y) {
    const R mvp = c1f * D.muv.ld(i, j + 1, 0) + c2f, mvm = c1f * D.muv.ld(i, j, 0) + c2f;
    const R vp = k < nz ? D.v2.ld(i, j + 1, k) + D.v2.ld(i, j + 1, k - 1) : R(D.cfn) * D.v2.ld(i, j + 1, nz - 1) + R(D.cfn1) * D.v2.ld(i, j + 1, nz - 2);
    const R vm = k < nz ? D.v2.ld(i, j, k) + D.v2.ld(i, j, k - 1) : R(D.cfn) * D.v2.ld(i, j, nz - 1) + R(D.cfn1) * D.v2.ld(i, j, nz - 2);
    const R cy = div_msf((k < nz ? R(0.25) : R(0.5)) * R(D.rdy), D.msfty(i, j));
    const int o = ph_horder(j, D.ny, D.spec_y, 0, OP && D.open_x);
    if (o == 6) t = t - cy * ((mvp * vp * D.msfvy(i, j + 1) + mvm * vm * D.msfvy(i, j)) * r60 * grad6<R, 0, 1>(D, i, j, k));
    else if (o == 4) t = t - cy * ((mvp * vp * D.msfvy(i, j + 1) + mvm * vm * D.msfvy(i, j)) * r12 * grad4<R, 0, 1>(D, i, j, k));
    else if (o == 2)
      t = t - cy * (mvp * vp * D.msfvy(i, j + 1) * dfwd<R, 0, 1>(D, i, j, k) + mvm * vm * D.msfvy(i, j) * dfwd<R, 0, 1>(D, i, j - 1, k));
  }
  const R mup = c1f * D.muu.ld(i + 1, j, 0) + c2f, mum = c1f * D.muu.ld(i, j, 0) + c2f;
  const R up = k < nz ? D.u2.ld(i + 1, j, k) + D.u2.ld(i + 1, j, k - 1) : R(D.cfn) * D.u2.ld(i + 1, j, nz - 1) + R(D.cfn1) * D.u2.ld(i + 1, j, nz - 2);
  const R um = k < nz ? D.u2.ld(i, j, k) + D.u2.ld(i, j, k - 1) : R(D.cfn) * D.u2.ld(i, j, nz - 1) + R(D.cfn1) * D.u2.ld(i, j, nz - 2);
  const R cx = div_msf((k < nz ? R(0.25) : R(0.5)) * R(D.rdx), D.msfty(i, j));
  const int o = ph_horder(i, D.nx, D.spec_x, 1, OP && D.open_x);
  if (o == 6) t = t - cx * ((mup * up * D.msfux(i + 1, j) + mum * um * D.msfux(i, j)) * r60 * grad6<R, 1, 0>(D, i, j, k));
  else if (o == 2)
    t = t - cx * (mup * up * D.msfux(i + 1, j) * dfwd<R, 1, 0>(D, i, j, k) + mum * um * D.msfux(i, j) * dfwd<R, 1, 0>(D, i - 1, j, k));
  else if (o == 4) t = t - cx * ((mup * up * D.msfux(i + 1, j) + mum * um * D.msfux(i, j)) * r12 * grad4<R, 1, 0>(D, i, j, k));
  // open boundaries (:636-663, after the advection, south/north then west/east): inflow advection of ph by the
  // normal wind interpolated to the w level (top: level nz - 1, except the west lid level, which adds nothing)
  if (OP && D.open_y && (j == 0 || j == D.ny - 1)) {
    const int kz = k < nz - 1 ? k : nz - 1;
    const int a = j == 0 ? 0 : D.ny - 1, b = j == 0 ? 1 : D.ny;
    const R vb = R(0.5) * (R(D.fnm[kz]) * (D.v2.ld(i, b, kz) + D.v2.ld(i, a, kz)) +
                           R(D.fnp[kz]) * (D.v2.ld(i, b, kz - 1) + D.v2.ld(i, a, kz - 1)));
    const R muf = c1f * D.mut.ld(i, j, 0) + c2f;
    if (j == 0) {
      const R vl = vb < R(0) ? vb : R(0);
      t = t - R(D.rdy) * muf * (vl * (D.ph2.ld(i, 1, k) - D.ph2.ld(i, 0, k)));
    } else {
      const R vr = vb > R(0) ? vb : R(0);
      t = t - R(D.rdy) * muf * (vr * (D.ph2.ld(i, j, k) - D.ph2.ld(i, j - 1, k)));
    }
  }
  if (OP && D.open_x && (i == 0 || i == D.nx - 1) && !(i == 0 && k == nz)) {
    const int kz = k < nz ? k : nz - 1;
    const int a = i == 0 ? 0 : D.nx - 1, b = i == 0 ? 1 : D.nx;
    const R ub = R(0.5) * (R(D.fnm[kz]) * (D.u2.ld(b, j, kz) + D.u2.ld(a, j, kz)) +
                           R(D.fnp[kz]) * (D.u2.ld(b, j, kz - 1) + D.u2.ld(a, j, kz - 1)));
    const R muf = c1f * D.mut.ld(i, j, 0) + c2f;
    if (i == 0) {
      const R ul = ub < R(0) ? ub : R(0);
      t = t - (div_msf(D.msftx(i, j), D.msfty(i, j))) * R(D.rdx) * muf * (ul * (D.ph2.ld(1, j, k) - D.ph2.ld(0, j, k)));
    } else {
      const R ur = ub > R(0) ? ub : R(0);
      t = t - (div_msf(D.msftx(i, j), D.msfty(i, j))) * R(D.rdx) * muf * (ur * (D.ph2.ld(i, j, k) - D.ph2.ld(i - 1, j, k)));
    }
  }
  if (use_tendf) t = t + div_msf(D.ph_tendf.ld(i, j, k), D.msfty(i, j));
  return t;
}

// ------------------------------------------------------------------ lateral boundaries
// LateralBC (src/dyn/lateral_bc.cpp:21-196): the ring of a variable, slabs (pos, k, b) pos fastest;
// side order S, N, W, E = slabs ys, ye, xs, xe.
__device__ __forceinline__ int slab_of_side(int side) { return side < 2 ? side + 2 : side - 2; }
struct Ring {
  int ibe, jbe;
  __device__ __forceinline__ bool map(int pos, int side, int b, int& i, int& j) const {
    switch (side) {
      case 0: j = b; i = pos; return pos >= b && pos <= ibe - b;
      case 1: j = jbe - b; i = pos; return pos >= b && pos <= ibe - b;
      case 2: i = b; j = pos; return pos >= b + 1 && pos <= jbe - b - 1;
      default: i = ibe - b; j = pos; return pos >= b + 1 && pos <= jbe - b - 1;
    }
  }
};
__device__ __forceinline__ Ring ring_for(int nx, int ny, char var) {
  return Ring{var == 'u' ? nx : nx - 1, var == 'v' ? ny : ny - 1};
}
template <class R>
__device__ __forceinline__ R slab_at(const Slabs<R>& s, int tend, int sl, int pos, int k, int b) {
  const int np = s.npos[sl];
  return (tend ? s.t[sl] : s.v[sl])[pos + k * np + b * np * s.nk];
}
template <class R>
__device__ __forceinline__ R slab_val(const Slabs<R>& s, int sl, int pos, int k, int b, R dtbc) {
  return slab_at(s, 0, sl, pos, k, b) + dtbc * slab_at(s, 1, sl, pos, k, b);
}

// The ring row b and side / position of point (i, j) of a variable whose last indices are ibe, jbe (the
// inverse of Ring::map: south / north rows span pos = b .. ibe - b, west / east columns the rest).
__device__ __forceinline__ bool ring_locate(int ibe, int jbe, int i, int j, int& side, int& b, int& pos) {
  if (i < 0 || i > ibe || j < 0 || j > jbe) return false;
  const int dS = j, dN = jbe - j, dW = i, dE = ibe - i;
  const int dsn = dS < dN ? dS : dN, dwe = dW < dE ? dW : dE;
  if (dsn <= dwe) {
    b = dsn;
    side = dS <= dN ? 0 : 1;
    pos = i;
  } else {
    b = dwe;
    side = dW <= dE ? 2 : 3;
    pos = j;
  }
  return b < 5;
}

// KRelax (lateral_bc.cpp:79-118) at ring point (pos, side, b) level k of one variable: returns
// fa = fcx * fls0 and fb = gcx * (fls1 + fls2 + fls3 + fls4 - 4 fls0); the relaxation term is fa - fb.
template <class R, bool Two>
__device__ void relax_terms(const Dom<R>& D, const V3<R>& f, const double* c1, const double* c2, const Slabs<R>& s,
                            Ring r, int pos, int side, int b, int k, int i, int j, R& fa, R& fb) {
  const int sl = slab_of_side(side);
  const R dtbc = R(*D.dtbc);
  auto BV = [&](int p, int bb) { return slab_val(s, sl, p, k, bb, dtbc); };
  auto FV = [&](int ii, int jj) -> R {
    const R x = Two ? f.ld(ii, jj, 0) : f.ld(ii, jj, k);
    return c1 ? x * (R(c1[k]) * D.mut.ld(ii, jj, 0) + R(c2[k])) : x;
  };
  R fls0, fls1, fls2, fls3, fls4;
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
  fa = R(D.fcx[b]) * fls0;
  fb = R(D.gcx[b]) * (fls1 + fls2 + fls3 + fls4 - R(4) * fls0);
}

// The ring point (side, row b, pos) of (i, j) when it lies in rows b_lo .. b_hi of the variable's ring;
// then fa, fb of its relaxation term (relax_terms).
template <class R, bool Two>
__device__ __forceinline__ bool relax_at(const Dom<R>& D, const V3<R>& f, const double* c1, const double* c2,
                                         const Slabs<R>& s, Ring r, int i, int j, int k, R& fa, R& fb) {
  int side, b, pos;
  if (!ring_locate(r.ibe, r.jbe, i, j, side, b, pos) || b < 1 || b > 3) return false;
  relax_terms<R, Two>(D, f, c1, c2, s, r, pos, side, b, k, i, j, fa, fb);
  return true;
}
// (i, j) in the spec zone (row 0) of the ring: slab index sl and position pos of its boundary value
__device__ __forceinline__ bool spec_at(Ring r, int i, int j, int& sl, int& pos) {
  int side, b;
  if (!ring_locate(r.ibe, r.jbe, i, j, side, b, pos) || b != 0) return false;
  sl = slab_of_side(side);
  return true;
}

// LargeStep::tendencies (large_step.cpp:798-861): the five tendencies of a point, each for the points of
// its own range: ru (u_i0 .. u_i1), rv (v_j0 .. v_j1, 3-D), rw and ph (levels 1..nz), theta (mass cells).
// Also mu_tend = 0 (zero_tend of a run with lateral boundaries) at rk 2 and 3, and with lateral
// boundaries the spec zone's tendencies from the boundary slabs.
// PART: the tendencies a launch computes (1 u, 2 v, 4 w and phi, 8 theta and mu): the FP64 form runs the kernel as two
// launches, (u, v) and (w, phi, theta, mu), whose smaller code misses the instruction cache less (the same values)
template <class R, int NM, int SH, bool OP, int PART = 15>
__global__ void __launch_bounds__(PX, 10) k_tend(const __grid_constant__ Pack<R, NM> P, int rk) {
  constexpr bool PU = PART & 1, PV = PART & 2, PW = PART & 4, PT = PART & 8;
  constexpr int SX = shape_x(SH), SY = shape_y(SH);
  // the horizontal face fluxes of the block's tile, each evaluated once (u, v, w, theta): x faces i0 .. i0 + SX
  // of each row, y faces j0 .. j0 + SY of each column
  __shared__ R sfx[4][SY][SX + 1];
  __shared__ R sfy[4][SY + 1][SX];
  const Dom<R>* Dp;
  int i, j, k;
  Range r;
  const bool in = thread_index<SH>(P, RG_STAG, Dp, i, j, k, r);
  const Dom<R>& D = *Dp;
  const int tx = int(threadIdx.x) % SX, ty = int(threadIdx.x) / SX;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const bool use_tendf = D.lbc || D.dd_on;
  const int ui0 = D.bc_x != CW_BC_PERIODIC ? 1 : 0;
  const int vj0 = (D.bc_y != CW_BC_PERIODIC && D.do_y) ? 1 : 0;
  const bool dy = D.do_y;
  // the faces a point of each tendency's range uses (x faces f of its row, y faces f of its column), within the
  // member's range: up to the face after its last point, in its rows (x faces) / columns (y faces)
  const bool rx = j < r.j1, ry = i < r.i1;
  auto ux = [&](int f) { return rx && j < ny && k < nz && f >= ui0 && f <= nx && f <= r.i1; };
  auto uy = [&](int f) { return ry && dy && i >= ui0 && i < nx && k < nz && f >= 0 && f <= ny && f <= r.j1; };
  auto vx = [&](int f) { return rx && dy && j >= vj0 && j < ny && k < nz && f >= 0 && f <= nx && f <= r.i1; };
  auto vy = [&](int f) { return ry && dy && i < nx && k < nz && f >= vj0 && f <= ny && f <= r.j1; };
  auto wx = [&](int f) { return rx && j < ny && k >= 1 && f >= 0 && f <= nx && f <= r.i1; };
  auto wy = [&](int f) { return ry && dy && i < nx && k >= 1 && f >= 0 && f <= ny && f <= r.j1; };
  auto tx_ = [&](int f) { return rx && j < ny && k < nz && f >= 0 && f <= nx && f <= r.i1; };
  auto ty_ = [&](int f) { return ry && dy && i < nx && k < nz && f >= 0 && f <= ny && f <= r.j1; };
  // the tile's last column / row also takes the next face, in a loop: one call site per flux function, so that each
  // flux body is inlined once (the kernel's size is what its instruction-cache misses follow)
  const bool xe = tx == SX - 1, ye = ty == SY - 1;
#pragma unroll 1
  for (int e = 0; e <= int(xe); ++e) {
    const int f = i + e;
    if (PU && ux(f)) sfx[0][ty][tx + e] = tu_fx(D, f, j, k);
    if (PV && vx(f)) sfx[1][ty][tx + e] = tv_fx(D, f, j, k);
    if (PW && wx(f)) sfx[2][ty][tx + e] = tw_fx(D, f, j, k);
    if (PT && tx_(f)) sfx[3][ty][tx + e] = sc_fx(D, D.t2, D.ru, f, j, k, false);
  }
#pragma unroll 1
  for (int e = 0; e <= int(ye); ++e) {
    const int f = j + e;
    if (PU && uy(f)) sfy[0][ty + e][tx] = tu_fy(D, i, f, k);
    if (PV && vy(f)) sfy[1][ty + e][tx] = tv_fy(D, i, f, k);
    if (PW && wy(f)) sfy[2][ty + e][tx] = tw_fy(D, i, f, k);
    if (PT && ty_(f)) sfy[3][ty + e][tx] = sc_fy(D, D.t2, D.rv, i, f, k, false);
  }
  __syncthreads();
  if (!in) return;
  auto F = [&](int v, R& fx0, R& fx1, R& fy0, R& fy1) {
    fx0 = sfx[v][ty][tx];
    fx1 = sfx[v][ty][tx + 1];
    fy0 = sfy[v][ty][tx];
    fy1 = sfy[v][ty + 1][tx];
  };
  R fx0, fx1, fy0, fy1;
  const bool lbc = D.lbc;
  int sl, pos;
  // every tendency is computed before the first store (the stores cannot alias the loads then)
  // LateralBC::spec_dry (lateral_bc.cpp:337-351): the spec zone (row 0) takes the boundary tendency
  bool has_u = PU, has_v = PV;
  R tu = 0, tv = 0;
  if (!PU) {
  } else if (lbc && k < nz && spec_at(ring_for(nx, ny, 'u'), i, j, sl, pos)) {
    tu = slab_at(D.lbc_var[0], 1, sl, pos, k, 0);
  } else if (OP && D.open_x && (i == 0 || i == nx) && j < ny && k < nz) {  // open boundaries: the faces are advanced too
    tu = tend_u_open_face(D, i, j, k, use_tendf);
  } else if (i >= ui0 && i < nx && j < ny && k < nz) {
    F(0, fx0, fx1, fy0, fy1);
    tu = tend_u<OP>(D, i, j, k, use_tendf, fx0, fx1, fy0, fy1);
  } else {
    has_u = false;
  }
  if (!PV) {
  } else if (lbc && k < nz && spec_at(ring_for(nx, ny, 'v'), i, j, sl, pos)) {
    tv = slab_at(D.lbc_var[1], 1, sl, pos, k, 0);
  } else if (OP && dy && D.open_y && (j == 0 || j == ny) && i < nx && k < nz) {
    tv = tend_v_open_face(D, i, j, k, use_tendf);
  } else if (dy && i < nx && j >= vj0 && j < ny && k < nz) {
    F(1, fx0, fx1, fy0, fy1);
    tv = tend_v<OP>(D, i, j, k, use_tendf, fx0, fx1, fy0, fy1);
  } else {
    has_v = false;
  }
  const bool mass = (PW || PT) && i < nx && j < ny;
  const bool spec = mass && lbc && spec_at(ring_for(nx, ny, 'h'), i, j, sl, pos);
  R tw = 0, tp = 0, tt = 0, tm = 0;
  bool has_p = false, has_m = false;
  if (mass) {
    if (PW && k >= 1) {
      F(2, fx0, fx1, fy0, fy1);
      tw = tend_w<OP>(D, i, j, k, use_tendf, fx0, fx1, fy0, fy1);
    }
    if (!PW) {
    } else if (spec) {
      tp = slab_at(D.lbc_var[3], 1, sl, pos, k, 0);
      has_p = true;
    } else if (k >= 1) {
      tp = tend_ph<OP>(D, i, j, k, lbc);
      has_p = true;
    }
    if (PT && k < nz) {
      if (spec) {
        tt = slab_at(D.lbc_var[2], 1, sl, pos, k, 0);
      } else {
        F(3, fx0, fx1, fy0, fy1);
        tt = tend_t<OP>(D, i, j, k, use_tendf, D.n_moist > 0, fx0, fx1, fy0, fy1);
      }
    }
    if (PT && k == 0 && lbc) {
      if (spec) {
        tm = slab_at(D.lbc_var[4], 1, sl, pos, 0, 0);
        has_m = true;
      } else if (rk != 1) {
        has_m = true;
      }
    }
  }
  if (has_u) D.ru_tend(i, j, k) = tu;
  if (has_v) D.rv_tend(i, j, k) = tv;
  if (mass) {
    if (PW && k >= 1) D.rw_tend(i, j, k) = tw;
    if (has_p) D.ph_tend(i, j, k) = tp;
    if (PT && k < nz) D.t_tend(i, j, k) = tt;
    if (has_m) D.mu_tend(i, j, 0) = tm;
  }
}

// ------------------------------------------------------------------ constant-K diffusion (rk 1)
// DiffusionDriver::dynamics, diff_opt 1 / km_opt 1 (src/dyn/diffusion_driver.cpp:153-187) with the kernels
// of src/dyn/diffusion/big_step_diffusion.hpp:26-336. KIsotropicKm makes every eddy viscosity a constant
// (khdif, khdif / prandtl), so it is used directly. The held tendencies start from zero (init_zero_tendency,
// large_step.cpp:888-894), then the horizontal and vertical diffusion are added in the reference's order.
template <class R>
__device__ __forceinline__ R mk(const double* c1, const double* c2, const V3<R>& mut, int i, int j, int k) {
  return R(c1[k]) * mut.ld(i, j, 0) + R(c2[k]);
}
// the horizontal eddy viscosity at a mass point: the constant of km_opt 1 (KIsotropicKm, km_kh.hpp:35-45), or the
// per-point field that cal_dampkm raised near the top (damp_opt 1)
template <class R>
struct XkConst {
  R v;
  __device__ __forceinline__ R operator()(int, int, int) const { return v; }
};
template <class R>
struct XkField {
  V3<R> a;
  __device__ __forceinline__ R operator()(int i, int j, int k) const { return a.ld(i, j, k); }
};
template <class R, class XK>
__device__ R hdiff_u(const Dom<R>& D, const V3<R>& f, const V3<R>& mut, XK X, int i, int j, int k) {
  const double *c1 = D.c1h, *c2 = D.c2h;
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  const R mkrdxm = (div_msf(D.msftx(i - 1, j), D.msfty(i - 1, j))) * mk(c1, c2, mut, i - 1, j, k) * X(i - 1, j, k) * rdx;
  const R mkrdxp = (div_msf(D.msftx(i, j), D.msfty(i, j))) * mk(c1, c2, mut, i, j, k) * X(i, j, k) * rdx;
  const R mrdx = D.msfux(i, j) * D.msfuy(i, j) * rdx;
  const R mkrdym = ((D.msfuy(i, j) + D.msfuy(i, j - 1)) / (D.msfux(i, j) + D.msfux(i, j - 1))) * R(0.25) *
                   (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i - 1, j - 1, k) + mk(c1, c2, mut, i - 1, j, k)) *
                   R(0.25) * (X(i, j, k) + X(i, j - 1, k) + X(i - 1, j - 1, k) + X(i - 1, j, k)) * rdy;
  const R mkrdyp = ((D.msfuy(i, j) + D.msfuy(i, j + 1)) / (D.msfux(i, j) + D.msfux(i, j + 1))) * R(0.25) *
                   (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i - 1, j + 1, k) + mk(c1, c2, mut, i - 1, j, k)) *
                   R(0.25) * (X(i, j, k) + X(i, j + 1, k) + X(i - 1, j + 1, k) + X(i - 1, j, k)) * rdy;
  const R mrdy = D.msfux(i, j) * D.msfuy(i, j) * rdy;
  return mrdx * (mkrdxp * (f.ld(i + 1, j, k) - f.ld(i, j, k)) - mkrdxm * (f.ld(i, j, k) - f.ld(i - 1, j, k))) +
         mrdy * (mkrdyp * (f.ld(i, j + 1, k) - f.ld(i, j, k)) - mkrdym * (f.ld(i, j, k) - f.ld(i, j - 1, k)));
}
template <class R, class XK>
__device__ R hdiff_v(const Dom<R>& D, const V3<R>& f, const V3<R>& mut, XK X, int i, int j, int k) {
  const double *c1 = D.c1h, *c2 = D.c2h;
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  const R mkrdxm = ((D.msfvx(i, j) + D.msfvx(i - 1, j)) / (D.msfvy(i, j) + D.msfvy(i - 1, j))) * R(0.25) *
                   (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i - 1, j - 1, k) + mk(c1, c2, mut, i - 1, j, k)) *
                   R(0.25) * (X(i, j, k) + X(i, j - 1, k) + X(i - 1, j - 1, k) + X(i - 1, j, k)) * rdx;
  const R mkrdxp = ((D.msfvx(i, j) + D.msfvx(i + 1, j)) / (D.msfvy(i, j) + D.msfvy(i + 1, j))) * R(0.25) *
                   (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i + 1, j - 1, k) + mk(c1, c2, mut, i + 1, j, k)) *
                   R(0.25) * (X(i, j, k) + X(i, j - 1, k) + X(i + 1, j - 1, k) + X(i + 1, j, k)) * rdx;
  const R mrdx = D.msfvx(i, j) * D.msfvy(i, j) * rdx;
  const R mkrdym = (div_msf(D.msfty(i, j - 1), D.msftx(i, j - 1))) * X(i, j - 1, k) * rdy;
  const R mkrdyp = (div_msf(D.msfty(i, j), D.msftx(i, j))) * X(i, j, k) * rdy;
  const R mrdy = D.msfvx(i, j) * D.msfvy(i, j) * rdy;
  return mrdx * (mkrdxp * (f.ld(i + 1, j, k) - f.ld(i, j, k)) - mkrdxm * (f.ld(i, j, k) - f.ld(i - 1, j, k))) +
         mrdy * (mkrdyp * (f.ld(i, j + 1, k) - f.ld(i, j, k)) - mkrdym * (f.ld(i, j, k) - f.ld(i, j - 1, k)));
}
template <class R, class XK>
__device__ R hdiff_w(const Dom<R>& D, const V3<R>& f, const V3<R>& mut, XK X, int i, int j, int k) {
  const double *c1 = D.c1f, *c2 = D.c2f;
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  const R mkrdxm = (div_msf(D.msfux(i, j), D.msfuy(i, j))) * R(0.25) *
                   (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i - 1, j, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i - 1, j, k)) *
                   R(0.25) * (X(i, j, k) + X(i - 1, j, k) + X(i, j, k - 1) + X(i - 1, j, k - 1)) * rdx;
  const R mkrdxp = (div_msf(D.msfux(i + 1, j), D.msfuy(i + 1, j))) * R(0.25) *
                   (mk(c1, c2, mut, i + 1, j, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i + 1, j, k) + mk(c1, c2, mut, i, j, k)) *
                   R(0.25) * (X(i + 1, j, k) + X(i, j, k) + X(i + 1, j, k - 1) + X(i, j, k - 1)) * rdx;
  const R mrdx = D.msftx(i, j) * D.msfty(i, j) * rdx;
  const R mkrdym = (D.msfvy(i, j) * D.msfvx_inv(i, j)) * R(0.25) *
                   (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k)) *
                   R(0.25) * (X(i, j, k) + X(i, j - 1, k) + X(i, j, k - 1) + X(i, j - 1, k - 1)) * rdy;
  const R mkrdyp = (D.msfvy(i, j + 1) * D.msfvx_inv(i, j + 1)) * R(0.25) *
                   (mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i, j, k)) *
                   R(0.25) * (X(i, j + 1, k) + X(i, j, k) + X(i, j + 1, k - 1) + X(i, j, k - 1)) * rdy;
  const R mrdy = D.msftx(i, j) * D.msfty(i, j) * rdy;
  return mrdx * (mkrdxp * (f.ld(i + 1, j, k) - f.ld(i, j, k)) - mkrdxm * (f.ld(i, j, k) - f.ld(i - 1, j, k))) +
         mrdy * (mkrdyp * (f.ld(i, j + 1, k) - f.ld(i, j, k)) - mkrdym * (f.ld(i, j, k) - f.ld(i, j - 1, k)));
}
// KHorizDiffM1 (with_base = false) / KHorizDiff3DMP (base = t_init or qv_base)
template <class R, class XK>
__device__ R hdiff_m(const Dom<R>& D, const V3<R>& f, const VB<R>* base, const V3<R>& mut, XK X, int i, int j, int k) {
  const double *c1 = D.c1h, *c2 = D.c2h;
  const R rdx = R(D.rdx), rdy = R(D.rdy);
  const R mkrdxm = (div_msf(D.msfux(i, j), D.msfuy(i, j))) * R(0.5) * (X(i, j, k) + X(i - 1, j, k)) * R(0.5) * (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i - 1, j, k)) * rdx;
  const R mkrdxp = (div_msf(D.msfux(i + 1, j), D.msfuy(i + 1, j))) * R(0.5) * (X(i + 1, j, k) + X(i, j, k)) * R(0.5) * (mk(c1, c2, mut, i + 1, j, k) + mk(c1, c2, mut, i, j, k)) * rdx;
  const R mrdx = D.msftx(i, j) * D.msfty(i, j) * rdx;
  const R mkrdym = (D.msfvy(i, j) * D.msfvx_inv(i, j)) * R(0.5) * (X(i, j, k) + X(i, j - 1, k)) * R(0.5) * (mk(c1, c2, mut, i, j, k) + mk(c1, c2, mut, i, j - 1, k)) * rdy;
  const R mkrdyp = (D.msfvy(i, j + 1) * D.msfvx_inv(i, j + 1)) * R(0.5) * (X(i, j + 1, k) + X(i, j, k)) * R(0.5) * (mk(c1, c2, mut, i, j + 1, k) + mk(c1, c2, mut, i, j, k)) * rdy;
  const R mrdy = D.msftx(i, j) * D.msfty(i, j) * rdy;
  if (!base)
    return mrdx * (mkrdxp * (f.ld(i + 1, j, k) - f.ld(i, j, k)) - mkrdxm * (f.ld(i, j, k) - f.ld(i - 1, j, k))) +
           mrdy * (mkrdyp * (f.ld(i, j + 1, k) - f.ld(i, j, k)) - mkrdym * (f.ld(i, j, k) - f.ld(i, j - 1, k)));
  const VB<R>& b = *base;
  const R dxp = f.ld(i + 1, j, k) - f.ld(i, j, k) - b(i + 1, j, k) + b(i, j, k);
  const R dxm = f.ld(i, j, k) - f.ld(i - 1, j, k) - b(i, j, k) + b(i - 1, j, k);
  const R dyp = f.ld(i, j + 1, k) - f.ld(i, j, k) - b(i, j + 1, k) + b(i, j, k);
  const R dym = f.ld(i, j, k) - f.ld(i, j - 1, k) - b(i, j, k) + b(i, j - 1, k);
  return mrdx * (mkrdxp * dxp - mkrdxm * dxm) + mrdy * (mkrdyp * dyp - mkrdym * dym);
}
// the vertical diffusion flux of a column at interface k (vflux[k] of the reference's column kernels)
template <class R>
__device__ __forceinline__ R vflux_w(const Dom<R>& D, const V3<R>& f, R kv, int i, int j, int k) {
  if (k >= D.nz - 1) return 0;
  return (kv / D.alt.ld(i, j, k)) * R(D.rdnw[k]) * (f.ld(i, j, k + 1) - f.ld(i, j, k));
}
template <class R>
__device__ __forceinline__ R vflux_m(const Dom<R>& D, const V3<R>& f, const VB<R>* base, R kv, int i, int j, int k) {
  if (k >= D.nz - 1) return 0;
  const R dpert = base ? f.ld(i, j, k + 1) - f.ld(i, j, k) - (*base)(i, j, k + 1) + (*base)(i, j, k) : f.ld(i, j, k + 1) - f.ld(i, j, k);
  return kv * R(D.rdn[k + 1]) / (R(0.5) * (D.alt.ld(i, j, k) + D.alt.ld(i, j, k + 1))) * dpert;
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R vflux_uv(const Dom<R>& D, const V3<R>& f, const double* ub, R kv, int i, int j, int k) {
  if (k >= D.nz - 1) return 0;
  const R a = R(0.25) * (D.alt.ld(i, j, k) + D.alt.ld(i - DI, j - DJ, k) + D.alt.ld(i, j, k + 1) + D.alt.ld(i - DI, j - DJ, k + 1));
  const R dpert = f.ld(i, j, k + 1) - f.ld(i, j, k) - R(ub[k + 1]) + R(ub[k]);
  return kv * R(D.rdn[k + 1]) / a * dpert;
}
// vertical_diffusion 'w' (KVertDiffW1), 'm' / mp (KVertDiffM1 / MP1), u / v (KVertDiffU1 / V1): the
// increment of level k
template <class R>
__device__ __forceinline__ R vdiff_w(const Dom<R>& D, const V3<R>& f, const V3<R>& mut, R kv, int i, int j, int k) {
  const R G = R(k::g);
  const R mu = R(D.c1f[k]) * mut.ld(i, j, 0) + R(D.c2f[k]);
  const R alt_avg = R(0.5) * (D.alt.ld(i, j, k) + D.alt.ld(i, j, k - 1));
  return R(D.rdn[k]) * G * G / mu / alt_avg * (vflux_w(D, f, kv, i, j, k) - vflux_w(D, f, kv, i, j, k - 1));
}
template <class R>
__device__ __forceinline__ R vdiff_m(const Dom<R>& D, const V3<R>& f, const VB<R>* base, const V3<R>& mut, R kv, int i, int j, int k) {
  const R G = R(k::g);
  if (k == 0) {
    const R vf0 = vflux_m(D, f, base, kv, i, j, 0);
    return G * G / (R(D.c1h[0]) * mut.ld(i, j, 0) + R(D.c2h[0])) / D.alt.ld(i, j, 0) * R(D.rdnw[0]) * (vf0 - vf0);
  }
  const R mu = R(D.c1h[k]) * mut.ld(i, j, 0) + R(D.c2h[k]);
  return G * G / mu / D.alt.ld(i, j, k) * R(D.rdnw[k]) * (vflux_m(D, f, base, kv, i, j, k) - vflux_m(D, f, base, kv, i, j, k - 1));
}
template <class R, int DI, int DJ>
__device__ __forceinline__ R vdiff_uv(const Dom<R>& D, const V3<R>& f, const double* ub, const V3<R>& muf, R kv, int i, int j, int k) {
  const R G = R(k::g);
  if (k == 0) {
    const R vf0 = vflux_uv<R, DI, DJ>(D, f, ub, kv, i, j, 0);
    return G * G * R(D.rdnw[0]) / (R(D.c1h[0]) * muf.ld(i, j, 0) + R(D.c2h[0])) /
           (R(0.5) * (D.alt.ld(i - DI, j - DJ, 0) + D.alt.ld(i, j, 0))) * (vf0 - vf0);
  }
  const R mu = R(D.c1h[k]) * muf.ld(i, j, 0) + R(D.c2h[k]);
  const R a = R(0.5) * (D.alt.ld(i - DI, j - DJ, k) + D.alt.ld(i, j, k));
  return G * G * R(D.rdnw[k]) / mu / a * (vflux_uv<R, DI, DJ>(D, f, ub, kv, i, j, k) - vflux_uv<R, DI, DJ>(D, f, ub, kv, i, j, k - 1));
}

// rk 1: zero the held tendencies, add the constant-K diffusion; with lateral boundaries mu_tend = 0 and the
// relaxation of rows 1..3 (LateralBC::relax_dry, lateral_bc.cpp:294-335) added to the held tendencies
// sixth_order_diffusion (src/dyn/diffusion/sixth_order.hpp:13-183): the sixth-order horizontal filter of the first
// RK stage. d6(f, c) is the flux difference of the face below point c along (DI, DJ), zeroed against the local
// gradient when flux-limited (diff_6th_opt 2); the kinds differ in the masses averaged to the faces.
template <class R, int DI, int DJ>
__device__ __forceinline__ R d6(const V3<R>& f, int i, int j, int k, int opt) {
  auto F = [&](int s) { return f.ld(i + s * DI, j + s * DJ, k); };
  R d = R(10.0) * (F(0) - F(-1)) - R(5.0) * (F(1) - F(-2)) + (F(2) - F(-3));
  if (opt == 2 && d * (F(0) - F(-1)) <= R(0)) d = R(0);
  return d;
}
// the filter's index ranges (sixth_order.hpp:174-205): kind 'u', 'v', or 'm' (also w's levels 1..nz-1); open
// sides start 3 rows in and end 3 (u, v along their stagger) or 4 rows in, 'v' with open x takes the specified
// limits on all four sides
__device__ __forceinline__ bool d6_in(char kind, int nx, int ny, bool sp, bool px, bool ox, bool oy, int i, int j) {
  int is = 0, js = 0, ie, je;
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
  }
  return i >= is && i < ie && j >= js && j < je;
}
// the x and y parts of the filter's tendency at (i, j, k) (KSixthOrderU / V / M), coef = factor / 64 / (2 dt)
template <class R>
__device__ __forceinline__ void d6_tend(const Dom<R>& D, char kind, const V3<R>& f, const V3<R>& mut, const double* c1v,
                                        const double* c2v, R coef, int i, int j, int k, R& tx, R& ty) {
  const int opt = D.diff_6th_opt;
  const R c1 = R(c1v[k]), c2 = R(c2v[k]);
  auto M = [&](int a, int b) { return c1 * mut.ld(a, b, 0) + c2; };
  const R fx0 = d6<R, 1, 0>(f, i, j, k, opt), fx1 = d6<R, 1, 0>(f, i + 1, j, k, opt);
  const R fy0 = d6<R, 0, 1>(f, i, j, k, opt), fy1 = d6<R, 0, 1>(f, i, j + 1, k, opt);
  R mx0, mx1, my0, my1, sx, sy;
  if (kind == 'u') {
    mx0 = M(i - 1, j);
    mx1 = M(i, j);
    my0 = R(0.25) * (M(i - 1, j - 1) + M(i, j - 1) + M(i - 1, j) + M(i, j));
    my1 = R(0.25) * (M(i - 1, j) + M(i, j) + M(i - 1, j + 1) + M(i, j + 1));
    sx = D.msfux(i, j);
    sy = D.msfuy(i, j);
  } else if (kind == 'v') {
    mx0 = R(0.25) * (M(i - 1, j - 1) + M(i, j - 1) + M(i - 1, j) + M(i, j));
    mx1 = R(0.25) * (M(i, j - 1) + M(i + 1, j - 1) + M(i, j) + M(i + 1, j));
    my0 = M(i, j - 1);
    my1 = M(i, j);
    sx = D.msfvx(i, j);
    sy = D.msfvy(i, j);
  } else {
    mx0 = R(0.5) * (M(i - 1, j) + M(i, j));
    mx1 = R(0.5) * (M(i, j) + M(i + 1, j));
    my0 = R(0.5) * (M(i, j - 1) + M(i, j));
    my1 = R(0.5) * (M(i, j) + M(i, j + 1));
    sx = D.msftx(i, j);
    sy = D.msfty(i, j);
  }
  tx = coef * sx * (mx1 * fx1 - mx0 * fx0);
  ty = coef * sy * (my1 * fy1 - my0 * fy0);
}
template <class R>
__device__ __forceinline__ R d6_coef(const Dom<R>& D, R dt) {
  return R(D.diff_6th_factor) * R(0.015625) / (R(2.0) * dt);
}

// rk_rayleigh_damp, damp_opt 2 (src/dyn/diffusion/rayleigh_damp.hpp:26-245): at the first RK stage u, v, w and theta
// relax toward the base-state profile in the upper zdamp metres, with weight dampcoef sin^2(pi/2 (1 - (ztop - z) /
// zdamp)). Restated per point: the reference walks down each column from the top while the level's height is
// within zdamp of the top; level k >= 1 is damped when every level from k to the top is. The base value at the
// height is interpolated linearly in z_base. sin = cw_sin.
template <class R>
__device__ R ray_weight(const Dom<R>& D, R ztop, R z) {
  const R ratio = (ztop - z) / R(D.zdamp);
  const R m = ratio < R(1.0) ? ratio : R(1.0);
  const R dcoef = R(1.0) - m;
  const R s = R(cw_sin(double(R(0.5) * R(0x1.921fb54442d18p+1) * dcoef)));  // 2 asin(1) = pi
  return s * s;
}
// the u / v / theta term mu (w dampcoef) (val - base(z)) of level k, zlev(kk) the column's level heights; false when
// the level is not damped
template <class R, class Z>
__device__ bool ray_term(const Dom<R>& D, const double* base, R ztop, Z zlev, R mu, R val, int k, R& term) {
  const int ktf = D.nz - 1;
  if (k < 1) return false;
  const R thr = ztop - R(D.zdamp);
  for (int kk = ktf; kk >= k; --kk)
    if (!(zlev(kk) >= thr)) return false;
  const R z = zlev(k);
  int k2 = ktf;
  while (k2 > 0 && R(D.z_base[k2]) > z) k2 = k2 - 1;
  R b;
  if (k2 + 1 > ktf)
    b = R(base[k2]) + (R(base[k2]) - R(base[k2 - 1])) * (z - R(D.z_base[k2])) / (R(D.z_base[k2]) - R(D.z_base[k2 - 1]));
  else
    b = R(base[k2]) + (R(base[k2 + 1]) - R(base[k2])) * (z - R(D.z_base[k2])) / (R(D.z_base[k2 + 1]) - R(D.z_base[k2]));
  term = mu * (ray_weight(D, ztop, z) * R(D.dampcoef)) * (val - b);
  return true;
}
template <class R>
__device__ __forceinline__ R phz(const Dom<R>& D, int i, int j, int k) { return D.phb(i, j, k) + D.ph2.ld(i, j, k); }
// the column pair (a, b) of a u (v) point along its direction, as KRayleighDampU (V) picks it
__device__ __forceinline__ void ray_pair(int i, int n, bool periodic, int& a, int& b) {
  a = (i == n) ? (periodic ? 0 : n - 1) : i;
  b = (i == 0) ? (periodic ? n - 1 : 0) : i - 1;
}
template <class R>
__device__ bool ray_u(const Dom<R>& D, int i, int j, int k, R& term) {
  const int nz = D.nz;
  int a, b;
  ray_pair(i, D.nx, D.bc_x == CW_BC_PERIODIC, a, b);
  const R ztop = R(0.5) * (D.phb(a, j, nz) + D.phb(b, j, nz) + D.ph2.ld(a, j, nz) + D.ph2.ld(b, j, nz)) / R(k::g);
  auto zlev = [&](int kk) {
    return R(0.25) * (D.phb(a, j, kk) + D.phb(a, j, kk + 1) + D.phb(b, j, kk) + D.phb(b, j, kk + 1) + D.ph2.ld(a, j, kk) +
                      D.ph2.ld(a, j, kk + 1) + D.ph2.ld(b, j, kk) + D.ph2.ld(b, j, kk + 1)) / R(k::g);
  };
  return ray_term(D, D.u_base, ztop, zlev, R(D.c1h[k]) * D.muu.ld(i, j, 0) + R(D.c2h[k]), D.u2.ld(i, j, k), k, term);
}
template <class R>
__device__ bool ray_v(const Dom<R>& D, int i, int j, int k, R& term) {
  const int nz = D.nz;
  int a, b;
  ray_pair(j, D.ny, D.bc_y == CW_BC_PERIODIC, a, b);
  const R ztop = R(0.5) * (D.phb(i, a, nz) + D.phb(i, b, nz) + D.ph2.ld(i, a, nz) + D.ph2.ld(i, b, nz)) / R(k::g);
  auto zlev = [&](int kk) {
    return R(0.25) * (D.phb(i, a, kk) + D.phb(i, a, kk + 1) + D.phb(i, b, kk) + D.phb(i, b, kk + 1) + D.ph2.ld(i, a, kk) +
                      D.ph2.ld(i, a, kk + 1) + D.ph2.ld(i, b, kk) + D.ph2.ld(i, b, kk + 1)) / R(k::g);
  };
  return ray_term(D, D.v_base, ztop, zlev, R(D.c1h[k]) * D.muv.ld(i, j, 0) + R(D.c2h[k]), D.v2.ld(i, j, k), k, term);
}
template <class R>
__device__ bool ray_t(const Dom<R>& D, int i, int j, int k, R& term) {
  const R ztop = phz(D, i, j, D.nz) / R(k::g);
  auto zlev = [&](int kk) {
    return R(0.5) * (D.phb(i, j, kk) + D.phb(i, j, kk + 1) + D.ph2.ld(i, j, kk) + D.ph2.ld(i, j, kk + 1)) / R(k::g);
  };
  return ray_term(D, D.t_base, ztop, zlev, R(D.c1h[k]) * D.mut.ld(i, j, 0) + R(D.c2h[k]), D.t2.ld(i, j, k), k, term);
}
// w: every level (0..nz) within zdamp of the top, toward w = 0
template <class R>
__device__ bool ray_w(const Dom<R>& D, int i, int j, int k, R& term) {
  const R ztop = phz(D, i, j, D.nz) / R(k::g), z = phz(D, i, j, k) / R(k::g);
  if (!(z >= ztop - R(D.zdamp))) return false;
  term = (R(D.c1f[k]) * D.mut.ld(i, j, 0) + R(D.c2f[k])) * (ray_weight(D, ztop, z) * R(D.dampcoef)) * D.w2.ld(i, j, k);
  return true;
}

// ------------------------------------------------------------------ km_opt 4 (diff_opt 1)
// DiffusionDriver::prepare with km_opt 4: the 2-D Smagorinsky eddy viscosities (KSmag2dKm, km_kh.hpp:47-97) from the
// deformation defor11, defor22 (KDeformDiagAndDiv, deform_div.hpp:20-84) and defor12 (KDeform12 :86-156, with the
// edge copies of cal_deform_and_div :271-318) with their terrain terms from compute_diff_metrics' rdzw, zx, zy
// (diff_metrics.hpp:11-133, with set_physical_bc3d). Every one of them depends only on its neighbours' u, v, ph:
// they are evaluated where they are needed, in the reference's expressions, one thread per mass point.
template <class R>
__device__ __forceinline__ R dm_zw(const Dom<R>& D, int i, int j, int k) {
  return (D.ph2.ld(i, j, k) + D.phb(i, j, k)) / R(k::g);
}
template <class R>
__device__ __forceinline__ R dm_rdzw(const Dom<R>& D, int i, int j, int k) {
  return R(1.0) / (dm_zw(D, i, j, k + 1) - dm_zw(D, i, j, k));
}
// zx at U points i = 0..nx (KDiffMetricsZX; the boundary faces of specified / open sides copy the last column)
template <class R>
__device__ R dm_zx(const Dom<R>& D, int i, int j, int k) {
  const int nx = D.nx;
  const bool px = D.bc_x == CW_BC_PERIODIC, copy = D.lbc || D.open_x;
  if (px && k == D.nz && (i == 0 || i == nx)) return R(0);
  if (!px && (i == 0 || (i == nx && !copy))) return R(0);
  int i0 = i, im1 = i - 1;
  if (!px && i == nx) {
    i0 = nx - 1;
    im1 = nx - 2;
  } else {
    if (i == nx) i0 = 0;
    if (i == 0) im1 = nx - 1;
  }
  R v = R(D.rdx) * (D.phb(i0, j, k) - D.phb(im1, j, k)) / R(k::g);
  v += R(D.rdx) * (D.ph2.ld(i0, j, k) - D.ph2.ld(im1, j, k)) / R(k::g);
  return v;
}
// zy at V points j = 0..ny (KDiffMetricsZY)
template <class R>
__device__ R dm_zy(const Dom<R>& D, int i, int j, int k) {
  const int ny = D.ny;
  const bool py = D.bc_y == CW_BC_PERIODIC, copy = D.lbc || D.open_y;
  if (py && k == D.nz && (j == 0 || j == ny)) return R(0);
  if (!py && (j == 0 || (j == ny && !copy))) return R(0);
  int j0 = j, jm1 = j - 1;
  if (!py && j == ny) {
    j0 = ny - 1;
    jm1 = ny - 2;
  } else {
    if (j == ny) j0 = 0;
    if (j == 0) jm1 = ny - 1;
  }
  R v = R(D.rdy) * (D.phb(i, j0, k) - D.phb(i, jm1, k)) / R(k::g);
  v += R(D.rdy) * (D.ph2.ld(i, j0, k) - D.ph2.ld(i, jm1, k)) / R(k::g);
  return v;
}
// the average of two columns a(0, .), a(1, .) at w level k (the hatavg arrays of cal_deform_and_div)
template <class R, class A>
__device__ __forceinline__ R dm_hatavg(const Dom<R>& D, const A& a, int k) {
  const int nz = D.nz;
  if (k == 0)
    return R(0.5) * (R(D.cf1) * a(0, 0) + R(D.cf2) * a(0, 1) + R(D.cf3) * a(0, 2) + R(D.cf1) * a(1, 0) +
                     R(D.cf2) * a(1, 1) + R(D.cf3) * a(1, 2));
  if (k == nz) {
    const R cft2 = -R(0.5) * R(D.dnw[nz - 1]) / R(D.dn[nz - 1]), cft1 = R(1.0) - cft2;
    return R(0.5) * (cft1 * (a(0, nz - 1) + a(1, nz - 1)) + cft2 * (a(0, nz - 2) + a(1, nz - 2)));
  }
  return R(0.5) * (R(D.fnm[k]) * (a(0, k) + a(1, k)) + R(D.fnp[k]) * (a(0, k - 1) + a(1, k - 1)));
}
// defor12 at vorticity point (ci, cj), level k, after the edge copies: the point computed there
template <class R>
__device__ R dm_defor12(const Dom<R>& D, int ci, int cj, int k) {
  const int nx = D.nx, ny = D.ny;
  const bool px = D.bc_x == CW_BC_PERIODIC, py = D.bc_y == CW_BC_PERIODIC;
  const bool bx = !px && (D.lbc || D.open_x), by = !py && (D.lbc || D.open_y);
  int i = ci, j = cj;
  if (px) {
    if (i == nx) i = 0;
  } else if (bx) {
    if (i == 0) i = 1;
    if (i == nx) i = nx - 1;
  }
  if (py) {
    if (j == ny) j = 0;
  } else if (by) {
    if (j == 0) j = 1;
    if (j == ny) j = ny - 1;
  }
  const int im1 = i == 0 ? (px ? nx - 1 : 0) : i - 1, i0 = i == nx ? (px ? 0 : nx - 1) : i;
  const int jm1 = j == 0 ? (py ? ny - 1 : 0) : j - 1, j0 = j == ny ? (py ? 0 : ny - 1) : j;
  const R mm = R(0.25) * (D.msfux(i, jm1) + D.msfux(i, j0)) * (D.msfvy(im1, j) + D.msfvy(i0, j));
  auto hu = [&](int c, int kk) { const int m = c ? j0 : jm1; return div_msf(D.u2.ld(i, m, kk), D.msfux(i, m)); };
  auto hv = [&](int c, int kk) { const int m = c ? i0 : im1; return div_msf(D.v2.ld(m, j, kk), D.msfvy(m, j)); };
  const R tmpzy = R(0.25) * (dm_zy(D, im1, j, k) + dm_zy(D, i0, j, k) + dm_zy(D, im1, j, k + 1) + dm_zy(D, i0, j, k + 1));
  const R r00 = dm_rdzw(D, i0, j0, k), r10 = dm_rdzw(D, im1, j0, k), r11 = dm_rdzw(D, im1, jm1, k),
          r01 = dm_rdzw(D, i0, jm1, k);
  const R tmp1_u = (dm_hatavg(D, hu, k + 1) - dm_hatavg(D, hu, k)) * R(0.25) * tmpzy * (r00 + r10 + r11 + r01);
  const R term_u = mm * (R(D.rdy) * (hu(1, k) - hu(0, k)) - tmp1_u);
  const R tmpzx = R(0.25) * (dm_zx(D, i, jm1, k) + dm_zx(D, i, j0, k) + dm_zx(D, i, jm1, k + 1) + dm_zx(D, i, j0, k + 1));
  const R tmp1_v = (dm_hatavg(D, hv, k + 1) - dm_hatavg(D, hv, k)) * R(0.25) * tmpzx * (r00 + r01 + r11 + r10);
  const R term_v = mm * (R(D.rdx) * (hv(1, k) - hv(0, k)) - tmp1_v);
  return term_u + term_v;
}
// calculate_km_kh with km_opt 4 (km_kh.hpp:585-625): KSmag2dKm one row inside open and specified sides, 0 elsewhere
// (the reference zeroes the outermost rows of specified boundaries and never writes those of open ones)
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX) k_smag(const __grid_constant__ Pack<R, NM> P) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_MASS, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  if (D.km_opt != 4 || !D.diff_on) return;
  const int nx = D.nx, ny = D.ny;
  const bool bx = D.lbc || D.open_x, by = D.lbc || D.open_y;
  int is = bx ? 1 : 0, ie = bx ? nx - 1 : nx;
  const int js = by ? 1 : 0, je = by ? ny - 1 : ny;
  if (D.bc_x == CW_BC_PERIODIC) {
    is = 0;
    ie = nx;
  }
  if (!(i >= is && i < ie && j >= js && j < je)) {
    D.xkmh(i, j, k) = R(0);
    D.xkhh(i, j, k) = R(0);
    return;
  }
  const R mm = D.msftx(i, j) * D.msfty(i, j);
  auto au = [&](int c, int kk) { return div_msf(D.u2.ld(i + c, j, kk), D.msfuy(i + c, j)); };
  auto av = [&](int c, int kk) { return div_msf(D.v2.ld(i, j + c, kk), D.msfvx(i, j + c)); };
  const R rdzw = dm_rdzw(D, i, j, k);
  const R tmpzx = R(0.25) * (dm_zx(D, i, j, k) + dm_zx(D, i + 1, j, k) + dm_zx(D, i, j, k + 1) + dm_zx(D, i + 1, j, k + 1));
  const R tmp1_u = (dm_hatavg(D, au, k + 1) - dm_hatavg(D, au, k)) * tmpzx * rdzw;
  const R d11 = R(2.0) * (mm * (R(D.rdx) * (au(1, k) - au(0, k)) - tmp1_u));
  const R tmpzy = R(0.25) * (dm_zy(D, i, j, k) + dm_zy(D, i, j + 1, k) + dm_zy(D, i, j, k + 1) + dm_zy(D, i, j + 1, k + 1));
  const R tmp1_v = (dm_hatavg(D, av, k + 1) - dm_hatavg(D, av, k)) * tmpzy * rdzw;
  const R d22 = R(2.0) * (mm * (R(D.rdy) * (av(1, k) - av(0, k)) - tmp1_v));
  const R dd = d11 - d22;
  R def2 = R(0.25) * (dd * dd);
  const R d12 = R(0.25) * (dm_defor12(D, i, j, k) + dm_defor12(D, i, j + 1, k) + dm_defor12(D, i + 1, j, k) +
                           dm_defor12(D, i + 1, j + 1, k));
  def2 += d12 * d12;
  const R mlen_h = sqrt(div_msf(div_msf(R(D.dx), D.msftx(i, j)) * R(D.dy), D.msfty(i, j)));
  const R tmp = sqrt(def2);
  R kmh = R(0.25) * R(0.25) * mlen_h * mlen_h * tmp;
  kmh = kmh < R(10.0) * mlen_h ? kmh : R(10.0) * mlen_h;
  D.xkmh(i, j, k) = kmh;
  D.xkhh(i, j, k) = kmh / R(D.prandtl);
}

template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX, 10) k_tendf_rk1(const __grid_constant__ Pack<R, NM> P) {
  const Dom<R>* Dp;
  int i, j, k;
  if (!thread_index<SH>(P, RG_STAG, Dp, i, j, k)) return;
  const Dom<R>& D = *Dp;
  const int nx = D.nx, ny = D.ny, nz = D.nz, nyv = D.nyv;
  const bool dd = D.diff_on;
  const bool sp = D.lbc;  // specified boundaries (relaxation; the diffusion's index ranges)
  const bool px = D.bc_x == CW_BC_PERIODIC, ox = D.open_x, oy = D.open_y;
  // horizontal_diffusion / vertical_diffusion_u, _v loop limits (big_step_diffusion.hpp:359-398, :459-500): one row
  // in on the open sides, and on every side when any side is specified
  const bool bx = sp || ox, by = sp || oy;
  const R khdif = R(D.khdif), kvdif = R(D.kvdif);
  const R khh = R(D.khdif / D.prandtl);
  const bool d6on = D.diff_6th_opt != 0 && D.diff_6th_factor != 0.0;  // sixth_order_diffusion (diffusion_driver.cpp:266-280)
  const R c6 = d6_coef(D, R(D.dt));
  if (j < ny && k < nz) {  // ru_tendf: U points [0, nx] x [0, ny) x [0, nz)
    R t = 0;
    if (dd) {
      int is = bx ? 1 : 0, ie = bx ? nx : nx + 1;
      const int js = by ? 1 : 0, je = by ? ny - 1 : ny;
      if (px) { is = 0; ie = nx + 1; }
      if (i >= is && i < ie && j >= js && j < je) {
        if (D.xk_field) t += hdiff_u(D, D.u2, D.mut, XkField<R>{D.xkmh}, i, j, k);
        else t += hdiff_u(D, D.u2, D.mut, XkConst<R>{khdif}, i, j, k);
      }
      int vis = bx ? 1 : 0, vie = bx ? nx : nx + 1;
      if (px) { vis = 0; vie = nx + 1; }
      if (i >= vis && i < vie && k < nz - 1) t += vdiff_uv<R, 1, 0>(D, D.u2, D.u_base, D.muu, kvdif, i, j, k);
    }
    if (d6on && d6_in('u', nx, ny, sp, px, ox, oy, i, j)) {
      R tx, ty;
      d6_tend(D, 'u', D.u2, D.mut, D.c1h, D.c2h, c6, i, j, k, tx, ty);
      t = t + tx + ty;
    }
    R rt;
    if (D.damp_opt == 2 && ray_u(D, i, j, k, rt)) t = t - rt;
    R fa, fb;
    if (sp && relax_at<R, false>(D, D.ru, nullptr, nullptr, D.lbc_var[0], ring_for(nx, ny, 'u'), i, j, k, fa, fb))
      t += (fa - fb) * D.msfuy(i, j);
    D.ru_tendf(i, j, k) = t;
  }
  if (i < nx && j < nyv && k < nz) {  // rv_tendf
    R t = 0;
    if (dd && D.do_y) {
      int is = bx ? 1 : 0, ie = bx ? nx - 1 : nx;
      const int js = by ? 1 : 0, je = by ? ny : ny + 1;
      if (px) { is = 0; ie = nx; }
      if (i >= is && i < ie && j >= js && j < je) {
        if (D.xk_field) t += hdiff_v(D, D.v2, D.mut, XkField<R>{D.xkmh}, i, j, k);
        else t += hdiff_v(D, D.v2, D.mut, XkConst<R>{khdif}, i, j, k);
      }
      const int vjs = by ? 1 : 0, vje = by ? ny : ny + 1;
      if (j >= vjs && j < vje && k < nz - 1) t += vdiff_uv<R, 0, 1>(D, D.v2, D.v_base, D.muv, kvdif, i, j, k);
    }
    if (d6on && D.do_y && d6_in('v', nx, ny, sp, px, ox, oy, i, j)) {
      R tx, ty;
      d6_tend(D, 'v', D.v2, D.mut, D.c1h, D.c2h, c6, i, j, k, tx, ty);
      t = t + tx + ty;
    }
    R rt;
    if (D.damp_opt == 2 && ray_v(D, i, j, k, rt)) {
      t = t - rt;
      if (D.two_d) t = t - rt;  // the reference's columns j = 0 and j = ny are the same storage in 2-D
    }
    R fa, fb;
    if (sp && relax_at<R, false>(D, D.rv, nullptr, nullptr, D.lbc_var[1], ring_for(nx, ny, 'v'), i, j, k, fa, fb))
      t += (fa - fb) * D.msfvx(i, j);
    D.rv_tendf(i, j, k) = t;
  }
  if (i < nx && j < ny) {
    R tw = 0;
    if (dd && k >= 1 && k < nz) {
      int is = bx ? 1 : 0, ie = bx ? nx - 1 : nx;
      const int js = by ? 1 : 0, je = by ? ny - 1 : ny;
      if (px) { is = 0; ie = nx; }
      if (i >= is && i < ie && j >= js && j < je) {
        if (D.xk_field) tw += hdiff_w(D, D.w2, D.mut, XkField<R>{D.xkmh}, i, j, k);
        else tw += hdiff_w(D, D.w2, D.mut, XkConst<R>{khdif}, i, j, k);
      }
      tw += vdiff_w(D, D.w2, D.mut, kvdif, i, j, k);
    }
    if (d6on && k >= 1 && k < nz && d6_in('m', nx, ny, sp, px, ox, oy, i, j)) {
      R tx, ty;
      d6_tend(D, 'w', D.w2, D.mut, D.c1f, D.c2f, c6, i, j, k, tx, ty);
      tw = tw + tx + ty;
    }
    R rt;
    if (D.damp_opt == 2 && ray_w(D, i, j, k, rt)) tw = tw - rt;
    D.rw_tendf(i, j, k) = tw;
    R fa, fb;
    R tp = 0;
    if (sp && relax_at<R, false>(D, D.ph2, D.c1f, D.c2f, D.lbc_var[3], ring_for(nx, ny, 'h'), i, j, k, fa, fb)) tp += fa - fb;
    D.ph_tendf(i, j, k) = tp;
    if (k < nz) {
      R tt = 0;
      if (dd) {
        int is = bx ? 1 : 0, ie = bx ? nx - 1 : nx;
        const int js = by ? 1 : 0, je = by ? ny - 1 : ny;
        if (px) { is = 0; ie = nx; }
        if (i >= is && i < ie && j >= js && j < je) {
          if (D.xk_field) tt += hdiff_m(D, D.t2, &D.t_init, D.mut, XkField<R>{D.xkhh}, i, j, k);
          else tt += hdiff_m(D, D.t2, &D.t_init, D.mut, XkConst<R>{khh}, i, j, k);
        }
        tt += vdiff_m(D, D.t2, &D.t_init, D.mut, R(3.) * kvdif, i, j, k);
      }
      if (d6on && d6_in('m', nx, ny, sp, px, ox, oy, i, j)) {
        R tx, ty;
        d6_tend(D, 'm', D.t2, D.mut, D.c1h, D.c2h, c6, i, j, k, tx, ty);
        tt = tt + tx + ty;
      }
      if (D.damp_opt == 2 && ray_t(D, i, j, k, rt)) tt = tt - rt;
      if (sp && relax_at<R, false>(D, D.t2, D.c1h, D.c2h, D.lbc_var[2], ring_for(nx, ny, 't'), i, j, k, fa, fb)) tt += fa - fb;
      D.t_tendf(i, j, k) = tt;
    }
    if (k == 0 && sp) {
      R tm = 0;
      if (relax_at<R, true>(D, D.mu2, nullptr, nullptr, D.lbc_var[4], ring_for(nx, ny, 'm'), i, j, 0, fa, fb)) tm += fa - fb;
      D.mu_tend(i, j, 0) = tm;
    }
  }
}

// The remaining ring kernels (spec zone b = 0, thread (pos, level, side)): the end-of-step spec_bdy_final,
// flow_dep_bdy of the scalars without boundary data, zero_grad_bdy of w. The other boundary operations run
// inside the kernels that compute the same points (k_tendf_rk1, k_tend, k_uv, k_ac, k_q_tendf_rk1).
enum RingOp { RO_FINAL = 0, RO_FLOW_DEP, RO_ZERO_GRAD_W };
// the member computes point (i, j) of a field of staggering s ('u': x faces, 'v': y faces, else mass points): its
// patch's points (the whole domain's without a decomposition)
template <class R>
__device__ __forceinline__ bool owns(const Dom<R>& D, int i, int j, char s) {
  const int iu = (s == 'u' && D.pi1 == D.nx) ? D.nx + 1 : D.pi1;
  const int jv = (s == 'v' && D.pj1 == D.ny) ? D.nyv : D.pj1;
  return i >= D.pi0 && i < iu && j >= D.pj0 && j < jv;
}
template <class R, int NM>
__global__ void __launch_bounds__(PX) k_ring(const __grid_constant__ Pack<R, NM> P, int op, int rk) {
  const Dom<R>* Dp;
  int pos, k, side;
  if (!thread_index<0>(P, RG_RING, Dp, pos, k, side)) return;
  const Dom<R>& D = *Dp;
  if (!D.lbc) return;  // a member without boundary data in a pack with some: LateralBC belongs to the others only
  (void)rk;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  switch (op) {
    case RO_ZERO_GRAD_W: {  // zero_grad_bdy on w (KZeroGrad, lateral_bc.cpp:143-159)
      int i, j;
      const Ring r = ring_for(nx, ny, 'h');
      if (!r.map(pos, side, 0, i, j) || !owns(D, i, j, 'h')) return;
      const int ic = i < 1 ? 1 : (i > r.ibe - 1 ? r.ibe - 1 : i);
      const int jc = j < 1 ? 1 : (j > r.jbe - 1 ? r.jbe - 1 : j);
      switch (side) {
        case 0: D.w2(i, j, k) = D.w2(ic, 1, k); break;
        case 1: D.w2(i, j, k) = D.w2(ic, r.jbe - 1, k); break;
        case 2: D.w2(i, j, k) = D.w2(1, jc, k); break;
        default: D.w2(i, j, k) = D.w2(r.ibe - 1, jc, k); break;
      }
      return;
    }
    case RO_FINAL: {  // final (:425-455)
      int i, j;
      const int sl = slab_of_side(side);
      const R dtbc = R(*D.dtbc);
      if (k < nz && ring_for(nx, ny, 'u').map(pos, side, 0, i, j) && owns(D, i, j, 'u')) {
        const R bval = slab_val(D.lbc_var[0], sl, pos, k, 0, dtbc);
        D.u2(i, j, k) = D.msfuy(i, j) * bval / (R(D.c1h[k]) * D.muus(i, j, 0) + R(D.c2h[k]));
      }
      if (k < nz && ring_for(nx, ny, 'v').map(pos, side, 0, i, j) && owns(D, i, j, 'v')) {
        const R bval = slab_val(D.lbc_var[1], sl, pos, k, 0, dtbc);
        D.v2(i, j, k) = D.msfvx(i, j) * bval / (R(D.c1h[k]) * D.muvs(i, j, 0) + R(D.c2h[k]));
      }
      if (k < nz && ring_for(nx, ny, 't').map(pos, side, 0, i, j) && owns(D, i, j, 't')) {
        const R bval = slab_val(D.lbc_var[2], sl, pos, k, 0, dtbc);
        D.t2(i, j, k) = R(1) * bval / (R(D.c1h[k]) * D.muts(i, j, 0) + R(D.c2h[k]));
        for (int n = 0; n < D.n_scalars; ++n)
          if (D.lbc_q[n].have) {
            const R qb = slab_val(D.lbc_q[n], sl, pos, k, 0, dtbc);
            D.q2[n](i, j, k) = R(1) * qb / (R(D.c1h[k]) * D.muts(i, j, 0) + R(D.c2h[k]));
          }
      }
      if (ring_for(nx, ny, 'h').map(pos, side, 0, i, j) && owns(D, i, j, 'h')) {
        const R bval = slab_val(D.lbc_var[3], sl, pos, k, 0, dtbc);
        D.ph2(i, j, k) = R(1) * bval / (R(D.c1f[k]) * D.muts(i, j, 0) + R(D.c2f[k]));
      }
      if (k == 0 && ring_for(nx, ny, 'm').map(pos, side, 0, i, j) && owns(D, i, j, 'm')) {
        const R bval = slab_val(D.lbc_var[4], sl, pos, 0, 0, dtbc);
        D.mu2(i, j, 0) = R(1) * bval / R(1);
      }
      return;
    }
    case RO_FLOW_DEP: {  // flow_dep (:416-423) on the scalars without boundary data
      if (k >= nz) return;
      int i, j;
      const Ring r = ring_for(nx, ny, 'q');
      if (!r.map(pos, side, 0, i, j) || !owns(D, i, j, 'q')) return;
      const int ic = i < 1 ? 1 : (i > r.ibe - 1 ? r.ibe - 1 : i);
      const int jc = j < 1 ? 1 : (j > r.jbe - 1 ? r.jbe - 1 : j);
      for (int n = 0; n < D.n_scalars; ++n) {
        if (D.lbc_q[n].have) continue;
        const V3<R>& f = D.q2[n];
        switch (side) {
          case 0: f(i, j, k) = D.rv_m(i, j, k) < R(0) ? f(ic, 1, k) : R(0); break;
          case 1: f(i, j, k) = D.rv_m(i, j + 1, k) > R(0) ? f(ic, r.jbe - 1, k) : R(0); break;
          case 2: f(i, j, k) = D.ru_m(i, j, k) < R(0) ? f(1, jc, k) : R(0); break;
          default: f(i, j, k) = D.ru_m(i + 1, j, k) > R(0) ? f(r.ibe - 1, jc, k) : R(0); break;
        }
      }
      return;
    }
  }
}

// LateralBC::advance_time (lateral_bc.hpp:58): dtbc += dt at the start of every step
// LargeStep::cfl_max (src/dyn/large_step.cpp:672-687, :865-877) after stage rk's tendencies: the largest vertical
// Courant number |ww / (c1f mut + c2f) rdnw dt| and horizontal one max(|u rdx msfux dt|, |v rdy msfvy dt|) over the
// mass points of levels 1 .. nz-1. Maxima do not depend on the order: each block folds its values and raises the
// member's maxima by an atomic max on the bits of the positive doubles (NaN and zero never enter, as in WRF's
// running maxima, which start at 0).
template <class R, int NM, int SH>
__global__ void __launch_bounds__(PX) k_cfl(const __grid_constant__ Pack<R, NM> P, int rk) {
  const Dom<R>* Dp;
  int i, j, k;
  const bool in = thread_index<SH>(P, RG_MASS, Dp, i, j, k);
  const Dom<R>& D = *Dp;
  double vert = 0, horiz = 0;
  if (in && k >= 1) {
    const R dt = R(D.dt);
    const R x = D.ww.ld(i, j, k) / (R(D.c1f[k]) * D.mut.ld(i, j, 0) + R(D.c2f[k])) * R(D.rdnw[k]) * dt;
    vert = double(x < R(0) ? -x : x);
    R a = D.u2.ld(i, j, k) * R(D.rdx) * D.msfux(i, j) * dt, b = D.v2.ld(i, j, k) * R(D.rdy) * D.msfvy(i, j) * dt;
    a = a < R(0) ? -a : a;
    b = b < R(0) ? -b : b;
    horiz = double(b > a ? b : a);
  }
  if (!(vert > 0)) vert = 0;
  if (!(horiz > 0)) horiz = 0;
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, vert, o), h2 = __shfl_xor_sync(0xffffffffu, horiz, o);
    vert = v2 > vert ? v2 : vert;
    horiz = h2 > horiz ? h2 : horiz;
  }
  if ((threadIdx.x & 31) == 0) {  // every block lies in one member (pack block ranges)
    if (vert > 0) atomicMax(D.cfl + 2 * (rk - 1), (unsigned long long)__double_as_longlong(vert));
    if (horiz > 0) atomicMax(D.cfl + 2 * (rk - 1) + 1, (unsigned long long)__double_as_longlong(horiz));
  }
}

template <class R, int NM>
__global__ void k_advance_time(const __grid_constant__ Pack<R, NM> P) {
  const int m = blockIdx.x;
  if (m < P.n && threadIdx.x == 0 && P.d[m].lbc) *P.d[m].dtbc += P.d[m].dt;
}

}  // namespace cw
