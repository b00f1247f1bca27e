/* SPDX-License-Identifier: GPL-3.0-or-later
 *
 * cw_pow: the dycore's own double-precision pow(x, y), written from the mathematics:
 *   x = 2^e * m, m in [sqrt(1/2), sqrt(2)),   log m = 2 atanh(s), s = (m - 1) / (m + 1)
 *   y log x in double-double,                  exp(t) = 2^k * (1 + expm1(r / 256))^256 by the
 *                                              doubling identity expm1(2a) = expm1(a) * (2 + expm1(a))
 * with error-free transformations (Knuth's two_sum; the exact product error from one fused
 * multiply-add) and truncated Taylor series. Only IEEE-754 double add, subtract, multiply,
 * divide, fused multiply-add, floor and power-of-two scaling are used, each spelled as an
 * explicit rounding operation, so the same source gives bit-identical results on the host (C or
 * C++ fma(), compiled with -ffp-contract=off) and on the device (__dadd_rn / __dmul_rn /
 * __ddiv_rn / __fma_rn, which nvcc never contracts or reassociates, whatever --fmad says).
 *
 * Why the dycore needs its own: calc_p_rho_phi evaluates p = p1000 * pow(R theta / (p1000 a), cp/cv)
 * (reference src/dyn/small_step.cpp:474-475). The reference's CPU FP64 build takes that pow from
 * glibc (libmvec's 2-lane _ZGVbN2vv_pow or scalar libm pow, by the lane rule of
 * src/core/backend.hpp:144-175); glibc's algorithms are not available here, so the GPU path and
 * the oracle's interposed mode both call cw_pow instead. The accuracy is checked against
 * glibc pow and against a 60-digit decimal evaluation in tests/test_pow.py.
 *
 * cw_exp(x) is the same exponential on a double argument, cw_log(x) the same logarithm rounded to double;
 * cw_sin(x) and cw_cos(x) double-double Taylor series for |x| <= 2.
 *
 * Domain: any double x, y; special values follow C99 Annex F for the cases the dycore can meet
 * (x > 0 finite; NaN, 0, infinities and negative x are handled for robustness).
 */
#ifndef CW_POW_H
#define CW_POW_H

#if defined(__CUDACC__)
#define CW_HD __host__ __device__ __forceinline__
#else
#define CW_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define CW_ADD(a, b) __dadd_rn((a), (b))
#define CW_SUB(a, b) __dsub_rn((a), (b))
#define CW_MUL(a, b) __dmul_rn((a), (b))
#define CW_DIV(a, b) __ddiv_rn((a), (b))
#define CW_FLOOR(a) floor(a)
#define CW_FMA(a, b, c) __fma_rn((a), (b), (c))
#define CW_BITS(d) ((unsigned long long)__double_as_longlong(d))
#define CW_FROMBITS(u) __longlong_as_double((long long)(u))
#else
#include <math.h>
#include <string.h>
#define CW_ADD(a, b) ((a) + (b))
#define CW_SUB(a, b) ((a) - (b))
#define CW_MUL(a, b) ((a) * (b))
#define CW_DIV(a, b) ((a) / (b))
#define CW_FLOOR(a) floor(a)
#define CW_FMA(a, b, c) fma((a), (b), (c))
CW_HD unsigned long long cw_bits_host(double d) {
  unsigned long long u;
  memcpy(&u, &d, sizeof u);
  return u;
}
CW_HD double cw_frombits_host(unsigned long long u) {
  double d;
  memcpy(&d, &u, sizeof d);
  return d;
}
#define CW_BITS(d) cw_bits_host(d)
#define CW_FROMBITS(u) cw_frombits_host(u)
#endif

/* ---- error-free transformations ---- */
/* s + e = a + b exactly (Knuth) */
CW_HD void cw_two_sum(double a, double b, double* s, double* e) {
  const double t = CW_ADD(a, b);
  const double bb = CW_SUB(t, a);
  *s = t;
  *e = CW_ADD(CW_SUB(a, CW_SUB(t, bb)), CW_SUB(b, bb));
}
/* s + e = a + b exactly when |a| >= |b| (Dekker) */
CW_HD void cw_fast_two_sum(double a, double b, double* s, double* e) {
  const double t = CW_ADD(a, b);
  *s = t;
  *e = CW_SUB(b, CW_SUB(t, a));
}
/* p + e = a * b exactly: the rounding error of a double product is itself a double, and one fused multiply-add
 * (a single rounding of a*b - p, exact here) yields it; Dekker's split product gives the same e without an fma */
CW_HD void cw_two_prod(double a, double b, double* p, double* e) {
  const double q = CW_MUL(a, b);
  *p = q;
  *e = CW_FMA(a, b, -q);
}

/* ---- double-double arithmetic (hi, lo), |lo| <= ulp(hi)/2 ---- */
CW_HD void cw_dd_add(double ah, double al, double bh, double bl, double* rh, double* rl) {
  double s, e;
  cw_two_sum(ah, bh, &s, &e);
  e = CW_ADD(e, CW_ADD(al, bl));
  cw_fast_two_sum(s, e, rh, rl);
}
CW_HD void cw_dd_mul(double ah, double al, double bh, double bl, double* rh, double* rl) {
  double p, e;
  cw_two_prod(ah, bh, &p, &e);
  e = CW_ADD(e, CW_ADD(CW_MUL(ah, bl), CW_MUL(al, bh)));
  cw_fast_two_sum(p, e, rh, rl);
}
/* (ah, al) / (bh, bl): one Newton correction of the double quotient */
CW_HD void cw_dd_div(double ah, double al, double bh, double bl, double* rh, double* rl) {
  const double q1 = CW_DIV(ah, bh);
  double ph, pl, dh, dl;
  cw_dd_mul(q1, 0.0, bh, bl, &ph, &pl);
  cw_dd_add(ah, al, -ph, -pl, &dh, &dl);
  const double q2 = CW_DIV(dh, bh);
  cw_fast_two_sum(q1, q2, rh, rl);
}

/* 2^k for -1022 <= k <= 1023 */
CW_HD double cw_pow2i(int k) { return CW_FROMBITS((unsigned long long)(k + 1023) << 52); }

/* log(x) in double-double for finite x > 0 */
CW_HD void cw_log_dd(double x, double* rh, double* rl) {
  int e = 0;
  if (x < 0x1p-1022) { /* subnormal: scale into the normal range first (exact) */
    x = CW_MUL(x, 0x1p54);
    e = -54;
  }
  const unsigned long long b = CW_BITS(x);
  e += (int)((b >> 52) & 0x7ff) - 1023;
  double m = CW_FROMBITS((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1, 2) */
  if (m > 0x1.6a09e667f3bcdp+0) { /* > sqrt(2): halve (exact) */
    m = CW_MUL(m, 0.5);
    e += 1;
  }
  /* s = (m - 1) / (m + 1); m - 1 is exact (Sterbenz), m + 1 as a double-double */
  double dh, dl, sh, sl;
  cw_two_sum(m, 1.0, &dh, &dl);
  cw_dd_div(CW_SUB(m, 1.0), 0.0, dh, dl, &sh, &sl);
  double zh, zl;
  cw_dd_mul(sh, sl, sh, sl, &zh, &zl); /* s^2 <= 0.0295 */
  /* atanh(s)/s = sum_n s^(2n)/(2n+1): terms n >= 3 in double (they are < 3.6e-6 of the sum), the
   * first three in double-double; the last kept term, s^28/29, is below 2^-70 */
  const double z = zh;
  double q = 0x1.1a7b9611a7b96p-5; /* 1/29 */
  q = CW_ADD(0x1.2f684bda12f68p-5, CW_MUL(z, q)); /* 1/27 */
  q = CW_ADD(0x1.47ae147ae147bp-5, CW_MUL(z, q)); /* 1/25 */
  q = CW_ADD(0x1.642c8590b2164p-5, CW_MUL(z, q)); /* 1/23 */
  q = CW_ADD(0x1.8618618618618p-5, CW_MUL(z, q)); /* 1/21 */
  q = CW_ADD(0x1.af286bca1af28p-5, CW_MUL(z, q)); /* 1/19 */
  q = CW_ADD(0x1.e1e1e1e1e1e1ep-5, CW_MUL(z, q)); /* 1/17 */
  q = CW_ADD(0x1.1111111111111p-4, CW_MUL(z, q)); /* 1/15 */
  q = CW_ADD(0x1.3b13b13b13b14p-4, CW_MUL(z, q)); /* 1/13 */
  q = CW_ADD(0x1.745d1745d1746p-4, CW_MUL(z, q)); /* 1/11 */
  q = CW_ADD(0x1.c71c71c71c71cp-4, CW_MUL(z, q)); /* 1/9 */
  q = CW_ADD(0x1.2492492492492p-3, CW_MUL(z, q)); /* 1/7 */
  double ah, al;
  /* A = 1/5 + z q */
  cw_dd_add(0x1.999999999999ap-3, -0x1.999999999999ap-57, CW_MUL(z, q), 0.0, &ah, &al);
  /* A = 1/3 + z A */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(0x1.5555555555555p-2, 0x1.5555555555555p-56, ah, al, &ah, &al);
  /* A = 1 + z A */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(1.0, 0.0, ah, al, &ah, &al);
  /* log m = 2 s A */
  double lh, ll;
  cw_dd_mul(sh, sl, ah, al, &lh, &ll);
  lh = CW_MUL(lh, 2.0);
  ll = CW_MUL(ll, 2.0);
  /* + e log 2 */
  double eh, el;
  const double ed = (double)e;
  cw_two_prod(ed, 0x1.62e42fefa39efp-1, &eh, &el);
  el = CW_ADD(el, CW_MUL(ed, 0x1.abc9e3b39803fp-56));
  cw_dd_add(eh, el, lh, ll, rh, rl);
}

/* exp(th + tl) rounded to double */
CW_HD double cw_exp_dd(double th, double tl) {
  if (th > 709.8) return CW_MUL(0x1p1023, 2.0); /* overflow: +inf */
  if (th < -745.2) return 0.0;
  const double kd = CW_FLOOR(CW_ADD(CW_MUL(th, 0x1.71547652b82fep+0), 0.5));
  const int k = (int)kd;
  /* r = t - k log 2 (k log2_hi exact as a double-double) */
  double ph, pl, rh, rl;
  cw_two_prod(kd, 0x1.62e42fefa39efp-1, &ph, &pl);
  pl = CW_ADD(pl, CW_MUL(kd, 0x1.abc9e3b39803fp-56));
  cw_dd_add(th, tl, -ph, -pl, &rh, &rl);
  /* a = r / 256 (exact) */
  const double ah = CW_MUL(rh, 0x1p-8), al = CW_MUL(rl, 0x1p-8);
  /* expm1(a) = a + a^2 (1/2 + a/6 + a^2/24 + ... + a^6/40320); |a| < 0.00136 */
  double q = 0x1.a01a01a01a01ap-16;                /* 1/8! */
  q = CW_ADD(0x1.a01a01a01a01ap-13, CW_MUL(ah, q)); /* 1/7! */
  q = CW_ADD(0x1.6c16c16c16c17p-10, CW_MUL(ah, q)); /* 1/6! */
  q = CW_ADD(0x1.1111111111111p-7, CW_MUL(ah, q));  /* 1/5! */
  q = CW_ADD(0x1.5555555555555p-5, CW_MUL(ah, q));  /* 1/4! */
  q = CW_ADD(0x1.5555555555555p-3, CW_MUL(ah, q));  /* 1/3! */
  q = CW_MUL(ah, q);
  double ch, cl, a2h, a2l, mh, ml;
  cw_two_sum(0.5, q, &ch, &cl);
  cw_dd_mul(ah, al, ah, al, &a2h, &a2l);
  cw_dd_mul(a2h, a2l, ch, cl, &ch, &cl);
  cw_dd_add(ah, al, ch, cl, &mh, &ml);
  /* eight doublings: expm1(2a) = expm1(a) (2 + expm1(a)) */
  for (int n = 0; n < 8; ++n) {
    double th2, tl2;
    cw_dd_add(2.0, 0.0, mh, ml, &th2, &tl2);
    cw_dd_mul(mh, ml, th2, tl2, &mh, &ml);
  }
  double eh, el;
  cw_dd_add(1.0, 0.0, mh, ml, &eh, &el);
  const double r = CW_ADD(eh, el); /* the double nearest to exp(r) (up to the series' error) */
  /* scale by 2^k: in two exact steps where 2^k alone would not be a normal double */
  if (k > 1023) return CW_MUL(CW_MUL(r, cw_pow2i(1023)), cw_pow2i(k - 1023));
  if (k < -1022) return CW_MUL(CW_MUL(r, cw_pow2i(-1022)), cw_pow2i(k + 1022));
  return CW_MUL(r, cw_pow2i(k));
}

/* pow(x, y) */
CW_HD double cw_pow(double x, double y) {
  if (x != x || y != y) return CW_ADD(x, y);
  if (y == 0.0) return 1.0;
  if (x == 1.0) return 1.0;
  double sign = 1.0;
  if (x < 0.0) {
    const double fy = CW_FLOOR(y);
    if (fy != y) return CW_DIV(0.0, 0.0); /* NaN: negative base, non-integer exponent */
    /* integer y: odd when y/2 is not an integer (|y| < 2^53 here) */
    if (CW_FLOOR(CW_MUL(y, 0.5)) != CW_MUL(y, 0.5)) sign = -1.0;
    x = -x;
  }
  const double inf = CW_MUL(0x1p1023, 2.0);
  if (x == 0.0) return y > 0.0 ? CW_MUL(sign, 0.0) : CW_MUL(sign, inf);
  if (x == inf) return y > 0.0 ? CW_MUL(sign, inf) : CW_MUL(sign, 0.0);
  if (y == inf) return x > 1.0 ? inf : 0.0;
  if (y == -inf) return x > 1.0 ? 0.0 : inf;
  double lh, ll, th, tl, e;
  cw_log_dd(x, &lh, &ll);
  cw_two_prod(y, lh, &th, &e);
  e = CW_ADD(e, CW_MUL(y, ll));
  cw_fast_two_sum(th, e, &th, &tl);
  return CW_MUL(sign, cw_exp_dd(th, tl));
}

/* exp(x): the exponential core of cw_pow on a double argument (the Kessler microphysics' saturation vapour
 * pressure; the reference's CPU build takes glibc's exp there) */
CW_HD double cw_exp(double x) {
  if (x != x) return CW_ADD(x, x);
  return cw_exp_dd(x, 0.0);
}

/* log(x): the double-double logarithm of cw_pow rounded to double (calc_p_rho_phi's hypsometric_opt 2,
 * al = dphi / (p_mid log(p_bottom / p_top)); the reference's CPU build takes glibc's log there, libmvec's on the
 * lanes of its vectorised loop) */
CW_HD double cw_log(double x) {
  if (x != x) return CW_ADD(x, x);
  if (x < 0.0) return CW_DIV(0.0, 0.0);
  const double inf = CW_MUL(0x1p1023, 2.0);
  if (x == 0.0) return -inf;
  if (x == inf) return inf;
  if (x == 1.0) return 0.0;
  double h, l;
  cw_log_dd(x, &h, &l);
  return CW_ADD(h, l);
}

/* sin(x) for |x| <= 2 (NaN outside): the Taylor series sin x = x sum_n (-1)^n x^(2n) / (2n+1)!, its terms n >= 4
 * (below 2.5e-3 of the sum) in double and the first four in double-double, the last kept term 4^14 / 29! < 2^-75
 * (advance_w's Rayleigh damping of w, damp_opt 3: sin of arguments in [0, pi/2]; the reference's CPU build takes
 * glibc's sin there) */
CW_HD void cw_sin_dd(double x, double* sh, double* sl) { /* sin(x) in double-double, |x| <= 2, x != 0 */
  double zh, zl;
  cw_two_prod(x, x, &zh, &zl);
  const double z = zh;
  double t = 0x1.259f98b4358adp-103;               /* 1/29! */
  t = CW_ADD(-0x1.d1ab1c2dccea3p-94, CW_MUL(z, t)); /* 1/27! */
  t = CW_ADD(0x1.3f3ccdd165fa9p-84, CW_MUL(z, t));  /* 1/25! */
  t = CW_ADD(-0x1.761b41316381ap-75, CW_MUL(z, t)); /* 1/23! */
  t = CW_ADD(0x1.71b8ef6dcf572p-66, CW_MUL(z, t));  /* 1/21! */
  t = CW_ADD(-0x1.2f49b46814157p-57, CW_MUL(z, t)); /* 1/19! */
  t = CW_ADD(0x1.952c77030ad4ap-49, CW_MUL(z, t));  /* 1/17! */
  t = CW_ADD(-0x1.ae7f3e733b81fp-41, CW_MUL(z, t)); /* 1/15! */
  t = CW_ADD(0x1.6124613a86d09p-33, CW_MUL(z, t));  /* 1/13! */
  t = CW_ADD(-0x1.ae64567f544e4p-26, CW_MUL(z, t)); /* 1/11! */
  t = CW_ADD(0x1.71de3a556c734p-19, CW_MUL(z, t));  /* 1/9! */
  double ah, al;
  cw_dd_add(-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73, CW_MUL(z, t), 0.0, &ah, &al); /* -1/7! + z t */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(0x1.1111111111111p-7, 0x1.1111111111111p-63, ah, al, &ah, &al); /* 1/5! + z A */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(-0x1.5555555555555p-3, -0x1.5555555555555p-57, ah, al, &ah, &al); /* -1/3! + z A */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(1.0, 0.0, ah, al, &ah, &al); /* 1 + z A */
  cw_dd_mul(x, 0.0, ah, al, sh, sl);
}
CW_HD double cw_sin(double x) {
  if (x != x) return CW_ADD(x, x);
  if (x == 0.0) return x;
  if (!(x <= 2.0 && x >= -2.0)) return CW_DIV(0.0, 0.0);
  double sh, sl;
  cw_sin_dd(x, &sh, &sl);
  return CW_ADD(sh, sl);
}

/* cos(x) for |x| <= 2 (NaN outside): for |x| <= pi/4 the Taylor series cos x = sum_n (-1)^n x^(2n) / (2n)!, its terms
 * n >= 4 (below 4.1e-4 of the sum) in double and the first four in double-double, the last kept term
 * (pi/4)^26 / 26! < 2^-95; above pi/4, cos x = sin(pi/2 - x) with pi/2 - x in double-double from the exact
 * difference pio2_hi - x (Sterbenz) and the two lower parts of pi/2, so that the result keeps its relative accuracy
 * near pi/2 (the eddy-viscosity damping of damp_opt 1: cos of arguments in [0, pi/2]; the
 * reference's CPU build takes glibc's cos there, libmvec's on the lanes of its vectorised column loop) */
CW_HD double cw_cos(double x) {
  if (x != x) return CW_ADD(x, x);
  if (x < 0.0) x = -x;
  if (!(x <= 2.0)) return CW_DIV(0.0, 0.0);
  if (x > 0x1.921fb54442d18p-1) {
    /* u = pi/2 - x in double-double from a three-part pi/2; sin(uh + ul) = sin(uh) + ul cos(uh) to the last bit */
    double uh, ul;
    cw_dd_add(CW_SUB(0x1.921fb54442d18p+0, x), 0.0, 0x1.1a62633145c07p-54, -0x1.f1976b7ed8fbcp-110, &uh, &ul);
    double sh = 0.0, sl = 0.0;
    if (uh != 0.0) cw_sin_dd(uh, &sh, &sl);
    const double u2 = CW_MUL(uh, uh);
    const double c = CW_ADD(1.0, CW_MUL(u2, CW_ADD(-0.5, CW_MUL(u2, 0x1.5555555555555p-5)))); /* cos uh to its size here */
    return CW_ADD(sh, CW_ADD(sl, CW_MUL(ul, c)));
  }
  double zh, zl;
  cw_two_prod(x, x, &zh, &zl);
  const double z = zh;
  double t = -0x1.88e85fc6a4e5ap-89;               /* -1/26! */
  t = CW_ADD(0x1.f2cf01972f578p-80, CW_MUL(z, t));  /* 1/24! */
  t = CW_ADD(-0x1.0ce396db7f853p-70, CW_MUL(z, t)); /* -1/22! */
  t = CW_ADD(0x1.e542ba4020225p-62, CW_MUL(z, t));  /* 1/20! */
  t = CW_ADD(-0x1.6827863b97d97p-53, CW_MUL(z, t)); /* -1/18! */
  t = CW_ADD(0x1.ae7f3e733b81fp-45, CW_MUL(z, t));  /* 1/16! */
  t = CW_ADD(-0x1.93974a8c07c9dp-37, CW_MUL(z, t)); /* -1/14! */
  t = CW_ADD(0x1.1eed8eff8d898p-29, CW_MUL(z, t));  /* 1/12! */
  t = CW_ADD(-0x1.27e4fb7789f5cp-22, CW_MUL(z, t)); /* -1/10! */
  t = CW_ADD(0x1.a01a01a01a01ap-16, CW_MUL(z, t));  /* 1/8! */
  double ah, al;
  cw_dd_add(-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65, CW_MUL(z, t), 0.0, &ah, &al); /* -1/6! + z t */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(0x1.5555555555555p-5, 0x1.5555555555555p-59, ah, al, &ah, &al); /* 1/4! + z A */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(-0.5, 0.0, ah, al, &ah, &al); /* -1/2! + z A */
  cw_dd_mul(zh, zl, ah, al, &ah, &al);
  cw_dd_add(1.0, 0.0, ah, al, &ah, &al); /* 1 + z A */
  return CW_ADD(ah, al);
}

/* x / c correctly rounded (the IEEE quotient, bit for bit) for a positive constant c without a division, given
 * r = RN(1/c) (Markstein, "Computation of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
 * Dev. 34, 1990; Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018, section 4.9): q = RN(x r) is
 * within one ulp of x / c, so the remainder x - q c is a double and one fused multiply-add computes it exactly,
 * and RN(q + rem r) is then the correctly rounded quotient. The theorem needs the remainder to stay normal and the
 * operands finite; outside 2^-960 <= |x| <= 2^1020 (zeros, whose sign the correction would not keep; values whose
 * remainder could underflow; infinities, NaN) the IEEE division is taken. The flux statement functions divide by
 * 60 and 12 this way; tests/test_div_const.py compares it with the division bit for bit on the host (and the GPU
 * self-check cw_check_div_const on the device). */
CW_HD double cw_div_const(double x, double c, double r) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-960 && ax <= 0x1p+1020)) return CW_DIV(x, c);
  const double q = CW_MUL(x, r);
  const double rem = CW_FMA(-q, c, x);
  return CW_FMA(rem, r, q);
}

#endif /* CW_POW_H */
