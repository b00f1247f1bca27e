/* SPDX-License-Identifier: GPL-3.0-or-later
 * TEST INFRASTRUCTURE ONLY: linked into _ref/ref_harness_own ahead of libm / libmvec, it binds the two
 * pow entry points the reference's CPU build calls in calc_p_rho_phi (scalar libm pow and libmvec's
 * 2-lane _ZGVbN2vv_pow, src/core/backend.hpp:118, :169-175) to cw_pow, the pow of the GPU path, and the
 * scalar and libmvec 2-lane sin of the Rayleigh dampings (damp_opt 3, src/dyn/small_step.cpp:400; damp_opt 2,
 * src/dyn/diffusion/rayleigh_damp.hpp:16-25, :136) to cw_sin, and the scalar and libmvec 2-lane log of
 * calc_p_rho_phi's hypsometric_opt 2 (src/dyn/small_step.cpp:467, src/core/backend.hpp:176-184) to cw_log, and the
 * scalar and libmvec 2-lane cos of cal_dampkm (damp_opt 1, src/dyn/diffusion/km_kh.hpp:24-33) to cw_cos. The
 * reference's every other operation is unchanged, so bit-identity with this build is a fair test of them. */
#include <emmintrin.h>

#include "../cppwrf_b200/csrc/cw_pow.h"

double pow(double x, double y) { return cw_pow(x, y); }

__m128d _ZGVbN2vv_pow(__m128d x, __m128d y) {
  double a[2], b[2];
  _mm_storeu_pd(a, x);
  _mm_storeu_pd(b, y);
  return _mm_set_pd(cw_pow(a[1], b[1]), cw_pow(a[0], b[0]));
}

double sin(double x) { return cw_sin(x); }

__m128d _ZGVbN2v_sin(__m128d x) {
  double a[2];
  _mm_storeu_pd(a, x);
  return _mm_set_pd(cw_sin(a[1]), cw_sin(a[0]));
}

double log(double x) { return cw_log(x); }

__m128d _ZGVbN2v_log(__m128d x) {
  double a[2];
  _mm_storeu_pd(a, x);
  return _mm_set_pd(cw_log(a[1]), cw_log(a[0]));
}

double cos(double x) { return cw_cos(x); }

__m128d _ZGVbN2v_cos(__m128d x) {
  double a[2];
  _mm_storeu_pd(a, x);
  return _mm_set_pd(cw_cos(a[1]), cw_cos(a[0]));
}
