// SPDX-License-Identifier: GPL-3.0-or-later
// The mixed form's step (FP32 fields; FP64 in the column mass sum, the w tridiagonal solve and calc_p_rho):
// the same kernels as the FP64 form, instantiated with R = float in this translation unit, which is compiled
// with FMA contraction and single-precision denormals flushed to zero (division and square root stay IEEE).
// The form is held to a tolerance against the FP64 form, not to bit identity.
#include "cw_step.cuh"

namespace cw {

long long enqueue_mixed(cw_handle* h, bool plan) {
  Launcher L{h};
  L.plan = plan;
  enqueue_t<float>(h, L, h->t32);
  return L.count;
}

}  // namespace cw
