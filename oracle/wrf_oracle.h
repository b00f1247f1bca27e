/* SPDX-License-Identifier: GPL-3.0-or-later
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is a plain-C, single-threaded restatement of CPPWRF's
 * RK3 split-explicit dry dynamical core step (src/dyn/rk3.cpp:86-170 and the kernels it calls).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only as
 * the checker or the timed CPU reference; the product library never links or calls it.
 *
 * Parity pins (tests/test_oracle_golden.py): bit-for-bit equality with the reference's own
 * regression goldens (tools/regression/golden/{straka,warm_bubble,igw,rest_state}_cpu_fp64,
 * copied into tests/golden/ by tests/golden/make_golden.py) in OR_POW_GLIBC mode, and with the
 * reference's CPU FP64 build compiled from its sources (oracle/_ref, oracle/Makefile) on
 * terrain / moist / specified-boundary cases in OR_POW_OWN mode (pow interposed in both).
 */
#ifndef WRF_ORACLE_H
#define WRF_ORACLE_H

#include "../include/cw_dycore.h"

#ifdef __cplusplus
extern "C" {
#endif

/* calc_p_rho_phi's pow: OR_POW_GLIBC = glibc's libmvec 2-lane pow / scalar libm pow by the lane
 * rule of the reference CPU build (src/core/backend.hpp:144, :169-175); OR_POW_OWN = cw_pow. */
enum { OR_POW_OWN = 0, OR_POW_GLIBC = 1 };

typedef struct or_dom or_dom;

or_dom* or_create(const cw_grid* g, const cw_options* o);
void or_destroy(or_dom* d);
int or_layout(or_dom* d, int field, int n, cw_layout* out);
/* the allocation of a field (halo included), layout.total doubles */
double* or_field(or_dom* d, int field, int n);
int or_set_vertical(or_dom* d, const cw_vertical* v);
int or_set_lbc(or_dom* d, int var, int side, const double* values, const double* tends, size_t count);
int or_set_lbc_scalar(or_dom* d, int n, int side, const double* values, const double* tends, size_t count);
int or_set_lbc_time(or_dom* d, double dtbc);
void or_set_pow_mode(or_dom* d, int mode);
int or_n_sound(or_dom* d);
int or_step(or_dom* d, int nsteps);
/* dyn::Diagnostics::compute: max|u| max|v| max|w| min th' max th' dry_mass theta_mass total_energy max|q| */
int or_diagnostics(or_dom* d, double out[9]);
/* LargeStep::cfl_max after each RK stage's tendencies in the last step: (vertical, horizontal) for stages 1..3 */
int or_cfl_max(or_dom* d, double out[6]);
const char* or_last_error(or_dom* d);

#ifdef __cplusplus
}
#endif
#endif
