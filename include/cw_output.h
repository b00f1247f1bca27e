/* SPDX-License-Identifier: GPL-3.0-or-later
 *
 * cw_output.h -- CPPWRF's run outputs for the state of the B200 dynamical core, in the reference's own
 * formats, so that a run on the device is read by the reference's tools and compared with its goldens:
 *   - the diag.csv row: dyn::Diagnostics::compute (src/dyn/diagnostics.hpp:13-38, diagnostics.cpp:56-80),
 *     reduced on the device in the reference CPU build's summation order, written by io::DiagWriter's
 *     formatting (src/io/output.hpp:79-91, output.cpp:344-389);
 *   - the snapshot pair snap_NNNNNN.{json,bin}: io::SnapshotWriter (src/io/output.hpp:68-74,
 *     output.cpp:222-340) of the variables of dyn::snapshot_vars (src/dyn/diagnostics.cpp:82-153).
 */
#ifndef CW_OUTPUT_H
#define CW_OUTPUT_H

#include <stddef.h>

#include "cw_dycore.h"

#ifdef __cplusplus
extern "C" {
#endif

/* dyn::DiagRow (src/dyn/diagnostics.hpp:13-17): dry_mass [kg], theta_mass [kg K], total_energy [J]; a NaN or
 * Inf in a field makes its maximum +Inf. max_abs_q: over every scalar (not a diag.csv column). */
typedef struct cw_diag {
  double max_abs_u, max_abs_v, max_abs_w, min_th_pert, max_th_pert, dry_mass, theta_mass, total_energy;
  double max_abs_q;
} cw_diag;

/* Diagnostics::compute of a member's current state (the handle's step work is waited for). With moist
 * species, species 0 is qv and t_2 holds theta_m - t0 (use_theta_m = 1). FP64 handles give the reference
 * CPU build's values to the bit, except that total_energy's pow is cw_pow (the CPU build: glibc's pow). */
int cw_diagnostics(cw_handle* h, int member, cw_diag* out);

/* The diag.csv header line and one row ("step,time,max_abs_u,...,total_energy,wall_s"), as io::DiagWriter
 * writes them, without the newline. Return the text's length, or -1 when n is too small. */
int cw_diag_header(char* buf, size_t n);
int cw_diag_format_row(long long step, double time, const cw_diag* d, double wall_s, char* buf, size_t n);

/* Whole-allocation host arrays (the fields' layouts, cw_layout_of) of the state a snapshot is made of. q_2:
 * n_scalars arrays (may be NULL without scalars); rainnc, rainncv: with mp_physics != 0. */
typedef struct cw_snapshot_fields {
  const double *u_2, *v_2, *w_2, *t_2, *p, *ph_2, *mu_2;
  const double *pb, *phb, *t_init, *mub;
  const double* const* q_2;
  const double *rainnc, *rainncv;
} cw_snapshot_fields;

/* Writes dir/snap_<step, 6 digits>.bin and .json (each through a temporary file and a rename): u v w th_pert
 * theta [theta_m] p p_pert ph mu mu_pert z_m, the scalars, and with microphysics rainnc, rainncv (the physics'
 * extra 2-D fields), float64, (k, j, i) order. q_names: n_scalars names (NULL: species 0 "qv" when there are moist species,
 * with Kessler 1 and 2 "qc" and "qr", the others "q<n>"). */
int cw_snapshot_write_host(const char* dir, long long step, double time, const cw_grid* g, const cw_options* o,
                           const cw_snapshot_fields* f, const char* const* q_names);
/* The same of a member of a handle (its fields downloaded first). */
int cw_snapshot_write(cw_handle* h, int member, const char* dir, long long step, double time,
                      const char* const* q_names);
/* The reason of the last failed cw_snapshot_write* / cw_diag_* call of the calling thread. */
const char* cw_output_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CW_OUTPUT_H */
