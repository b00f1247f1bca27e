/* SPDX-License-Identifier: GPL-3.0-or-later
 *
 * cw_serve.h -- the served form of the B200 dynamical core: a request loop that admits domain-forecast
 * requests by device-memory footprint, keeps their state resident on the device, and advances every
 * resident request together in batched steps (continuous batching: requests that arrive while others run
 * join the batch at the next step; finished ones leave it and free their memory and slot).
 *
 * No counterpart in the reference: CPPWRF runs one forecast per process (src/main.cpp:98) or its nests one
 * after the other (src/cases/nest_driver.cpp:871). Each request's result is the same as the request run
 * alone through cw_step (the batched kernels compute every member independently, in the same order).
 *
 * Threading: three host threads started by cw_serve_create on the configured device, so that setting up and
 * reading back requests overlaps with stepping: an admitter (FIFO admission by footprint, each admitted request
 * set up in a single-domain handle of its own), a stepper (ready requests join their batch without a copy,
 * cw_batch_adopt; every batch's step is launched before any is waited for, and each batch tunes its kernels' block
 * shapes over its first six steps, cw_set_autotune; finished requests leave without a copy, cw_batch_release) and a
 * reader (the finished request's state downloaded on its own stream, its device
 * memory freed). A request holds its footprint of the budget from admission until its state is read back.
 * Every call below may be made from any thread.
 *
 * Failures: a request whose set-up, step or read-back fails is marked failed (cw_serve_wait returns -2) and its
 * memory is returned to the budget; a batch whose step fails is dropped with its requests, and the next request
 * of that acoustic step count makes a new one.
 */
#ifndef CW_SERVE_H
#define CW_SERVE_H

#include <stddef.h>

#include "cw_dycore.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cw_server cw_server;

typedef struct cw_serve_config {
  double hbm_budget_bytes; /* device memory the resident requests may take (cw_footprint sum); default 150e9 */
  int max_resident;        /* at most this many requests on the device at once (<= 256); default 256 */
  int precision;           /* enum cw_precision of every request (a case's own setting is overridden) */
  int device;              /* CUDA device of the loop */
  int keep_results;        /* 1: keep each finished request's prognostic fields for cw_serve_result */
  int test_fail_creates;   /* test hook, 0 in use: the first n batch-handle creations fail with an injected
                              error (the failure path is exercised without a device fault) */
} cw_serve_config;

typedef struct cw_serve_stats {
  long long submitted, completed, failed, rejected, ticks;
  int resident, pending, max_resident_seen;
  double used_bytes, max_used_bytes;
  double p50_s, p99_s, mean_s, max_s; /* request latency: submission to result, seconds (completed requests) */
  double gp_steps;                    /* sum over completed requests of nx*ny*nz*nsteps */
  double wall_s;                      /* first submission to last completion */
  double gp_steps_per_s;              /* gp_steps / wall_s */
} cw_serve_stats;

int cw_serve_default_config(cw_serve_config* c);
int cw_serve_create(const cw_serve_config* c, cw_server** out);
/* Ends the loop; requests still pending or running are dropped. */
int cw_serve_destroy(cw_server* s);
/* Queues a request: the case (copied) advanced by nsteps RK3 steps (nsteps >= 1; otherwise -1). id: its handle
 * for the calls below. A request whose footprint exceeds the whole budget is rejected (-2). */
int cw_serve_submit(cw_server* s, const cw_case* c, int nsteps, long long* id);
/* 0 when the request has finished, 1 on timeout (seconds < 0: wait without limit), < 0 failed / unknown */
int cw_serve_wait(cw_server* s, long long id, double seconds);
/* Waits until every submitted request has finished. */
int cw_serve_drain(cw_server* s);
/* A finished request's field (U_2 V_2 W_2 T_2 PH_2 MU_2 P AL, Q_2 species n), whole allocation in the
 * field's layout (cw_layout_of of the request's grid), as doubles. Needs keep_results. */
int cw_serve_result(cw_server* s, long long id, int field, int n, double* host, size_t count);
int cw_serve_latency(cw_server* s, long long id, double* seconds);
/* Drops a finished request's stored result. */
int cw_serve_release(cw_server* s, long long id);
int cw_serve_stats_get(cw_server* s, cw_serve_stats* out);
const char* cw_serve_last_error(cw_server* s);

#ifdef __cplusplus
}
#endif

#endif /* CW_SERVE_H */
