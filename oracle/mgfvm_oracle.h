/*
 * mgfvm_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the reference solver's V-cycle
 * (akashu4295/Multigrid-FVM, Version-6-26-04.c) used as the parity checker of
 * the CUDA engine.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline call it.  It is pinned against the reference itself: tests compare it
 * bit for bit with fixtures produced by the reference code compiled with gcc
 * (tests/golden/, generated by tests/golden/make_golden.py through
 * oracle/ref_harness.c).
 */
#ifndef MGFVM_ORACLE_H
#define MGFVM_ORACLE_H

#include "mgfvm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_case orc_case;

/* init (:546-676) + rest_geom (:1391-1473); `inlet_u` (may be NULL) is a
 * per-face level-0 inlet profile of `n_inlet` rows applied between the two. */
int  orc_create(const mgfvm_config *cfg, const double *inlet_u, int n_inlet,
                orc_case **out);
void orc_destroy(orc_case *c);

int  orc_ngrid(const orc_case *c);
int  orc_dims(const orc_case *c, int level, int *npx, int *npy);
int  orc_get(const orc_case *c, int level, int field, double *out);
int  orc_set(orc_case *c, int level, int field, const double *in);
int  orc_get_tag(const orc_case *c, int level, int *out);
int  orc_get_obstacle_ranges(const orc_case *c, int level, int *out);

/* One V-cycle (:195-249); records the level-0 mass error and the fixed-point
 * change (see mgfvm_solve in mgfvm.h). */
void orc_cycle(orc_case *c);
/* Cycles until err < convergence or delta < fp_tol (fp_tol <= 0: off) or
 * max_cycles; returns cycles run. */
int  orc_solve(orc_case *c, int max_cycles, double fp_tol);
int  orc_history(const orc_case *c, double *err, double *delta, int cap);
/* One routine of enum mgfvm_op on `level`. */
int  orc_op(orc_case *c, int op, int level);
/* Mass error of the last masserror call on any level. */
double orc_last_err(const orc_case *c);

#ifdef __cplusplus
}
#endif
#endif
