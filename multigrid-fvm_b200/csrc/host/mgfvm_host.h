/*
 * mgfvm_host.h — host-side helpers shared by the engine and the command-line tool.
 */
#ifndef MGFVM_HOST_H
#define MGFVM_HOST_H

#include "mgfvm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Record a failure message for mgfvm_last_error() and return `status`. */
int mgfvm_fail(int status, const char *fmt, ...);
void mgfvm_clear_error(void);

/* Obstacle k mapped to level ig, {is, ie, js, je}; empty {1,0,1,0} at ig >= ig_obs. */
void mgfvm_obstacle_range(const mgfvm_config *c, int k, int ig, int r[4]);

/* Precomputed obstacle programs of one level (see obstacles.c). */
typedef struct mgfvm_obstacle_prog {
    /* update's pressure copy (:1153-1177) resolved to a gather:
     * p[dst[k]] = p_before[src[k]], k < ncopy; `hazard` != 0 when some src is also a
     * dst, so the gather must read every source before writing any destination. */
    int ncopy;
    int *dst, *src;
    int hazard;
    /* coefsc's obstacle-face diffusion (:939-963) as a per-cell sequence code:
     * cells[k] receives, in order, the additions encoded in codes[k] (see obstacles.c). */
    int nseq;
    int *cells;
    unsigned *codes;
    int max_adds;      /* longest sequence seen */
    int touches_outlet; /* a copy reads or writes column npx-2 or npx-1 (the outflow's columns) */
    /* The same copies grouped by the interior cell whose update thread performs them
     * (the source itself when it is interior, else the nearest interior cell):
     * owners[k] in increasing order, fan[2k] = destination | PFAN_LAST on the last copy
     * of an owner, fan[2k+1] = source index when it lies on the boundary ring (the
     * owner reads its value) or -1 (the owner's own updated pressure).  Built only when
     * hazard == 0. */
    int *owners;
    int *fan;
} mgfvm_obstacle_prog;

#define PFAN_LAST (1 << 30)

int mgfvm_build_obstacle_prog(const mgfvm_config *c, int ig, mgfvm_obstacle_prog *out);
void mgfvm_free_obstacle_prog(mgfvm_obstacle_prog *p);

#ifdef __cplusplus
}
#endif
#endif
