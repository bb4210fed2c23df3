// mg_adjoint.cuh — reverse-mode (adjoint) derivatives of the V-cycle iteration.
//
// The V-cycle (Version-6-26-04.c:195-249) is written here as a program of phases, each
// a parallel map of one cell routine of mg_cells.cuh over one level (or a pair of
// levels): an assembly of one equation, one half-sweep of one equation, masserror +
// coefp, update, the obstacle pressure copy, outflow, restv, the fine residuals, the
// FAS defects, the prolongation.  Every phase is non-interfering — no cell reads a
// location another cell of the same phase writes — which is what lets the forward
// sweep run each phase as one parallel pass and lets its transpose be formed cell by
// cell:
//
//   forward (taped)  before each phase, copy the arrays it overwrites to a tape; run it.
//   reverse          for each phase, last to first: restore its overwritten arrays from
//                    the tape (the state is then its input), then for every cell
//                      1. evaluate the cell routine once, reading the adjoints of the
//                         values it writes and clearing them (the writes replace them),
//                      2. evaluate it again once per value it reads, with that read
//                         seeded (a dual number of derivative 1), and add
//                         adjoint(out) * d(out)/d(read) to the read location's adjoint.
//
// Step 2 runs the same routine in the same dual arithmetic as the forward-mode tangent
// (mg_tangent.cuh), so the reverse sweep applies exactly the transpose of the Jacobian
// the tangent kernel applies, non-smooth points included.  Contributions are added
// with atomics (one location may be read by several cells), so the adjoint's rounding
// depends on the order in which they land; the derivative itself does not.
#pragma once

#include <vector>

#include "mg_kernels.cuh"
#include "mg_tangent.cuh"

namespace mg {

enum PhaseKind {
    P_ASM_U = 0, P_ASM_V, P_ASM_SC,   // coefu + umom, coefv + vmom, coefsc + scalar (one equation)
    P_SC_OUTFLOW,                      // the scalar ghost column of outflow (:1226), down leg
    P_GS,                              // one red-black half-sweep of one equation: a = eq, b = colour
    P_JAC_RING,                        // Jacobi: the ping-pong buffer's ring from the field: a = eq
    P_JAC_SWEEP,                       // one Jacobi sweep: a = eq, b = 0 field -> buffer, 1 buffer -> field
    P_JAC_COPY,                        // Jacobi, odd sweep count: the buffer back to the field: a = eq
    P_MASS_COEFP,                      // masserror + coefp: a = MC_COEF (p' = 0, coefficients) or MC_SU
    P_UPDATE,                          // update: a = 1 u, 2 v, 4 p
    P_PFIX,                            // update's obstacle pressure copy (no chained copies)
    P_PFIX_GATHER, P_PFIX_SCATTER,     // the same copy through its buffer (chained copies)
    P_OUTFLOW,                         // outflow of u, v, p (b = 1: and the scalar ghost)
    P_RESTV,                           // restv: coarse state and R(x_f) of a = 1 u, 2 v, 4 p, 8 sc
    P_FINE_RES,                        // fine residual of equation a (0 u, 1 v, 2 sc) into its buffer
    P_RESTRICT,                        // FAS defect of equation a on the coarse level
    P_PROL_CORR, P_PROL_APPLY,         // prolongation: coarse corrections, fine gather (a as restv)
    P_NKINDS
};

// One phase of a case's V-cycle program; `off` is the tape offset (doubles) of the
// arrays it overwrites.
struct Phase {
    int kind, ig, a, b;
    long long off;
};

// What a case's adjoint kernel reads: its program, tape, and the per-level adjoints
// of the viscosity and scalar diffusivity it accumulates (2 per level: amu, amusc).
struct CaseAdj {
    const Phase *prog;
    int nphase;
    double *tape;
    double *pacc;
    int generic;   // transpose every phase by dual-number probes (the closed forms' check)
};

// Bit `s` of the mask: slot s of the written level; PB_BIT: the pressure-copy buffer.
constexpr int PB_BIT = 63;
static_assert(NSLOTS <= PB_BIT, "slot masks need one bit per slot");

// The phase program of one V-cycle of a case and the tape doubles it needs.  Returns
// false for configurations the adjoint does not cover (periodic boundaries).
bool build_adj_program(const CaseDev &hc, const Sched &S, std::vector<Phase> &prog, long long &tape_doubles);

// One V-cycle of every case, taped, then its transpose: the adjoint arrays `dt` (the
// derivative storage of mg_tangent.cuh, one array per differentiable slot) go from the
// adjoint of the state after the cycle to that of the state before it.  A cluster of
// `cluster` (1..8) CTAs per case; a case with an empty program is skipped.
cudaError_t launch_adj_cycle(const CaseDev *dc, CaseState *ds, const CaseTan *dt, const CaseAdj *da, int ncases,
                             int cluster, cudaStream_t st);

// CTAs per case of launch_adj_cycle for a batch of `ncases` on `sms` multiprocessors:
// the largest power of two up to 8 that keeps every case's cluster resident at once.
int adj_cluster_size(int ncases, int sms);

// Copy the u, v, p, sc arrays of every level of every case to (dir 0) or from (dir 1)
// `buf`; case c's part starts at off[c] (doubles), levels and slots in order.
cudaError_t launch_live_copy(const CaseDev *dc, const long long *off, double *buf, int ncases, int maxcells,
                             int maxng, int dir, cudaStream_t st);

constexpr int ADJ_BLOCK = 1024;

}  // namespace mg
