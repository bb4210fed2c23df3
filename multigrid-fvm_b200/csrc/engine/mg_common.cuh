// mg_common.cuh — device-side data layout of the engine.
//
// HBM layout: one pool allocation per context.  Every (case, level) owns NSLOTS_LEVEL
// FP64 arrays of npx*npy in the reference's row-major order (ij = j*npx + i,
// Version-6-26-04.c:554), each aligned to 256 B, plus an int tag array and an
// optional per-cell obstacle-code array.  The reference keeps one set of
// coefficient arrays (aw, ae, as, an, ap, su) that each equation overwrites in
// turn (:815-1092); here each equation has its own set, so the u, v and scalar
// equations of a level visit — which depend only on the fluxes at the start of the
// visit — are assembled in one kernel and smoothed in the same launches.  The
// reference's single prolongation scratch `c` (:1745-2028) becomes one correction
// array per variable for the same reason.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mgfvm.h"

namespace mg {

enum Eq { EQ_U = 0, EQ_V = 1, EQ_PP = 2, EQ_SC = 3 };
enum CoefK { CK_AW = 0, CK_AE, CK_AS, CK_AN, CK_AP, CK_SU, NCOEF };

enum Slot {
    S_U = 0, S_V, S_P, S_PP, S_SC,
    S_RESU, S_RESV, S_RESSC, S_APU, S_APV, S_SPU, S_SPV, S_SPSC,
    S_CX, S_CY, S_AREAX, S_AREAY, S_RS,
    S_C,                     // scalar prolongation correction (the reference's c after prolsc)
    S_CU, S_CV, S_CP,        // u, v, p prolongation corrections
    S_RU, S_RV, S_RP, S_RSC, // R(x_f) of u, v, p, sc as restv computed them (the gather's corrections)
    S_TMP0, S_TMP1, S_TMP2,  // Jacobi ping-pong buffers (u or p', v, sc)
    S_CO,                    // 4 equations x {aw, ae, as, an, ap, su}
    NSLOTS_LEVEL = S_CO + 4 * NCOEF,
    S_PREV_U = NSLOTS_LEVEL, S_PREV_V, S_PREV_P, S_PREV_SC,   // level 0 only
    NSLOTS
};

__host__ __device__ constexpr int co_slot(int eq, int k) { return S_CO + NCOEF * eq + k; }

constexpr int MAXLEV = 16;
constexpr int RED_STRIDE = 16;   // doubles per block in the reduction partials

// One multigrid level of one case.
struct LevelDev {
    int npx, npy;
    int ncopy;          // pressure-copy program length (update's obstacle loop)
    int hazard;         // the copy program reads a cell it also writes
    double dx, dy;
    double amu;         // viscosity on this level (amuf, :419)
    double amusc;       // scalar diffusivity amuf/prsc (:867)
    double *f[NSLOTS];
    int *tag;
    const unsigned *seq;  // per-cell obstacle-face addition codes, or nullptr
    const int *pdst;
    const int *psrc;
    double *pbuf;
    const int *pcode;   // the same copies done by k_update (mgfvm_obstacle_prog.fan), or nullptr
    const int *pfan;
};

constexpr int PCODE_DST = 1 << 30;   // pcode bit: the copy writes this cell
constexpr int PFAN_END = 1 << 30;    // pfan bit: last copy of its owner (PFAN_LAST of the host)

// Stop-rule and status flags of one case.
enum CaseStatus { CASE_RUNNING = 0, CASE_CONVERGED_REF = 1, CASE_CONVERGED_FP = 2,
                  CASE_NONFINITE = 4, CASE_BAD_LAUNCH = 8, CASE_WAIT_TIMEOUT = 16,
                  CASE_TAPE_ESCAPE = 32 };   // an adjoint phase wrote outside its tape (mg_adjoint.cu)

// Read-only description of one case during a launch (the host rewrites it between
// launches): physics, boundary codes, the level table and where histories and
// reduction scratch live.  Kernels take it through a const __restrict__ pointer so
// the level pointers can be cached instead of reloaded after every store.
struct CaseDev {
    // physics and boundary codes shared by every level (Version-6-26-04.c:30-35)
    double relxm, relxp, sc_obs, dpdxm, dpdym, convergence;
    int ibc_xm, ibc_xp, ibc_ym, ibc_yp;
    int ngrid;
    int tail;           // first level run by the one-CTA coarse kernel (== ngrid: none)
    int hist_cap;
    int stop_enabled;   // evaluate the stop rule at the end of every cycle
    double fp_tol;
    double *hist_err, *hist_delta;
    double *partials;   // RED_STRIDE doubles per block, reduction scratch
    unsigned *counters; // [0] mass error, [1] end of cycle
    LevelDev lv[MAXLEV];
};

// The part of a case that kernels write.
struct CaseState {
    int done;           // stop rule fired; every kernel skips this case
    int status;         // enum CaseStatus bits
    int ncyc;           // cycles recorded in the history
    int have_prev;      // level-0 state of a previous cycle is in S_PREV_*
    double last_err;    // level-0 sum|div| of the current cycle
    double shift_d, shift_p;  // last cycle's mean p change and mean p (shifted sums)
};

// ---------------------------------------------------------------- modes
// Which cases a launch at level `ig` touches.  Transfers are launched at their fine
// level; M_*_C launches act on the coarse level of a transfer whose fine level is ig-1.
enum Mode {
    M_OP = 0,       // single-step op on level ig
    M_OP_PAIR,      // single-step transfer between ig and ig+1
    M_OP_C,         // coarse side (ig) of a single-step transfer from ig-1
    M_DOWN,         // down-leg SIMPLE step on a grid-run level
    M_RESTRICT,     // restriction ig -> ig+1 from a grid-run level
    M_RESTRICT_C,   // coarse side (ig) of M_RESTRICT at ig-1
    M_PROLONG,      // prolongation ig+1 -> ig into a grid-run level
    M_UP            // up-leg SIMPLE step on level ig after M_PROLONG
};

__host__ __device__ __forceinline__ bool mode_active(const CaseDev &C, int ig, int mode)
{
    switch (mode) {
    case M_OP: return ig < C.ngrid;
    case M_OP_PAIR: return ig + 1 < C.ngrid;
    case M_OP_C: return ig >= 1 && ig < C.ngrid;
    case M_DOWN: return ig < C.tail;
    case M_RESTRICT: return ig < C.tail && ig + 1 < C.ngrid;
    case M_RESTRICT_C: return ig >= 1 && ig - 1 < C.tail && ig < C.ngrid;
    case M_PROLONG:
    case M_UP: return ig + 1 <= C.tail && ig + 1 < C.ngrid;
    default: return false;
    }
}

__device__ __forceinline__ bool case_active(const CaseDev &C, const CaseState &S, int ig, int mode)
{
    return !S.done && mode_active(C, ig, mode);
}

}  // namespace mg
