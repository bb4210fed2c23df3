// mg_kernels.cuh — host-side launchers of the engine's kernels.
#pragma once

#include <cuda.h>

#include "mg_common.cuh"

namespace mg {

// One kernel launch of a V-cycle (or single-op) schedule.
enum KernelId {
    K_FLUXES = 0,    // fluxes only (single-op)
    K_ASM,           // fused assembly: a0 = AsmBits, a1 = 1: fluxes recomputed live
    K_MASS_COEFP,    // a0 = reduce the mass error into CaseDev::last_err
    K_UPDATE,
    K_PFIX,          // a0 = phase (0 gather, 1 scatter, 2 both)
    K_BOUND,         // a0 = bits: 1 periodic, 2 outflow u/v/p, 4 outflow sc
    K_SMOOTH,        // tile smoother: a0 = eq mask, a1 = first unit, a2 = units, a3 = dir, a4 = tile
    K_COPY,          // copy equations' buffers back: a0 = eq mask
    K_RESTV_FLUXES,  // restv + fine fluxes
    K_RESTRICT,      // restr{u,v,sc} + coarse fluxes
    K_PROL_CORR, K_PROL_APPLY,   // prol_apply: a0 = 1 forms the corrections itself (no K_PROL_CORR before it)
    K_TAIL, K_ENDCYCLE, K_PROL_APPLY_END,
    K_SMOOTH_F32,    // mixed precision: the tiles of K_SMOOTH on FP32 operands and corrections
                     // (a3 = flags: 1 first, 2 last, 4 read buffer 1, 8 operands read
                     // before the wait for the previous launch)
    K_PFIX_BOUND,    // K_PFIX then K_BOUND (a0 = bits), one CTA per case
    K_PP_LEVEL,      // masserror+coefp, p' smoothing, update on a one-CTA level: a0 = units,
                     // a1 = reduce, a2 = update fuse bits
    K_TAIL_TAN,      // K_TAIL with derivatives (a tangent context)
    K_LEVEL_VISIT,   // a whole one-CTA level visit, a cluster of 3 CTAs per case: K_PP_LEVEL's
                     // a0-a2, a3 = assembly bits (0: done), a4 = u/v/sc units
    K_SMOOTH_TMA,    // as K_SMOOTH, the region staged by TMA box loads (bw, bh, ptr)
    K_BAND_VISIT,    // a whole level visit, a cluster of grid.x CTAs per case (bands of rows):
                     // K_LEVEL_VISIT's arguments
    K_COARSE_CYCLE,  // the V-cycle from the restriction into level a0 (every level from a0
                     // one CTA holds) to the prolongation out of it, a cluster of 3 CTAs per
                     // case: a1 = p' units, a2 = u/v/sc units
    K_NKERNELS
};

struct Launch {
    int kernel;
    int ig;            // level (fine level for transfers)
    int mode;          // enum Mode
    int a0, a1, a2, a3, a4;
    dim3 grid;
    int block;
    int smem;
    int bw, bh;        // K_SMOOTH_TMA: box width and height
    int map;           // K_SMOOTH_TMA: index of its first tensor-map pair in the schedule's table
    const void *ptr;   // K_SMOOTH_TMA: that pair on the device (one per case)
};

// The tensor maps of one case for a TMA-staged smoother launch: the level's slot
// arrays as one (x, y, slot) tensor, with a box of NCOEF slots (the coefficients) and
// one of a single slot (the field).
struct __align__(64) SmoothMap {
    CUtensorMap coef, field;
};

// Polls of an mbarrier wait before a TMA-staged smoother CTA gives up on its loads.
constexpr int TMA_WAIT_POLLS = 1 << 22;

struct Sched {
    int isolve, nswpm, nswpp;
    int tma_wait_polls;   // first wait of a TMA-staged smoother CTA (mgfvm_tuning.tma_first_wait)
    bool pdl;             // launch with programmatic stream serialization (mgfvm_tuning.pdl)
};

// Tile smoother geometry: a CTA of SMOOTH_BLOCK (one per SM) or SMOOTH_BLOCK/2 (two per
// SM) threads, one vertical cell pair per thread, covers a tile plus a halo of one cell
// per unit on every side.
constexpr int SMOOTH_BLOCK = 1024;
// band visits: at most 8 CTAs per case (the portable cluster size) and this much
// dynamic shared memory per CTA (the band and its two halo rows, two buffers for Jacobi)
constexpr int BAND_MAX_CTAS = 8;
constexpr int BAND_SMEM_MAX = 80 * 1024;
// By default a level runs band visits in batches of at least this many cases (of one
// size at that level): a unit costs about a microsecond there (its cluster barrier),
// which only pays when the tile launches it replaces have enough work to be slow too
// (256^2 cases, levels 1-2: slower up to 16 cases, faster from 32)
constexpr int BAND_MIN_CASES = 32;
// interior rows of each band when G CTAs share a level of npy padded rows (even; the
// last band may be shorter)
__host__ __device__ __forceinline__ int band_rows(int npy, int G)
{
    const int b = (npy - 2 + G - 1) / G;
    return (b + 1) & ~1;
}
constexpr int MAX_UNITS = 10;   // default cap of half-sweeps (GS) or sweeps (Jacobi) per launch
constexpr int MIN_TILE = 8;     // smallest tile side a units cap may leave
int smooth_pairs_side(int units, int threads);   // tile side whose region fits `threads` pairs

struct CaseTan;
// `dtan`: the derivative storage of a tangent context (K_TAIL_TAN), else unused
cudaError_t launch_one(const Launch &L, const CaseDev *dcases, CaseState *dstate, const CaseTan *dtan,
                       const Sched &S, cudaStream_t stream);
cudaError_t configure_kernels();

// Kernels of the raw-pointer entry points.
cudaError_t raw_jacobi(const double *aw, const double *ae, const double *as, const double *an,
                       const double *ap, const double *su, double *phi, double *scratch, int npx,
                       int npy, int nx, int ny, int nsw, cudaStream_t s);
cudaError_t raw_rbgs(const double *aw, const double *ae, const double *as, const double *an,
                     const double *ap, const double *su, double *phi, int npx, int npy, int nx,
                     int ny, int nsw, cudaStream_t s);
cudaError_t raw_masserror(const double *u, const double *v, const double *ax, const double *ay,
                          double *su, double *pp, int npx, int npy, double *err_out,
                          double *partials, cudaStream_t s);
size_t raw_masserror_blocks(int npx, int npy);
cudaError_t raw_check_division(long long n, unsigned long long seed, unsigned long long *bad, cudaStream_t s);

constexpr int BLOCK = 256;
constexpr int PFIX_BOUND_BLOCK = 1024;
constexpr int SMOOTH_TMA_SMEM_MAX = 200 * 1024;   // dynamic shared memory of a TMA-staged smoother CTA
constexpr int TAIL_BLOCK = 512;
constexpr int TAIL_SMEM_MAX = 220 * 1024;   // dynamic shared memory of the coarse kernel (+ its static 256 B)

}  // namespace mg
