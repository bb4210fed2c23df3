/*
 * mgfvm.h — C ABI of the B200 engine for the staggered-grid SIMPLE solver with a
 * FAS multigrid V-cycle (akashu4295/Multigrid-FVM, Version-6-26-04.c).
 *
 * The reference is one C program whose state lives in globals (Version-6-26-04.c:27-39)
 * and in one `struct SoA` per multigrid level (:42-54).  This header replaces that
 * process-global interface with an opaque context that owns every level of every
 * case on one GPU.  A single solve is a batch of one case.
 *
 * Conventions shared by every entry point:
 *   - every function returns an int status (MGFVM_OK on success); the message of
 *     the last failure on the calling thread is returned by mgfvm_last_error();
 *     nothing in the library calls exit().  (The reference exits the process on
 *     any parse or allocation error: :283-291, :106-114, :2369-2378.)
 *   - arrays use the reference layout: level `ig` is npx x npy doubles with
 *     npx = nfx/2^ig + 2, npy = nfy/2^ig + 2 (:408-411), row-major, ij = j*npx + i.
 *   - host buffers passed in or out are plain host memory owned by the caller;
 *     device memory is owned by the context, except for the raw-pointer kernel
 *     entry points at the end of this file, which take caller-owned device memory.
 *   - calls on one context are not thread-safe; use one context per host thread.
 */
#ifndef MGFVM_H
#define MGFVM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGFVM_ABI_VERSION 1

/* ---------------------------------------------------------------- status */
enum mgfvm_status {
    MGFVM_OK = 0,
    MGFVM_EINVAL = 1,       /* malformed InputData/pattern or bad argument        */
    MGFVM_EIO = 2,          /* file missing or unreadable                         */
    MGFVM_EOOB = 3,         /* obstacle/inlet/outlet index range leaves the grid  */
    MGFVM_ENONFINITE = 4,   /* NaN or Inf in the mass-error history               */
    MGFVM_ETIMEOUT = 5,     /* a bounded device-side wait gave up                 */
    MGFVM_ECUDA = 6,        /* CUDA runtime error                                 */
    MGFVM_ENOMEM = 7,       /* host or device allocation failed                   */
    MGFVM_EUNSUPPORTED = 8  /* valid input this build does not handle             */
};

/* ---------------------------------------------------------------- fields */
/* One id per array of `struct SoA` (Version-6-26-04.c:42-54). */
enum mgfvm_field {
    MGFVM_F_U = 0, MGFVM_F_V, MGFVM_F_P, MGFVM_F_PP, MGFVM_F_SC,
    MGFVM_F_SU, MGFVM_F_RS, MGFVM_F_RESU, MGFVM_F_RESV, MGFVM_F_RESSC,
    MGFVM_F_C,
    MGFVM_F_AW, MGFVM_F_AE, MGFVM_F_AS, MGFVM_F_AN, MGFVM_F_AP,
    MGFVM_F_APU, MGFVM_F_APV, MGFVM_F_SPU, MGFVM_F_SPV, MGFVM_F_SPSC,
    MGFVM_F_CX, MGFVM_F_CY, MGFVM_F_AREAX, MGFVM_F_AREAY,
    MGFVM_NFIELDS
};

/* ------------------------------------------------------ single-step ops */
/* The per-level routines of one V-cycle, for parity tests and for callers that
 * drive their own cycle (Version-6-26-04.c:195-249).  `level` is the level the
 * routine acts on; RESTRICT acts on (level -> level+1), PROLONG on
 * (level+1 -> level). */
enum mgfvm_op {
    MGFVM_OP_FLUXES = 0,      /* fluxes        :678-694                          */
    MGFVM_OP_SOLVE_U,         /* solve_u       :696-703   coefu, umom, smoother   */
    MGFVM_OP_SOLVE_V,         /* solve_v       :705-712                          */
    MGFVM_OP_SOLVE_PP,        /* solve_pprime  :714-728   masserror..update       */
    MGFVM_OP_PBOUND,          /* pbound        :1179-1210                        */
    MGFVM_OP_OUTFLOW,         /* outflow       :1211-1228                        */
    MGFVM_OP_SOLVE_SC,        /* solve_sc      :729-737                          */
    MGFVM_OP_RESTRICT,        /* restv, fluxes(c), fluxes(f), restru, restrv, restrsc :211-220 */
    MGFVM_OP_PROLONG,         /* prolu, prolv, prolp, prolsc :230-233           */
    MGFVM_OP_SMOOTH_U,        /* the smoother alone on u with the current coefficients */
    MGFVM_OP_SMOOTH_V,
    MGFVM_OP_SMOOTH_PP,
    MGFVM_OP_SMOOTH_SC,
    MGFVM_NOPS
};

/* Linear smoothers (InputData isolve, :1231-1351). */
enum { MGFVM_JACOBI = 1, MGFVM_GAUSS_SEIDEL = 2 };

/* Arithmetic of the V-cycle. */
enum mgfvm_precision {
    MGFVM_PREC_FP64 = 0,   /* every array and every operation in FP64, as the reference */
    MGFVM_PREC_MIXED = 1   /* the smoothers iterate an FP32 correction against an FP64
                              residual taken at the start of every smoother launch; the
                              coarsest level, assembly, transfers, defects and norms stay
                              FP64, so fixed points are those of the FP64 equations      */
};

#define MGFVM_MAX_PORTS 10   /* inlet/outlet arrays of the reference hold 10 (:29, :38) */

/* ------------------------------------------------------------ one case */
/* Everything InputData and pattern.txt hold, field for field (README.md:6-29,
 * readInput Version-6-26-04.c:280-401, read_obstacle_data :2367-2400). */
typedef struct mgfvm_config {
    /* InputData line 1 */
    int nfx, nfy, ngrid, ig_obs, ibeg_obs, ig_inlt, ig_outlt;
    int nvcycle, nswpm, nswpp, isolve;
    double omega, convergence;
    /* line 2 */
    double xl, yl, amuf, prsc, relxm, relxp;
    /* line 3: 1 fixed value, 2 p' Dirichlet, 3 periodic, 4 outflow (x+ only) */
    int ibc_xm, ibc_xp, ibc_ym, ibc_yp;
    /* lines 4-7 */
    double u_xm, v_xm, p_xm, sc_xm;
    double u_xp, v_xp, p_xp, sc_xp;
    double u_ym, v_ym, p_ym, sc_ym;
    double u_yp, v_yp, p_yp, sc_yp;
    /* line 8 */
    double u_guess, v_guess, p_guess, sc_guess;
    /* line 9 */
    double sc_obs;
    /* discrete inlets and outlets */
    int ninlt;
    int jfinlt[MGFVM_MAX_PORTS], jlinlt[MGFVM_MAX_PORTS];
    double uinlt[MGFVM_MAX_PORTS], vinlt[MGFVM_MAX_PORTS], scinlt[MGFVM_MAX_PORTS];
    int noutlt;
    int jfoutlt[MGFVM_MAX_PORTS], jloutlt[MGFVM_MAX_PORTS];
    double uoutlt[MGFVM_MAX_PORTS], voutlt[MGFVM_MAX_PORTS], scoutlt[MGFVM_MAX_PORTS];
    /* pattern.txt: nobs rectangles {if, il, jf, jl} (1-based, on level ig_obs-1) */
    int nobs;
    int *obs;          /* 4*nobs ints; owned by whoever filled the struct */
    /* body-force pressure gradients; declared but never read by the reference (:33) */
    double dpdxm, dpdym;
} mgfvm_config;

/* Context options. */
typedef struct mgfvm_options {
    int device;        /* CUDA device ordinal                                        */
    int precision;     /* enum mgfvm_precision                                       */
    int tail_level;    /* first level run by the one-CTA-per-case coarse kernel;
                          -1 = chosen by the tuner, >= ngrid = no coarse kernel      */
    int use_graph;     /* replay V-cycles from a captured CUDA graph (1) or launch
                          every kernel directly (0)                                   */
    int sync_every;    /* cycles per chunk of mgfvm_solve; the host reads a chunk's stop
                          flags while the next chunk runs (stopped cases skip it)     */
    int tangent;       /* 1: every case also carries the derivative of its state along
                          one parameter direction (mgfvm_set_direction); FP64 only, and
                          the whole V-cycle runs in the one-CTA-per-case kernel       */
} mgfvm_options;

/* Per-level schedule choices (index = level; 0 = the engine's default).  Every choice
 * gives the same bits; only the launch shapes change. */
#define MGFVM_MAX_LEVELS 16
typedef struct mgfvm_tuning {
    int smooth_units[MGFVM_MAX_LEVELS];    /* smoother units (GS half-sweeps or Jacobi
                                              sweeps) per tile launch, >= 1             */
    int smooth_threads[MGFVM_MAX_LEVELS];  /* smoother CTA: 1024 (one per SM), 512 (two)
                                              or 256 threads (four)                     */
    int asm_slices[MGFVM_MAX_LEVELS];      /* assembly threads per cell: 1 or 3         */
    int restrict_slices[MGFVM_MAX_LEVELS]; /* restriction threads per cell: 1 or 3      */
    int update_pfix[MGFVM_MAX_LEVELS];     /* obstacle pressure copy inside update where
                                              legal: 0 or 2 yes, 1 no (own kernel)      */
    int odd_chunks[MGFVM_MAX_LEVELS];      /* an odd number of tile-smoother launches may
                                              leave the result in the ping-pong buffers
                                              for the next kernel to take: 0 or 2 yes,
                                              1 no (even launch counts only)            */
    int pp_level[MGFVM_MAX_LEVELS];        /* on a level one CTA per case holds: the
                                              whole visit (assembly, u/v/sc smoothing,
                                              p', update) in one launch: 0 or 2 yes,
                                              1 no                                      */
    int smooth_tma[MGFVM_MAX_LEVELS];      /* tile smoother regions staged in shared memory
                                              by TMA box loads: 2 yes, 0 or 1 no        */
    int coarse_kernel[MGFVM_MAX_LEVELS];   /* 2: this level and every coarser one run in
                                              the one-CTA-per-case coarse kernel (the
                                              first level marked 2 counts); 0 or 1
                                              everywhere: mgfvm_options.tail_level      */
    int prol_fused[MGFVM_MAX_LEVELS];      /* prolongation into this level forms the coarse
                                              corrections in the gather from the
                                              restriction's saved R(x_f) (no separate
                                              correction kernel): 0 or 2 yes, 1 no      */
    int tma_first_wait;                    /* polls of a TMA-staged smoother CTA's first
                                              wait for its loads before it gives up and
                                              the call fails with MGFVM_ETIMEOUT: 0 = the
                                              default (2^22), n > 0 = n, -1 = none (the
                                              wait gives up at once; exercises the
                                              timeout path)                             */
    int pdl;                               /* programmatic dependent launch between the
                                              V-cycle's kernels (a kernel's CTAs are
                                              scheduled while its predecessor finishes
                                              and wait for it on the device): 0 or 2
                                              yes, 1 no                                 */
    int band_visit[MGFVM_MAX_LEVELS];      /* on a level too large for one CTA per case but
                                              held by a cluster of at most 8 (bands of
                                              rows, halo rows exchanged in distributed
                                              shared memory; FP64 in either precision):
                                              the whole visit in one launch: 2 yes, 1 no,
                                              0 yes in batches of at least 32 cases
                                              that all have the level at one size      */
    int coarse_cluster;                    /* every level from the first one a CTA per case
                                              holds down to the coarsest, with the
                                              transfers into and out of it, as one launch
                                              of a cluster of three CTAs per case: 2 yes,
                                              0 or 1 no (measured slower: its transfers
                                              run on three SMs)                         */
} mgfvm_tuning;

typedef struct mgfvm_ctx mgfvm_ctx;

/* ------------------------------------------------------ configuration */
void mgfvm_config_default(mgfvm_config *cfg);
void mgfvm_options_default(mgfvm_options *opt);

/* Parse InputData and pattern.txt exactly as readInput/read_obstacle_data do
 * (Version-6-26-04.c:280-401, :2367-2400; pattern.txt is read between lines 8
 * and 9 of InputData, :357).  cfg->obs is allocated by the library; release it
 * with mgfvm_config_release.  `verbose` != 0 prints the reference's echo lines
 * to stdout. */
int mgfvm_config_read(const char *inputdata_path, const char *pattern_path,
                      mgfvm_config *cfg, int verbose);
void mgfvm_config_release(mgfvm_config *cfg);

/* Check a configuration against the grid: level sizes divisible by 2^(ngrid-1),
 * every obstacle/inlet/outlet range inside the padded grid of every level it
 * touches, supported boundary codes.  Returns MGFVM_EINVAL/MGFVM_EOOB/... */
int mgfvm_config_validate(const mgfvm_config *cfg);

/* ------------------------------------------------------------ context */
/* Build the device state of `ncases` independent cases (AllocateMemorySoA :402-506,
 * init :546-676, rest_geom :1391-1473) and upload it.  All cases must share
 * isolve, nswpm and nswpp; grid sizes, ngrid, physics and obstacles may differ. */
int mgfvm_create(const mgfvm_config *cases, int ncases, const mgfvm_options *opt,
                 mgfvm_ctx **out);
int mgfvm_destroy(mgfvm_ctx *ctx);

/* Return every case to its initial state (init + rest_geom) and clear histories. */
int mgfvm_reset(mgfvm_ctx *ctx);

/* Per-face inlet profile: level-0 u at the x- boundary face of rows j = 1..n
 * (n = nfy), applied after init and before rest_geom, so coarse levels take the
 * face average of it (rest_geom :1440-1446).  Resets that case. */
int mgfvm_set_inlet_profile(mgfvm_ctx *ctx, int icase, const double *u, int n);

/* Run exactly `ncycles` V-cycles on every case (no stop test). */
int mgfvm_cycle(mgfvm_ctx *ctx, int ncycles);

/* Run V-cycles until every case has stopped or `max_cycles` have run.  A case stops
 * after the cycle whose level-0 mass error is below its `convergence` (the
 * reference test, :247-248), or whose fixed-point change is below `fp_tol`
 * (fp_tol <= 0 disables that rule).  The fixed-point change of cycle k is
 *   max over f in {u, v, sc, p - mean(p)} of ||f_k - f_{k-1}||_2 / ||f_k||_2
 * over the level-0 interior.  cycles_out[c] (may be NULL) receives the number of
 * cycles case c ran. */
int mgfvm_solve(mgfvm_ctx *ctx, int max_cycles, double fp_tol, int *cycles_out);

/* Per-cycle history of case `icase`: err[k] = level-0 sum |div| measured before the
 * cycle's p' correction (convergence_data, :717-724); delta[k] = the fixed-point
 * change defined above, tracked only by mgfvm_solve with fp_tol > 0 (0 for the
 * first cycle of such a solve and for every cycle run otherwise).  Either pointer may
 * be NULL.  *n_out = cycles recorded (<= cap are copied). */
int mgfvm_history(mgfvm_ctx *ctx, int icase, double *err, double *delta, int cap,
                  int *n_out);

/* --------------------------------------------------------- data access */
int mgfvm_num_levels(mgfvm_ctx *ctx, int icase, int *ngrid);
int mgfvm_level_dims(mgfvm_ctx *ctx, int icase, int level, int *npx, int *npy);
/* Copy one array of one level of one case (npx*npy doubles) to or from the host. */
int mgfvm_get_field(mgfvm_ctx *ctx, int icase, int level, int field, double *out);
int mgfvm_set_field(mgfvm_ctx *ctx, int icase, int level, int field, const double *in);
/* Zero-copy access: the device address of one array of one level of one case
 * (npx*npy doubles, row-major ij = j*npx + i), owned by the context and valid until
 * mgfvm_destroy.  Reads and writes through it must be ordered with the context's
 * stream (mgfvm_stream).  For the coefficient fields (aw ... ap) the address is that
 * of the equation most recently assembled on the level at the time of the call. */
int mgfvm_field_device_ptr(mgfvm_ctx *ctx, int icase, int level, int field, double **ptr, int *npx,
                           int *npy);
/* The cell tag of one level (1 fluid, 0 obstacle; init :617-641), npx*npy ints. */
int mgfvm_get_tag(mgfvm_ctx *ctx, int icase, int level, int *out);
/* Obstacle index ranges of one level after the level mapping of :468-478.  Levels
 * at or above ig_obs hold the empty range {1, 0, 1, 0}.  out: 4*nobs ints
 * {is, ie, js, je}. */
int mgfvm_get_obstacle_ranges(mgfvm_ctx *ctx, int icase, int level, int *out);

/* Run one single-step op (enum mgfvm_op) on `level` of every case. */
int mgfvm_op(mgfvm_ctx *ctx, int op, int level);

/* Number of kernels this context launched since creation (graph replays count
 * each kernel node). */
int mgfvm_kernel_launches(mgfvm_ctx *ctx, long long *out);

/* Wall-clock of the last mgfvm_cycle/mgfvm_solve measured with CUDA events on the
 * context stream, in milliseconds. */
int mgfvm_last_elapsed_ms(mgfvm_ctx *ctx, double *ms);

/* The CUDA stream the context launches on (a cudaStream_t). */
int mgfvm_stream(mgfvm_ctx *ctx, void **stream);

/* Time `reps` back-to-back runs of single-step op `op` on `level` of every case with
 * CUDA events on the context stream: the op's launches are captured into a CUDA graph
 * once and the graph is replayed `reps` times after one untimed replay, so no host
 * launch overhead sits between the events.
 * *ms_total = elapsed milliseconds, *launches = kernels launched in that window. */
int mgfvm_time_op(mgfvm_ctx *ctx, int op, int level, int reps, double *ms_total, int *launches);

/* Run one V-cycle with every kernel launched directly and a CUDA event recorded
 * after each launch on the context stream; ms[k] = time between the events around
 * launch k (its device duration plus any gap before it), kernel[k] = the engine's
 * kernel id, level[k] = its level.  Up to `cap` entries; *n_out = launches. */
int mgfvm_profile_cycle(mgfvm_ctx *ctx, double *ms, int *kernel, int *level, int cap, int *n_out);

/* The context's schedule choices, and replacing them (the V-cycle graph is rebuilt).
 * Values outside the allowed sets are rejected with MGFVM_EINVAL. */
int mgfvm_get_tuning(mgfvm_ctx *ctx, mgfvm_tuning *t);
int mgfvm_set_tuning(mgfvm_ctx *ctx, const mgfvm_tuning *t);

/* Autotuner: time V-cycles of this batch under candidate schedule choices (level by
 * level, `cycles` graph-replayed cycles per candidate, best of two) and keep the
 * fastest.  The batch's state is saved before and restored after, so results are as
 * if the call had not happened.  *ms_before / *ms_after = milliseconds per cycle
 * under the initial and the chosen schedule (either may be NULL); `chosen` may be
 * NULL.  No counterpart in the reference. */
int mgfvm_autotune(mgfvm_ctx *ctx, int cycles, mgfvm_tuning *chosen, double *ms_before, double *ms_after);

/* ------------------------------------------------------------ derivatives
 * Forward-mode (tangent-linear) derivatives of the V-cycle iteration.  In a context
 * created with mgfvm_options.tangent = 1, every value of every case is paired with
 * its derivative along the case's parameter direction; each V-cycle advances both
 * with the reference's operations (same value bits as a plain context), so after n
 * cycles the derivative arrays hold d(state after n cycles)/d(parameter) exactly,
 * the quantity a central finite difference of the reference's n cycles
 * approximates.  A batch of cases with the same inputs and different directions
 * gives a whole gradient in one run.  No counterpart in the reference.
 *
 * Directions: the level-0 inlet velocity u at face row index+1 of the x- boundary
 * (index in [0, nfy), the per-face inlet profile of mgfvm_set_inlet_profile), the
 * viscosity amuf, the Prandtl-type number prsc (scalar diffusivity amuf/prsc). */
enum mgfvm_direction { MGFVM_DIR_NONE = 0, MGFVM_DIR_INLET = 1, MGFVM_DIR_AMUF = 2, MGFVM_DIR_PRSC = 3 };

/* Set case `icase`'s direction and return it to its initial state with the
 * derivative seeded (zero state derivative; the inlet face's own value, the coarse
 * faces rest_geom averages from it, or the derivatives of amu and amusc). */
int mgfvm_set_direction(mgfvm_ctx *ctx, int icase, int kind, int index);

/* Derivative array of a field (npx*npy, as mgfvm_get_field); zeros for arrays no
 * parameter changes (face areas, obstacle sources). */
int mgfvm_get_tangent(mgfvm_ctx *ctx, int icase, int level, int field, double *out);

/* Objective of the level-0 state: J = mean_j p(1, j) - mean_j p(npx-2, j) +
 * mean_j sc(npx-1, j) over the interior rows j = 1 .. npy-2 (uniform dy, so the
 * dy-weighted means are plain means): the inlet-to-outlet pressure drop plus the
 * mean outlet scalar.  *dJ (tangent contexts; may be NULL) = its derivative along
 * the case's direction.  Either pointer may be NULL. */
int mgfvm_objective(mgfvm_ctx *ctx, int icase, double *J, double *dJ);

/* Whole gradient of J after `ncycles` V-cycles from the initial state of `cfg` with
 * the given per-face inlet profile (may be empty): creates a tangent context of
 * nfy + 2 cases (every inlet face, amuf, prsc) on `device`, runs it and releases it;
 * where the device cannot hold them all, the directions run in batches of half the
 * size, halved again until one fits (the environment variable MGFVM_GRADIENT_BATCH,
 * if set to n >= 1, caps a batch at n directions).  dJ_dinlet receives nfy values; any output may be
 * NULL. */
int mgfvm_gradient(const mgfvm_config *cfg, const double *inlet_u, int n_inlet, int ncycles, int device,
                   double *J, double *dJ_dinlet, double *dJ_damuf, double *dJ_dprsc);

/* Reverse mode (discrete adjoint) of the same iteration: every case of a plain FP64
 * context is returned to its initial state and run `ncycles` V-cycles, then the
 * transpose of those cycles is applied from the adjoint of J (mgfvm_objective) back to
 * the initial state, so one call gives the whole gradient of every case's J after
 * ncycles cycles — the inlet faces, amuf and prsc — at the cost of a few V-cycles per
 * cycle instead of nfy + 2 tangent runs.  Each cycle is transposed phase by phase:
 * the cycle is re-run with the arrays every phase overwrites saved, then each phase,
 * last to first, restores them and passes the adjoints of its outputs to its inputs
 * with the derivatives the forward mode uses (so the two agree to rounding).  Earlier
 * cycles' states come back from checkpoints of u, v, p, sc taken every ~sqrt(ncycles)
 * cycles and re-runs between them.  Afterwards u, v, p, sc and the histories are
 * those after ncycles cycles (other arrays unspecified).  Periodic boundaries are not
 * covered (MGFVM_EUNSUPPORTED).  A case that turns non-finite within the cycles (the
 * reference diverges on such inputs too) has no gradient; the others are unaffected.  Replaces no routine of the reference: the reference computes
 * no derivatives. */
int mgfvm_adjoint(mgfvm_ctx *ctx, int ncycles);

/* The last mgfvm_adjoint's result for case `icase`: J after the cycles and its
 * gradient (dJ_dinlet: nfy values, the inlet faces of mgfvm_set_inlet_profile).  Any
 * pointer may be NULL.  MGFVM_ENONFINITE (gradient set to NaN) for a case that turned
 * non-finite. */
int mgfvm_adjoint_gradient(mgfvm_ctx *ctx, int icase, double *J, double *dJ_dinlet, double *dJ_damuf,
                           double *dJ_dprsc);

/* Bytes this context copied host->device and device->host since it was created. */
int mgfvm_transfer_bytes(mgfvm_ctx *ctx, long long *h2d, long long *d2h);

/* Message of the last failed call on this thread ("" if none). */
const char *mgfvm_last_error(void);

/* ------------------------------------------------- pattern generators */
/* Seeded versions of the reference's interactive generators (which seed rand()
 * with time(NULL)).  Host only; no GPU needed.
 *
 * Staggered lattice of 1x1 base blocks on an (n_base*scale)^2 sub-pixel grid:
 * variant 1 inline, 2 staggered, >= 3 the (variant-2)-th random perturbation of the
 * staggered lattice.  Replaces create_patterns_staggered.c:71-200.  grid: dim^2 ints. */
int mgfvm_pattern_staggered(int n_base, int scale, int spacing_x, int spacing_y, int variant,
                            unsigned long long seed, int *grid);
/* Non-overlapping particles of side 3, 2, 1 at a target filled fraction; rects
 * (may be NULL) receives {r1, r2, c1, c2} 1-based per particle, the reference's
 * pattern-file rows.  Replaces create_patterns_random.c:18-181. */
int mgfvm_pattern_random(int n_grid, double ratio, double pct1, double pct2, double pct3,
                         unsigned long long seed, int *grid, int *rects, int max_rects,
                         int *n_rects);
/* One obstacle per occupied pixel {r+1, r+1, c+1, c+1} (create_patterns_staggered.c:47-54). */
int mgfvm_pattern_pixels(const int *grid, int dim, int *obs, int max_obs, int *count);

/* ------------------------------------------------------- output files */
/* The reference's output files, byte for byte.  Host only.
 * write_vtk_2d_cc (Version-6-26-04.c:2261-2363): legacy ASCII VTK of the level-0
 * interior (u, v, p, sc of npx*npy host arrays; obs_ranges = level-0 ranges from
 * mgfvm_get_obstacle_ranges), then the three diagnostic stdout lines; diag_out (may
 * be NULL) receives mean |velocity|, mean x-velocity and tortuosity. */
int mgfvm_write_vtk(const char *path, const mgfvm_config *cfg, int npx, int npy, const double *u,
                    const double *v, const double *p, const double *sc, const int *obs_ranges,
                    int iter, double diag_out[3]);
/* write_convergence_data_file (:2544-2558): rows 1..nconverged of the history, and a
 * stdout line reporting `nvcycle` records when verbose. */
int mgfvm_write_convergence(const char *path, const double *hist, int nconverged, int nvcycle,
                            int verbose);

/* ------------------------------------- raw-pointer kernel entry points */
/* These take caller-owned DEVICE pointers to one level laid out as above and
 * launch on `stream` (a cudaStream_t, NULL = legacy default stream).  They are
 * the drop-in replacements of the reference's per-level routines for callers
 * that keep their own level storage. */

/* Jacobi, `nsw` sweeps of phi <- (sum a_nb phi_nb + su) / (ap + 1e-30) over
 * i in [1, nx-1], j in [1, ny-1], ping-ponging through `scratch` (npx*npy doubles,
 * caller-owned); the result is left in phi.  Replaces solver(),
 * Version-6-26-04.c:1231-1296 (which mallocs its scratch on every call). */
int mgfvm_jacobi_f64(const double *aw, const double *ae, const double *as,
                     const double *an, const double *ap, const double *su,
                     double *phi, double *scratch, int npx, int npy, int nx, int ny,
                     int nsw, void *stream);

/* Red-black Gauss-Seidel, `nsw` sweeps of a red pass ((i+j) even) then a black
 * pass, in place, phi <- (sum a_nb phi_nb + su) / ap.  Replaces solvergs(),
 * Version-6-26-04.c:1297-1351. */
int mgfvm_rbgs_f64(const double *aw, const double *ae, const double *as,
                   const double *an, const double *ap, const double *su,
                   double *phi, int npx, int npy, int nx, int ny, int nsw,
                   void *stream);

/* Mass residual: su = -div, pp = 0 on the interior and *err_out (device) =
 * sum |div|, reduced in a fixed order through `partials` (caller-owned device
 * scratch of mgfvm_masserror_scratch_doubles(npx, npy) doubles).  Replaces
 * masserror(), Version-6-26-04.c:1096-1125. */
int mgfvm_masserror_f64(const double *u, const double *v, const double *areax,
                        const double *areay, double *su, double *pp, int npx,
                        int npy, double *err_out, double *partials, void *stream);
size_t mgfvm_masserror_scratch_doubles(int npx, int npy);

/* Self-test of the smoothers' division by a precomputed reciprocal (two Markstein
 * correction steps after RN(1/b), with the IEEE division outside its safe range):
 * n pseudo-random operand pairs from `seed` (half raw bit patterns, half values of
 * moderate exponent) are divided both ways on `device`; *mismatches counts results
 * whose bits differ from a / b.  No counterpart in the reference. */
int mgfvm_check_division(int device, long long n, unsigned long long seed, long long *mismatches);

/* mgfvm_masserror_f64 for callers that cannot allocate device memory (a host
 * program whose device memory another runtime owns, or a path that must not enter
 * the CUDA allocator).  No counterpart in the reference: its reduction scratch is a
 * fixed ~512 KiB array of static device memory inside this library, held by every
 * GPU that loads it until exit.  Levels with more than 1,048,576 interior cells
 * ((npx-2)*(npy-2)) are rejected with MGFVM_EINVAL.  Allocates nothing.  All calls
 * on a device share that array: calls that overlap on the GPU race.  The first call
 * on each device looks up the array's device address; make it before any stream
 * capture.  That address is cached per device for the life of the process and does
 * not survive a cudaDeviceReset of that device.  A non-null `stream` must belong to
 * the current device (MGFVM_EINVAL otherwise). */
int mgfvm_masserror_f64_noalloc(const double *u, const double *v, const double *areax,
                                const double *areay, double *su, double *pp, int npx,
                                int npy, double *err_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MGFVM_H */
