/*
 * ref_harness.c — TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * Builds the unmodified reference solver Version-6-26-04.c into a shared library
 * (oracle/_ref/libmgref.so) so parity tests and the CPU baseline can drive its
 * routines one by one.  The reference source is textually included from where it
 * lies; REF_SRC is set by oracle/Makefile.  Three macros wrap it without changing
 * any arithmetic:
 *   main   -> ref_main    so this file can provide the entry points below;
 *   printf -> ref_printf  which drops the per-cycle echo unless ref_verbose(1);
 *   exit   -> ref_exit    which longjmps back to the harness entry point, so a
 *                         parse error returns a status instead of ending the caller.
 *
 * Deviations from running the raw binary, all outside the reference's own code:
 *   1. levels ig >= ig_obs get the empty obstacle range {1,0,1,0}.  The reference
 *      leaves them uninitialised (:471 fills ig < ig_obs only) yet coefsc (:939) and
 *      update (:1153) loop over them on every level.  With ig_obs == ngrid this is a
 *      no-op.
 *   2. convergence_data[3000] (:39) is indexed modulo 3000 so long runs stay in
 *      bounds; the harness keeps its own unbounded history.
 *   3. an optional per-face inlet profile is written into level-0 u[j*npx+0] after
 *      init() and before rest_geom(), mirroring mgfvm_set_inlet_profile.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdarg.h>
#include <string.h>
#include <setjmp.h>
#include <unistd.h>
#include <math.h>
#include <time.h>

static int ref_verbose_flag = 0;
static jmp_buf ref_jmp;
static int ref_jmp_armed = 0;

static int ref_printf(const char *fmt, ...)
{
    if (!ref_verbose_flag) return 0;
    va_list ap;
    va_start(ap, fmt);
    int r = vprintf(fmt, ap);
    va_end(ap);
    return r;
}

static void ref_exit(int code)
{
    if (ref_jmp_armed) longjmp(ref_jmp, code == 0 ? 1 : code);
    exit(code);
}

#define printf ref_printf
#define exit(code) ref_exit(code)
#define main ref_main
#include REF_SRC
#undef main
#undef exit
#undef printf

/* ------------------------------------------------------------------ state */
static struct SoA *R = NULL;       /* the level array of the loaded case */
static double *hist_err = NULL;    /* per-cycle level-0 sum|div|         */
static int hist_cap = 0, hist_n = 0;

enum { F_U = 0, F_V, F_P, F_PP, F_SC, F_SU, F_RS, F_RESU, F_RESV, F_RESSC, F_C,
       F_AW, F_AE, F_AS, F_AN, F_AP, F_APU, F_APV, F_SPU, F_SPV, F_SPSC,
       F_CX, F_CY, F_AREAX, F_AREAY, NF };

static double *field_ptr(struct SoA *s, int f)
{
    switch (f) {
    case F_U: return s->u;      case F_V: return s->v;      case F_P: return s->p;
    case F_PP: return s->pp;    case F_SC: return s->sc;    case F_SU: return s->su;
    case F_RS: return s->rs;    case F_RESU: return s->resu; case F_RESV: return s->resv;
    case F_RESSC: return s->ressc; case F_C: return s->c;
    case F_AW: return s->aw;    case F_AE: return s->ae;    case F_AS: return s->as;
    case F_AN: return s->an;    case F_AP: return s->ap;    case F_APU: return s->apu;
    case F_APV: return s->apv;  case F_SPU: return s->spu;  case F_SPV: return s->spv;
    case F_SPSC: return s->spsc; case F_CX: return s->cx;   case F_CY: return s->cy;
    case F_AREAX: return s->areax; case F_AREAY: return s->areay;
    }
    return NULL;
}

void ref_verbose(int on) { ref_verbose_flag = on; }

void ref_free(void)
{
    if (R) {
        for (int ig = 0; ig < ngrid; ++ig) {
            free(R[ig].spsc); free(R[ig].tag);
            free(R[ig].isobs); free(R[ig].ieobs); free(R[ig].jsobs); free(R[ig].jeobs);
            free(R[ig].jsinlt); free(R[ig].jeinlt); free(R[ig].jsoutlt); free(R[ig].jeoutlt);
        }
        FreeMemorySoA(R);
        R = NULL;
    }
    free(hist_err); hist_err = NULL; hist_cap = hist_n = 0;
}

/* Load InputData + pattern.txt from directory `dir` (the reference reads them from
 * the working directory, :282, :357).  Returns 0 on success, else the code the
 * reference passed to exit(). */
int ref_load(const char *dir, const double *inlet_u, int n_inlet)
{
    ref_free();
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return -1;
    if (chdir(dir) != 0) return -2;
    int rc = setjmp(ref_jmp);
    if (rc != 0) {
        ref_jmp_armed = 0;
        if (chdir(cwd) != 0) return -3;
        R = NULL;
        return rc;
    }
    ref_jmp_armed = 1;
    memset(convergence_data, 0, sizeof convergence_data);
    readInput();
    ref_jmp_armed = 0;
    if (chdir(cwd) != 0) return -3;

    R = AllocateMemorySoA();
    for (int ig = ig_obs < 0 ? 0 : ig_obs; ig < ngrid; ++ig)
        for (int k = 0; k < nobs; ++k) {
            R[ig].isobs[k] = 1; R[ig].ieobs[k] = 0;
            R[ig].jsobs[k] = 1; R[ig].jeobs[k] = 0;
        }
    init(R);
    if (inlet_u && n_inlet > 0) {
        int npx = R[0].npx;
        for (int j = 1; j <= n_inlet && j < R[0].npy - 1; ++j)
            R[0].u[j * npx + 0] = inlet_u[j - 1];
    }
    rest_geom(R);
    nvcycle_converged = 0;
    return 0;
}

int ref_ngrid(void) { return R ? ngrid : 0; }
int ref_npx(int ig) { return R ? R[ig].npx : 0; }
int ref_npy(int ig) { return R ? R[ig].npy : 0; }
int ref_nobs(void) { return nobs; }

int ref_get(int ig, int f, double *out)
{
    if (!R || ig < 0 || ig >= ngrid || f < 0 || f >= NF) return -1;
    memcpy(out, field_ptr(&R[ig], f), sizeof(double) * R[ig].npx * R[ig].npy);
    return 0;
}

int ref_set(int ig, int f, const double *in)
{
    if (!R || ig < 0 || ig >= ngrid || f < 0 || f >= NF) return -1;
    memcpy(field_ptr(&R[ig], f), in, sizeof(double) * R[ig].npx * R[ig].npy);
    return 0;
}

int ref_get_tag(int ig, int *out)
{
    if (!R || ig < 0 || ig >= ngrid) return -1;
    memcpy(out, R[ig].tag, sizeof(int) * R[ig].npx * R[ig].npy);
    return 0;
}

int ref_get_obstacle_ranges(int ig, int *out)
{
    if (!R || ig < 0 || ig >= ngrid) return -1;
    for (int k = 0; k < nobs; ++k) {
        out[4 * k + 0] = R[ig].isobs[k]; out[4 * k + 1] = R[ig].ieobs[k];
        out[4 * k + 2] = R[ig].jsobs[k]; out[4 * k + 3] = R[ig].jeobs[k];
    }
    return 0;
}

/* The globals readInput filled, for checking the product's InputData parser:
 * ints {nfx,nfy,ngrid,ig_obs,ibeg_obs,ig_inlt,ig_outlt,nvcycle,nswpm,nswpp,isolve,
 *       ibc_xm,ibc_xp,ibc_ym,ibc_yp,nobs,ninlt,noutlt}
 * dbls {omega,convergence,xl,yl,amuf,prsc,relxm,relxp, u/v/p/sc _xm,_xp,_ym,_yp,
 *       u/v/p/sc _guess, sc_obs} */
void ref_get_config(int *iv, double *dv, int *obs, int *ports_i, double *ports_d)
{
    int ii[] = {nfx, nfy, ngrid, ig_obs, ibeg_obs, ig_inlt, ig_outlt, nvcycle, nswpm,
                nswpp, isolve, ibc_xm, ibc_xp, ibc_ym, ibc_yp, nobs, ninlt, noutlt};
    memcpy(iv, ii, sizeof ii);
    double dd[] = {omega, convergence, xl, yl, amuf, prsc, relxm, relxp,
                   u_xm, v_xm, p_xm, sc_xm, u_xp, v_xp, p_xp, sc_xp,
                   u_ym, v_ym, p_ym, sc_ym, u_yp, v_yp, p_yp, sc_yp,
                   u_guess, v_guess, p_guess, sc_guess, sc_obs};
    memcpy(dv, dd, sizeof dd);
    for (int k = 0; k < nobs; ++k) {
        obs[4 * k] = ifobs[k]; obs[4 * k + 1] = ilobs[k];
        obs[4 * k + 2] = jfobs[k]; obs[4 * k + 3] = jlobs[k];
    }
    for (int k = 0; k < 10; ++k) {
        ports_i[4 * k] = jfinlt[k]; ports_i[4 * k + 1] = jlinlt[k];
        ports_i[4 * k + 2] = jfoutlt[k]; ports_i[4 * k + 3] = jloutlt[k];
        ports_d[6 * k] = uinlt[k]; ports_d[6 * k + 1] = vinlt[k]; ports_d[6 * k + 2] = scinlt[k];
        ports_d[6 * k + 3] = uoutlt[k]; ports_d[6 * k + 4] = voutlt[k]; ports_d[6 * k + 5] = scoutlt[k];
    }
}

static void hist_push(double e)
{
    if (hist_n == hist_cap) {
        hist_cap = hist_cap ? 2 * hist_cap : 1024;
        hist_err = (double *)realloc(hist_err, sizeof(double) * hist_cap);
    }
    hist_err[hist_n++] = e;
}

/* One V-cycle, the body of the loop at Version-6-26-04.c:195-249. */
void ref_cycle(int icyc)
{
    int slot = icyc % 3000;
    for (int ig = 0; ig < ngrid; ++ig) {
        struct SoA *a = &R[ig];
        fluxes(a);
        solve_u(a);
        solve_v(a);
        solve_pprime(a, slot, ig);
        pbound(a);
        outflow(a);
        solve_sc(a);
        if (ig != ngrid - 1) {
            struct SoA *b = &R[ig + 1];
            restv(a, b);
            fluxes(b);
            fluxes(a);
            restru(a, b);
            restrv(a, b);
            restrsc(a, b);
        }
    }
    for (int ig = ngrid - 1; ig > 0; ig--) {
        struct SoA *b = &R[ig], *a = &R[ig - 1];
        prolu(a, b);
        prolv(a, b);
        prolp(a, b);
        prolsc(a, b);
        if (ig != 1) {
            fluxes(a);
            solve_u(a);
            solve_v(a);
            solve_pprime(a, slot, ig);
            pbound(a);
            solve_sc(a);
            outflow(a);
        }
    }
    nvcycle_converged = icyc;
    hist_push(convergence_data[slot]);
}

int ref_history(double *out, int cap)
{
    int n = hist_n < cap ? hist_n : cap;
    if (out) memcpy(out, hist_err, sizeof(double) * n);
    return hist_n;
}

/* Single reference routines on level ig, numbered as enum mgfvm_op.  `leg` selects
 * the solve_pprime ig argument (0 = down leg at level ig, else the up-leg value). */
int ref_op(int op, int ig, int icyc_slot)
{
    if (!R || ig < 0 || ig >= ngrid) return -1;
    struct SoA *a = &R[ig];
    switch (op) {
    case 0: fluxes(a); break;
    case 1: solve_u(a); break;
    case 2: solve_v(a); break;
    case 3: solve_pprime(a, icyc_slot % 3000, ig); break;
    case 4: pbound(a); break;
    case 5: outflow(a); break;
    case 6: solve_sc(a); break;
    case 7: {
        if (ig + 1 >= ngrid) return -1;
        struct SoA *b = &R[ig + 1];
        restv(a, b); fluxes(b); fluxes(a); restru(a, b); restrv(a, b); restrsc(a, b);
        break;
    }
    case 8: {
        if (ig + 1 >= ngrid) return -1;
        struct SoA *b = &R[ig + 1];
        prolu(a, b); prolv(a, b); prolp(a, b); prolsc(a, b);
        break;
    }
    case 9:  if (isolve == 1) solver(a, a->u, a->npx - 2, a->npy - 1);
             else solvergs(a, a->u, a->npx - 2, a->npy - 1); break;
    case 10: if (isolve == 1) solver(a, a->v, a->npx - 1, a->npy - 2);
             else solvergs(a, a->v, a->npx - 1, a->npy - 2); break;
    case 11: if (isolve == 1) solver(a, a->pp, a->npx - 1, a->npy - 1);
             else solvergs(a, a->pp, a->npx - 1, a->npy - 1); break;
    case 12: if (isolve == 1) solver(a, a->sc, a->npx - 1, a->npy - 1);
             else solvergs(a, a->sc, a->npx - 1, a->npy - 1); break;
    default: return -1;
    }
    return 0;
}

double ref_last_err(int icyc) { return convergence_data[icyc % 3000]; }

/* Time `ncyc` V-cycles of the loaded case on this thread (CPU seconds of wall clock). */
double ref_time_cycles(int first_cycle, int ncyc)
{
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int c = 0; c < ncyc; ++c) ref_cycle(first_cycle + c);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    return (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
}
