/*
 * config.c — InputData / pattern.txt parser and configuration checks.
 *
 * Reads the two input files with the same fscanf sequence as the reference
 * (readInput, Version-6-26-04.c:280-401; read_obstacle_data :2367-2400), including
 * its ordering quirk: pattern.txt is read after line 8 of InputData (:357).  The
 * echo lines printed when `verbose` is set are the reference's, byte for byte, so
 * the command-line tool's stdout matches the reference binary's.  Unlike the
 * reference, every failure returns a status and a message instead of exiting, and
 * the obstacle list is sized from the file instead of a fixed 1000 entries (:29).
 */
#include "mgfvm_host.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[512];

const char *mgfvm_last_error(void) { return g_err; }

int mgfvm_fail(int status, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return status;
}

void mgfvm_clear_error(void) { g_err[0] = 0; }

void mgfvm_config_default(mgfvm_config *c)
{
    memset(c, 0, sizeof *c);
    c->nfx = 64; c->nfy = 64; c->ngrid = 3;
    c->nvcycle = 2000; c->nswpm = 2; c->nswpp = 10; c->isolve = MGFVM_JACOBI;
    c->omega = 1.0; c->convergence = 1e-6;
    c->xl = 1.0; c->yl = 1.0; c->amuf = 0.01; c->prsc = 1.0; c->relxm = 0.7; c->relxp = 0.3;
    c->ibc_xm = 1; c->ibc_xp = 4; c->ibc_ym = 1; c->ibc_yp = 1;
    c->u_xm = 1.0; c->sc_xm = 1.0;
}

void mgfvm_options_default(mgfvm_options *o)
{
    memset(o, 0, sizeof *o);
    o->device = 0;
    o->precision = MGFVM_PREC_FP64;
    o->tail_level = -1;
    o->use_graph = 1;
    o->sync_every = 64;
}

void mgfvm_config_release(mgfvm_config *c)
{
    if (!c) return;
    free(c->obs);
    c->obs = NULL;
    c->nobs = 0;
}

/* read_obstacle_data, Version-6-26-04.c:2367-2400 */
static int read_pattern(const char *path, mgfvm_config *c, int verbose)
{
    FILE *f = fopen(path, "r");
    if (!f) return mgfvm_fail(MGFVM_EIO, "ERROR: Could not open file %s", path);
    int n = 0;
    if (fscanf(f, "%d", &n) != 1) {
        fclose(f);
        return mgfvm_fail(MGFVM_EINVAL, "ERROR: failed reading obstacle line of inputData");
    }
    if (verbose) printf("nobs %d \n", n);
    c->nobs = n > 0 ? n : 0;
    c->obs = NULL;
    if (n > 0) {
        c->obs = (int *)malloc(sizeof(int) * 4 * (size_t)n);
        if (!c->obs) { fclose(f); return mgfvm_fail(MGFVM_ENOMEM, "out of host memory for %d obstacles", n); }
        for (int k = 0; k < n; ++k) {
            int *r = &c->obs[4 * k];
            if (fscanf(f, " %d %d %d %d", &r[0], &r[1], &r[2], &r[3]) != 4) {
                fclose(f);
                free(c->obs); c->obs = NULL; c->nobs = 0;
                return mgfvm_fail(MGFVM_EINVAL, "ERROR: failed reading coordinates for obstacle %d", k);
            }
        }
    }
    fclose(f);
    return MGFVM_OK;
}

#define LINE_FAIL(which) do { fclose(f); mgfvm_config_release(c); \
    return mgfvm_fail(MGFVM_EINVAL, "ERROR: failed reading " which " of inputData"); } while (0)

int mgfvm_config_read(const char *input_path, const char *pattern_path, mgfvm_config *c,
                      int verbose)
{
    mgfvm_clear_error();
    mgfvm_config_default(c);
    c->ibc_xp = 1; c->u_xm = 0.0; c->sc_xm = 0.0;
    FILE *f = fopen(input_path, "r");
    if (!f) return mgfvm_fail(MGFVM_EIO, "ERROR opening inputData: %s", input_path);

    if (fscanf(f, "%d %d %d %d %d %d %d %d %d %d %d %lf %lf", &c->nfx, &c->nfy, &c->ngrid,
               &c->ig_obs, &c->ibeg_obs, &c->ig_inlt, &c->ig_outlt, &c->nvcycle, &c->nswpm,
               &c->nswpp, &c->isolve, &c->omega, &c->convergence) != 13)
        LINE_FAIL("first line");
    if (verbose)
        printf("nx_fine = %d, ny_fine = %d, ngrid = %d, nvcycle = %d, "
               "nswpm = %d, nswpp = %d, isolve = %d,omega = %lf, convergence = %e\n",
               c->nfx, c->nfy, c->ngrid, c->nvcycle, c->nswpm, c->nswpp, c->isolve, c->omega,
               c->convergence);

    if (fscanf(f, "%lf %lf %lf %lf %lf %lf", &c->xl, &c->yl, &c->amuf, &c->prsc, &c->relxm,
               &c->relxp) != 6)
        LINE_FAIL("second line");
    if (verbose)
        printf("xlength = %lf, ylength = %lf, viscosity = %lf, scalar Prandtl number = %lf, "
               "relax_momentum = %lf, relax_press = %lf\n",
               c->xl, c->yl, c->amuf, c->prsc, c->relxm, c->relxp);

    if (fscanf(f, "%d %d %d %d", &c->ibc_xm, &c->ibc_xp, &c->ibc_ym, &c->ibc_yp) != 4)
        LINE_FAIL("third line");
    if (verbose)
        printf("ibc_xm = %d, ibc_xp = %d, ibc_ym = %d, ibc_yp = %d\n", c->ibc_xm, c->ibc_xp,
               c->ibc_ym, c->ibc_yp);

    if (fscanf(f, "%lf %lf %lf %lf", &c->u_xm, &c->v_xm, &c->p_xm, &c->sc_xm) != 4)
        LINE_FAIL("fourth line");
    if (verbose)
        printf("u_xm = %lf, v_xm = %lf, p_xm = %lf, sc_xm = %lf\n", c->u_xm, c->v_xm, c->p_xm, c->sc_xm);
    if (fscanf(f, "%lf %lf %lf %lf", &c->u_xp, &c->v_xp, &c->p_xp, &c->sc_xp) != 4)
        LINE_FAIL("fifth line");
    if (verbose)
        printf("u_xp = %lf, v_xp = %lf, p_xp = %lf, sc_xp = %lf\n", c->u_xp, c->v_xp, c->p_xp, c->sc_xp);
    if (fscanf(f, "%lf %lf %lf %lf", &c->u_ym, &c->v_ym, &c->p_ym, &c->sc_ym) != 4)
        LINE_FAIL("sixth line");
    if (verbose)
        printf("u_ym = %lf, v_ym = %lf, p_ym = %lf, sc_ym = %lf\n", c->u_ym, c->v_ym, c->p_ym, c->sc_ym);
    if (fscanf(f, "%lf %lf %lf %lf", &c->u_yp, &c->v_yp, &c->p_yp, &c->sc_yp) != 4)
        LINE_FAIL("seventh line");
    if (verbose)
        printf("u_yp = %lf, v_yp = %lf, p_yp = %lf, sc_yp = %lf\n", c->u_yp, c->v_yp, c->p_yp, c->sc_yp);
    if (fscanf(f, "%lf %lf %lf %lf", &c->u_guess, &c->v_guess, &c->p_guess, &c->sc_guess) != 4)
        LINE_FAIL("eighth line");
    if (verbose)
        printf("u_guess = %lf, v_guess = %lf, p_guess = %lf, sc_guess = %lf\n", c->u_guess,
               c->v_guess, c->p_guess, c->sc_guess);

    int rc = read_pattern(pattern_path, c, verbose);
    if (rc) { fclose(f); return rc; }

    if (fscanf(f, "%lf", &c->sc_obs) != 1) LINE_FAIL("obstacle temperature line");
    if (verbose) printf("obs_sc %lf\n", c->sc_obs);

    if (fscanf(f, "%d", &c->ninlt) != 1) LINE_FAIL("inlet and outlet line");
    if (verbose) printf("ninlt %d\n", c->ninlt);
    if (c->ninlt > MGFVM_MAX_PORTS) {
        fclose(f); mgfvm_config_release(c);
        return mgfvm_fail(MGFVM_EINVAL, "ninlt = %d exceeds %d inlets", c->ninlt, MGFVM_MAX_PORTS);
    }
    for (int k = 0; k < c->ninlt; ++k)    /* unchecked in the reference (:373); checked here */
        if (fscanf(f, " %d %d %lf %lf %lf", &c->jfinlt[k], &c->jlinlt[k], &c->uinlt[k],
                   &c->vinlt[k], &c->scinlt[k]) != 5)
            LINE_FAIL("an inlet line");
    if (verbose)
        for (int k = 0; k < c->ninlt; ++k)
            printf(" jfinlt = %d, jlinlt = %d, uinlt = %lf, vinlt = %lf,tinlt = %lf\n",
                   c->jfinlt[k], c->jlinlt[k], c->uinlt[k], c->vinlt[k], c->scinlt[k]);

    if (fscanf(f, "%d", &c->noutlt) != 1) LINE_FAIL("inlet and outlet line");
    if (verbose) printf("noutlt %d \n", c->noutlt);
    if (c->noutlt > MGFVM_MAX_PORTS) {
        fclose(f); mgfvm_config_release(c);
        return mgfvm_fail(MGFVM_EINVAL, "noutlt = %d exceeds %d outlets", c->noutlt, MGFVM_MAX_PORTS);
    }
    for (int k = 0; k < c->noutlt; ++k)
        if (fscanf(f, " %d %d %lf %lf %lf", &c->jfoutlt[k], &c->jloutlt[k], &c->uoutlt[k],
                   &c->voutlt[k], &c->scoutlt[k]) != 5)
            LINE_FAIL("an outlet line");
    if (verbose)
        for (int k = 0; k < c->noutlt; ++k)
            printf(" jfoutlt = %d, jloutlt = %d, uoutlt = %lf, voutlt = %lf,scoutlt = %lf\n",
                   c->jfoutlt[k], c->jloutlt[k], c->uoutlt[k], c->voutlt[k], c->scoutlt[k]);
    fclose(f);
    return MGFVM_OK;
}

/* ---------------------------------------------------------------- checks */
static int pow2(int e) { return 1 << e; }

int mgfvm_config_validate(const mgfvm_config *c)
{
    if (c->ngrid < 1 || c->ngrid > 16)
        return mgfvm_fail(MGFVM_EINVAL, "ngrid = %d out of range [1, 16]", c->ngrid);
    if (c->nfx < 1 || c->nfy < 1)
        return mgfvm_fail(MGFVM_EINVAL, "grid %d x %d is empty", c->nfx, c->nfy);
    int f = pow2(c->ngrid - 1);
    if (c->nfx % f || c->nfy % f)
        return mgfvm_fail(MGFVM_EINVAL, "nfx = %d, nfy = %d not divisible by 2^(ngrid-1) = %d",
                          c->nfx, c->nfy, f);
    if (c->nfx / f < 2 || c->nfy / f < 2)
        return mgfvm_fail(MGFVM_EINVAL, "coarsest level %d x %d is smaller than 2 x 2",
                          c->nfx / f, c->nfy / f);
    if ((long long)(c->nfx + 2) * (c->nfy + 2) > (1LL << 31) / 2)
        return mgfvm_fail(MGFVM_EINVAL, "grid %d x %d too large", c->nfx, c->nfy);
    if (c->isolve != MGFVM_JACOBI && c->isolve != MGFVM_GAUSS_SEIDEL)
        return mgfvm_fail(MGFVM_EINVAL, "isolve = %d (1 Jacobi, 2 Gauss-Seidel)", c->isolve);
    if (c->nswpm < 0 || c->nswpp < 0)
        return mgfvm_fail(MGFVM_EINVAL, "negative sweep count");
    if (c->relxm == 0.0 || c->prsc == 0.0)
        return mgfvm_fail(MGFVM_EINVAL, "relxm and prsc must be nonzero");
    int b[4] = {c->ibc_xm, c->ibc_xp, c->ibc_ym, c->ibc_yp};
    for (int k = 0; k < 4; ++k)
        if (b[k] < 0 || b[k] > 4)
            return mgfvm_fail(MGFVM_EINVAL, "boundary code %d unknown", b[k]);
    if (c->nobs > 0 && (c->ig_obs < 0 || c->ig_obs > c->ngrid))
        return mgfvm_fail(MGFVM_EINVAL, "ig_obs = %d outside [0, ngrid = %d]", c->ig_obs, c->ngrid);
    if (c->ninlt > 0 && (c->ig_inlt < 0 || c->ig_inlt > c->ngrid))
        return mgfvm_fail(MGFVM_EINVAL, "ig_inlt = %d outside [0, ngrid]", c->ig_inlt);
    if (c->noutlt > 0 && (c->ig_outlt < 0 || c->ig_outlt > c->ngrid))
        return mgfvm_fail(MGFVM_EINVAL, "ig_outlt = %d outside [0, ngrid]", c->ig_outlt);
    if (c->ninlt < 0 || c->ninlt > MGFVM_MAX_PORTS || c->noutlt < 0 || c->noutlt > MGFVM_MAX_PORTS)
        return mgfvm_fail(MGFVM_EINVAL, "ninlt/noutlt outside [0, %d]", MGFVM_MAX_PORTS);
    if (c->nobs > 0 && !c->obs)
        return mgfvm_fail(MGFVM_EINVAL, "nobs = %d but no obstacle list", c->nobs);

    /* Every index the level routines touch must stay inside the padded grid. */
    for (int ig = 0; ig < c->ngrid; ++ig) {
        int npx = c->nfx / pow2(ig) + 2, npy = c->nfy / pow2(ig) + 2;
        if (ig < c->ig_obs)
            for (int k = 0; k < c->nobs; ++k) {
                int r[4];
                mgfvm_obstacle_range(c, k, ig, r);
                /* update's row copies run whenever is <= ie and its column copies
                 * whenever js <= je, even if the other range is empty (:1153-1176);
                 * init and coefsc need both ranges. */
                int rows = r[0] <= r[1], cols = r[2] <= r[3];
                int in_i0 = r[0] >= 1 && r[0] <= npx - 2, in_i1 = r[1] >= 1 && r[1] <= npx - 2;
                int in_j0 = r[2] >= 1 && r[2] <= npy - 2, in_j1 = r[3] >= 1 && r[3] <= npy - 2;
                int ok_r = !rows || (in_i0 && in_i1 && in_j0 && in_j1);
                int ok_c = !cols || (in_i0 && in_i1 && in_j0 && in_j1);
                if (!ok_r || !ok_c)
                    return mgfvm_fail(MGFVM_EOOB,
                                      "obstacle %d maps to i %d..%d, j %d..%d on level %d, outside "
                                      "the interior 1..%d x 1..%d",
                                      k, r[0], r[1], r[2], r[3], ig, npx - 2, npy - 2);
            }
        for (int k = 0; k < c->ninlt && ig < c->ig_inlt; ++k) {
            int fac = pow2(c->ig_inlt - 1 - ig);
            int js = (c->jfinlt[k] - 1) * fac + 1, je = c->jlinlt[k] * fac;
            if (js <= je && (js < 0 || je > npy - 1))
                return mgfvm_fail(MGFVM_EOOB, "inlet %d rows %d..%d outside level %d", k, js, je, ig);
        }
        for (int k = 0; k < c->noutlt && ig < c->ig_outlt; ++k) {
            int fac = pow2(c->ig_outlt - 1 - ig);
            int js = (c->jfoutlt[k] - 1) * fac + 1, je = c->jloutlt[k] * fac;
            if (js <= je && (js < 0 || je > npy - 1))
                return mgfvm_fail(MGFVM_EOOB, "outlet %d rows %d..%d outside level %d", k, js, je, ig);
        }
    }
    return MGFVM_OK;
}

/* Obstacle k on level ig: the mapping of AllocateMemorySoA :468-478 for ig < ig_obs,
 * the empty range {1, 0, 1, 0} above (the reference leaves those uninitialised). */
void mgfvm_obstacle_range(const mgfvm_config *c, int k, int ig, int r[4])
{
    if (ig < c->ig_obs) {
        int fac = pow2(c->ig_obs - 1 - ig);
        const int *o = &c->obs[4 * k];
        r[0] = (o[0] + c->ibeg_obs - 1) * fac + 1;
        r[1] = (o[1] + c->ibeg_obs) * fac;
        r[2] = (o[2] - 1) * fac + 1;
        r[3] = o[3] * fac;
    } else {
        r[0] = 1; r[1] = 0; r[2] = 1; r[3] = 0;
    }
}
