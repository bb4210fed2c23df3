/*
 * mgfvm_sweep.c — batch driver replacing run_patterns_and_save_vtk.sh:13-78.
 *
 * The reference sweeps obstacle patterns and Reynolds numbers with a shell loop that
 * runs its solver once per (Re, pattern): for every Re it rewrites the viscosity on
 * InputData line 2 (column 3, 1/Re from `bc` with scale=6, i.e. truncated to six
 * decimals, :23-27), then for every patterns/pattern_<n>.txt it copies the pattern
 * to pattern.txt, runs the solver and moves convergence.csv and vtk_acc.vtk to
 * solution/Re_<Re>/convergence_files/convergence_<n>.csv and
 * solution/Re_<Re>/vtk_files/vtk_<n>.vtk (:36-76).
 *
 * This driver builds every (Re, pattern) case from ./InputData and the pattern
 * files, solves them together in one context on the GPU (chunks of --chunk cases),
 * each with the reference's stop rule, and writes the same files into the same
 * layout; a file is written under the same condition as the reference program writes
 * it (:264-268).  Usage:
 *
 *   mgfvm_sweep [--re 20,50,...] [--patterns DIR] [--out DIR] [--chunk N]
 *               [--mixed] [--autotune] [--device D]
 *
 * Without --re the viscosity of ./InputData is used as is (one sweep, labelled with
 * the Re it implies).  Line 1 of InputData is used as given.
 */
#include <dirent.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "mgfvm.h"
#include "mgfvm_host.h"

typedef struct {
    char re_label[64];
    char number[256];
    mgfvm_config cfg;
} sweep_case;

static int mkdirs(const char *path)
{
    char buf[4096];
    snprintf(buf, sizeof buf, "%s", path);
    for (char *p = buf + 1; *p; ++p)
        if (*p == '/') {
            *p = 0;
            if (mkdir(buf, 0755) && errno != EEXIST) return -1;
            *p = '/';
        }
    if (mkdir(buf, 0755) && errno != EEXIST) return -1;
    return 0;
}

static int cmp_str(const void *a, const void *b) { return strcmp(*(char *const *)a, *(char *const *)b); }

/* pattern_<n>.txt files of `dir`, sorted by name (the shell glob's order) */
static char **list_patterns(const char *dir, int *count)
{
    DIR *d = opendir(dir);
    *count = 0;
    if (!d) return NULL;
    char **names = NULL;
    int cap = 0;
    struct dirent *e;
    while ((e = readdir(d))) {
        const size_t n = strlen(e->d_name);
        if (strncmp(e->d_name, "pattern_", 8) || n < 13 || strcmp(e->d_name + n - 4, ".txt")) continue;
        if (*count == cap) {
            cap = cap ? 2 * cap : 64;
            names = (char **)realloc(names, sizeof(char *) * cap);
        }
        names[(*count)++] = strdup(e->d_name);
    }
    closedir(d);
    if (*count) qsort(names, (size_t)*count, sizeof(char *), cmp_str);
    return names;
}

/* 1/Re as `echo "scale=6; 1 / Re" | bc` gives it: truncated to six decimals */
static double inv_re_bc(double re) { return floor(1.0e6 / re) / 1.0e6; }

static int solve_chunk(sweep_case *cs, int n, const char *out, const mgfvm_options *opt, int autotune)
{
    mgfvm_config *cfgs = (mgfvm_config *)malloc(sizeof(mgfvm_config) * (size_t)n);
    int nvmax = 0;
    for (int k = 0; k < n; ++k) {
        cfgs[k] = cs[k].cfg;
        if (cfgs[k].nvcycle > nvmax) nvmax = cfgs[k].nvcycle;
    }
    mgfvm_ctx *ctx = NULL;
    int rc = mgfvm_create(cfgs, n, opt, &ctx);
    free(cfgs);
    if (rc) return rc;
    if (autotune) {
        double before = 0, after = 0;
        rc = mgfvm_autotune(ctx, 3, NULL, &before, &after);
        if (rc) { mgfvm_destroy(ctx); return rc; }
        printf("  autotuned launch shapes: %.3f -> %.3f ms per V-cycle\n", before, after);
    }
    int *ran = (int *)calloc((size_t)n, sizeof(int));
    rc = mgfvm_solve(ctx, nvmax, 0.0, ran);
    if (rc && rc != MGFVM_ENONFINITE) { free(ran); mgfvm_destroy(ctx); return rc; }
    double ms = 0;
    mgfvm_last_elapsed_ms(ctx, &ms);
    printf("  %d cases solved together in %.3f s on the GPU\n", n, ms / 1e3);
    for (int k = 0; k < n; ++k) {
        const mgfvm_config *c = &cs[k].cfg;
        int npx = 0, npy = 0, nh = 0;
        mgfvm_level_dims(ctx, k, 0, &npx, &npy);
        const size_t m = (size_t)npx * npy;
        double *hist = (double *)calloc((size_t)(ran[k] > 0 ? ran[k] : 1), sizeof(double));
        double *u = (double *)malloc(m * sizeof(double)), *v = (double *)malloc(m * sizeof(double));
        double *p = (double *)malloc(m * sizeof(double)), *sc = (double *)malloc(m * sizeof(double));
        int *rng = (int *)malloc(sizeof(int) * 4 * (size_t)(c->nobs > 0 ? c->nobs : 1));
        mgfvm_history(ctx, k, hist, NULL, ran[k], &nh);
        mgfvm_get_field(ctx, k, 0, MGFVM_F_U, u);
        mgfvm_get_field(ctx, k, 0, MGFVM_F_V, v);
        mgfvm_get_field(ctx, k, 0, MGFVM_F_P, p);
        mgfvm_get_field(ctx, k, 0, MGFVM_F_SC, sc);
        mgfvm_get_obstacle_ranges(ctx, k, 0, rng);
        const int last = ran[k] > 0 ? ran[k] - 1 : 0;
        const int converged = ran[k] > 0 && hist[last] < c->convergence;
        printf("  -> pattern_%s.txt, Re = %s: %d V-cycles, mass error %e\n", cs[k].number, cs[k].re_label, ran[k],
               ran[k] > 0 ? hist[last] : 0.0);
        /* the reference writes its files when the entry it tests (:264-268) is below
         * `convergence`; after a loop that ran out that entry is 0.0 */
        if ((converged ? hist[last] : 0.0) < c->convergence) {
            char dv[4096], dc[4096], fv[4352], fc[4352];
            snprintf(dv, sizeof dv, "%s/Re_%s/vtk_files", out, cs[k].re_label);
            snprintf(dc, sizeof dc, "%s/Re_%s/convergence_files", out, cs[k].re_label);
            if (mkdirs(dv) || mkdirs(dc)) {
                fprintf(stderr, "cannot create %s or %s\n", dv, dc);
                rc = MGFVM_EIO;
            } else {
                snprintf(fv, sizeof fv, "%s/vtk_%s.vtk", dv, cs[k].number);
                snprintf(fc, sizeof fc, "%s/convergence_%s.csv", dc, cs[k].number);
                int r1 = mgfvm_write_vtk(fv, c, npx, npy, u, v, p, sc, rng, 0, NULL);
                int r2 = mgfvm_write_convergence(fc, hist, last, c->nvcycle, 0);
                if (r1 || r2) rc = r1 ? r1 : r2;
            }
        } else {
            printf("  [Error] no output for pattern_%s.txt (the reference writes none in this case)\n", cs[k].number);
        }
        free(hist); free(u); free(v); free(p); free(sc); free(rng);
    }
    free(ran);
    mgfvm_destroy(ctx);
    return rc;
}

int main(int argc, char **argv)
{
    const char *pdir = "patterns", *out = "solution", *re_list = NULL;
    int chunk = 256, autotune = 0;
    mgfvm_options opt;
    mgfvm_options_default(&opt);
    opt.sync_every = 64;
    for (int k = 1; k < argc; ++k) {
        if (!strcmp(argv[k], "--re") && k + 1 < argc) re_list = argv[++k];
        else if (!strcmp(argv[k], "--patterns") && k + 1 < argc) pdir = argv[++k];
        else if (!strcmp(argv[k], "--out") && k + 1 < argc) out = argv[++k];
        else if (!strcmp(argv[k], "--chunk") && k + 1 < argc) chunk = atoi(argv[++k]);
        else if (!strcmp(argv[k], "--mixed")) opt.precision = MGFVM_PREC_MIXED;
        else if (!strcmp(argv[k], "--autotune")) autotune = 1;
        else if (!strcmp(argv[k], "--device") && k + 1 < argc) opt.device = atoi(argv[++k]);
        else {
            fprintf(stderr, "usage: %s [--re R1,R2,...] [--patterns DIR] [--out DIR] [--chunk N] [--mixed] "
                            "[--autotune] [--device D]\n", argv[0]);
            return 2;
        }
    }
    if (chunk < 1) chunk = 1;
    int npat = 0;
    char **pats = list_patterns(pdir, &npat);
    if (!npat) {
        fprintf(stderr, "no %s/pattern_*.txt files\n", pdir);
        return 1;
    }
    /* Reynolds numbers: the --re list, or the one InputData implies */
    char res[64][64];
    int nre = 0;
    if (re_list) {
        char buf[4096];
        snprintf(buf, sizeof buf, "%s", re_list);
        for (char *t = strtok(buf, ","); t && nre < 64; t = strtok(NULL, ",")) snprintf(res[nre++], 64, "%s", t);
    }
    int rc = 0, total = nre ? nre * npat : npat;
    sweep_case *cs = (sweep_case *)calloc((size_t)(chunk < total ? chunk : total), sizeof(sweep_case));
    int filled = 0, done = 0;
    for (int r = 0; r < (nre ? nre : 1) && !rc; ++r) {
        for (int k = 0; k < npat && !rc; ++k) {
            sweep_case *s = &cs[filled];
            char path[4352];
            snprintf(path, sizeof path, "%s/%s", pdir, pats[k]);
            rc = mgfvm_config_read("InputData", path, &s->cfg, 0);
            if (rc) break;
            if (nre) {
                const double re = atof(res[r]);
                if (!(re > 0)) {
                    fprintf(stderr, "bad Reynolds number %s\n", res[r]);
                    rc = MGFVM_EINVAL;
                    break;
                }
                s->cfg.amuf = inv_re_bc(re);
                snprintf(s->re_label, sizeof s->re_label, "%s", res[r]);
            } else {
                snprintf(s->re_label, sizeof s->re_label, "%g", 1.0 / s->cfg.amuf);
            }
            const size_t L = strlen(pats[k]);
            snprintf(s->number, sizeof s->number, "%.*s", (int)(L - 12), pats[k] + 8);
            if (++filled == chunk || done + filled == total) {
                printf("Solving %d case(s) (%d of %d)\n", filled, done + filled, total);
                rc = solve_chunk(cs, filled, out, &opt, autotune);
                for (int q = 0; q < filled; ++q) mgfvm_config_release(&cs[q].cfg);
                done += filled;
                filled = 0;
            }
        }
    }
    for (int q = 0; q < filled; ++q) mgfvm_config_release(&cs[q].cfg);
    for (int k = 0; k < npat; ++k) free(pats[k]);
    free(pats);
    free(cs);
    if (rc) {
        fprintf(stderr, "%s\n", mgfvm_last_error());
        return 1;
    }
    printf("All processing completed successfully.\n");
    return 0;
}
