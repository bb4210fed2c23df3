/*
 * mgfvm_patterns.c — seeded, non-interactive counterpart of the reference's obstacle
 * pattern generators (create_patterns_staggered.c:71-200, create_patterns_random.c:
 * 18-181).  Those programs prompt for their parameters and seed rand() with time(NULL),
 * so their patterns cannot be reproduced; this tool takes the same parameters as
 * arguments plus a seed and writes the same files in the same layout:
 *
 *   mgfvm_patterns staggered N_BASE SHIFT SX SY COUNT [SEED]
 *       SHIFT: 1 quarter, 2 half, 3 full pixel (the reference's menu).  Directory
 *       n<N_BASE>_por_<porosity %.1f>_sx<SX>_sy<SY>_scale<S>x with pattern_1 (inline
 *       lattice), pattern_2 (staggered) and pattern_3 ... pattern_<COUNT+2> (random
 *       one-step moves of every block).
 *   mgfvm_patterns random N RATIO COUNT PCT1 PCT2 PCT3 [SEED]
 *       Directory n_<N>/p_<RATIO %.2f> with pattern_1 ... pattern_<COUNT>: non-
 *       overlapping particles of side 1, 2 and 3 in the given percentages.
 *
 * Each pattern is written as <name>.txt (obstacle count, then `r1 r2 c1 c2` per
 * obstacle: the pattern.txt format the solver reads) and <name>.pgm (P2 image, 0 for
 * solid, 255 for open).
 */
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "mgfvm.h"

static int mkdirs(const char *path)
{
    char buf[1024];
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

static int write_files(const char *dir, const char *name, const int *grid, int dim, const int *rects, int nrects)
{
    char path[1400];
    snprintf(path, sizeof path, "%s/%s.txt", dir, name);
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    fprintf(f, "%d\n", nrects);
    for (int k = 0; k < nrects; ++k)
        fprintf(f, "%d %d %d %d\n", rects[4 * k], rects[4 * k + 1], rects[4 * k + 2], rects[4 * k + 3]);
    fclose(f);
    snprintf(path, sizeof path, "%s/%s.pgm", dir, name);
    f = fopen(path, "w");
    if (!f) return -1;
    fprintf(f, "P2\n%d %d\n255\n", dim, dim);
    for (int r = 0; r < dim; ++r) {
        for (int c = 0; c < dim; ++c) fprintf(f, "%d ", grid[r * dim + c] == 1 ? 0 : 255);
        fprintf(f, "\n");
    }
    fclose(f);
    return 0;
}

static int usage(const char *argv0)
{
    fprintf(stderr,
            "usage: %s staggered N_BASE SHIFT(1 quarter|2 half|3 full) SX SY COUNT [SEED]\n"
            "       %s random N RATIO COUNT PCT1 PCT2 PCT3 [SEED]\n",
            argv0, argv0);
    return 2;
}

int main(int argc, char **argv)
{
    if (argc < 2) return usage(argv[0]);
    if (!strcmp(argv[1], "staggered")) {
        if (argc < 7) return usage(argv[0]);
        const int n_base = atoi(argv[2]), shift = atoi(argv[3]), sx = atoi(argv[4]), sy = atoi(argv[5]);
        const int count = atoi(argv[6]);
        const unsigned long long seed = argc > 7 ? strtoull(argv[7], NULL, 10) : 1ull;
        const int scale = shift == 1 ? 4 : shift == 2 ? 2 : shift == 3 ? 1 : 0;
        if (!scale || n_base < 1 || sx < 0 || sy < 0 || count < 0) return usage(argv[0]);
        const double porosity = 100.0 * (1.0 - 1.0 / ((1.0 + sx) * (1.0 + sy)));
        char dir[256];
        snprintf(dir, sizeof dir, "n%d_por_%.1f_sx%d_sy%d_scale%dx", n_base, porosity, sx, sy, scale);
        if (mkdirs(dir)) { fprintf(stderr, "cannot create %s\n", dir); return 1; }
        const int dim = n_base * scale;
        int *grid = (int *)malloc(sizeof(int) * (size_t)dim * dim);
        int *rects = (int *)malloc(sizeof(int) * 4 * (size_t)dim * dim);
        for (int v = 1; v <= count + 2; ++v) {
            int n = 0;
            if (mgfvm_pattern_staggered(n_base, scale, sx, sy, v, seed, grid) ||
                mgfvm_pattern_pixels(grid, dim, rects, dim * dim, &n)) {
                fprintf(stderr, "%s\n", mgfvm_last_error());
                return 1;
            }
            char name[32];
            snprintf(name, sizeof name, "pattern_%d", v);
            if (write_files(dir, name, grid, dim, rects, n)) { fprintf(stderr, "cannot write %s/%s\n", dir, name); return 1; }
        }
        printf("Done! Calculated Porosity: %.2f%%\nGenerated output in directory: '%s'\n", porosity, dir);
        free(grid);
        free(rects);
        return 0;
    }
    if (!strcmp(argv[1], "random")) {
        if (argc < 8) return usage(argv[0]);
        const int n = atoi(argv[2]), count = atoi(argv[4]);
        const double ratio = atof(argv[3]), p1 = atof(argv[5]), p2 = atof(argv[6]), p3 = atof(argv[7]);
        const unsigned long long seed = argc > 8 ? strtoull(argv[8], NULL, 10) : 1ull;
        if (n < 7 || count < 0) return usage(argv[0]);
        char dir[256];
        snprintf(dir, sizeof dir, "n_%d/p_%.2f", n, ratio);
        if (mkdirs(dir)) { fprintf(stderr, "cannot create %s\n", dir); return 1; }
        printf("Saving outputs to folder: %s\n", dir);
        int *grid = (int *)malloc(sizeof(int) * (size_t)n * n);
        int *rects = (int *)malloc(sizeof(int) * 4 * (size_t)n * n);
        for (int p = 0; p < count; ++p) {
            int nr = 0;
            /* pattern p draws from its own stream: seed + p */
            if (mgfvm_pattern_random(n, ratio, p1, p2, p3, seed + (unsigned long long)p, grid, rects, n * n, &nr)) {
                fprintf(stderr, "%s\n", mgfvm_last_error());
                return 1;
            }
            char name[32];
            snprintf(name, sizeof name, "pattern_%d", p + 1);
            if (write_files(dir, name, grid, n, rects, nr)) { fprintf(stderr, "cannot write %s/%s\n", dir, name); return 1; }
        }
        free(grid);
        free(rects);
        return 0;
    }
    return usage(argv[0]);
}
