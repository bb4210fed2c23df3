/*
 * patterns.c — seeded obstacle-pattern generators.
 *
 * The reference ships two interactive generators seeded with time(NULL)
 * (create_patterns_staggered.c, create_patterns_random.c), so their patterns cannot
 * be reproduced.  These are the same constructions driven by an explicit seed:
 *   - staggered: a square lattice of 1x1 base blocks on a sub-pixel grid
 *     (scale 4 / 2 / 1 for quarter / half / full pixel shifts), then every odd
 *     column shifted by half a lattice step (create_patterns_staggered.c:133-164),
 *     then each block moved one sub-pixel up, down, left or right, or left in
 *     place, with probability 1/5 each (:166-185);
 *   - random: non-overlapping square particles of side 3, then 2, then 1, placed
 *     uniformly at random until a target filled fraction (create_patterns_random.c:62-138).
 * The random draws come from splitmix64 (Steele, Lea & Flood, OOPSLA 2014) instead of
 * libc rand(); `seed` fully determines every pattern.
 */
#include "mgfvm_host.h"

#include <stdlib.h>
#include <string.h>

typedef struct { unsigned long long s; } rng_t;

static unsigned long long rng_next(rng_t *r)
{
    unsigned long long z = (r->s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static int rng_below(rng_t *r, int n) { return (int)(rng_next(r) % (unsigned long long)n); }

typedef struct { int r1, r2, c1, c2; } rect_t;

static void render(const rect_t *o, int n, int *grid, int dim)
{
    memset(grid, 0, sizeof(int) * (size_t)dim * dim);
    for (int k = 0; k < n; ++k)
        for (int r = o[k].r1; r <= o[k].r2; ++r)
            for (int c = o[k].c1; c <= o[k].c2; ++c)
                if (r >= 0 && r < dim && c >= 0 && c < dim) grid[r * dim + c] = 1;
}

int mgfvm_pattern_staggered(int n_base, int scale, int spacing_x, int spacing_y, int variant,
                            unsigned long long seed, int *grid)
{
    if (n_base < 1 || (scale != 1 && scale != 2 && scale != 4) || spacing_x < 0 ||
        spacing_y < 0 || variant < 1 || !grid)
        return mgfvm_fail(MGFVM_EINVAL, "staggered pattern: bad arguments");
    int dim = n_base * scale, obj = scale;
    int sx = spacing_x * scale, sy = spacing_y * scale, pad = 5 * scale;
    int step_x = obj + sx, step_y = obj + sy, npad = dim + 2 * pad;
    int half = obj / 2;
    int cap = (npad / step_x + 3) * (npad / step_y + 3);
    rect_t *o = (rect_t *)malloc(sizeof(rect_t) * (size_t)cap);
    rect_t *w = (rect_t *)malloc(sizeof(rect_t) * (size_t)cap);
    if (!o || !w) { free(o); free(w); return mgfvm_fail(MGFVM_ENOMEM, "staggered pattern: out of memory"); }
    int n = 0;
    for (int r = -half; r <= npad; r += step_y)            /* inline lattice */
        for (int c = -half; c <= npad; c += step_x) {
            o[n].r1 = r - pad; o[n].r2 = r + obj - 1 - pad;
            o[n].c1 = c - pad; o[n].c2 = c + obj - 1 - pad;
            ++n;
        }
    if (variant >= 2)                                        /* staggered: odd columns shift */
        for (int k = 0; k < n; ++k) {
            int col = (o[k].c1 + pad + half) / step_x;
            if (col % 2 == 1) { o[k].r1 += step_y / 2; o[k].r2 += step_y / 2; }
        }
    rng_t g = {seed};
    const rect_t *use = o;
    for (int v = 3; v <= variant; ++v) {                     /* perturbed draws, in order */
        memcpy(w, o, sizeof(rect_t) * (size_t)n);
        for (int k = 0; k < n; ++k) {
            int move = rng_below(&g, 5);
            int dr = move == 1 ? -1 : move == 2 ? 1 : 0;
            int dc = move == 3 ? -1 : move == 4 ? 1 : 0;
            w[k].r1 += dr; w[k].r2 += dr; w[k].c1 += dc; w[k].c2 += dc;
        }
        use = w;
    }
    render(use, n, grid, dim);
    free(o); free(w);
    return MGFVM_OK;
}

int mgfvm_pattern_random(int n_grid, double ratio, double pct1, double pct2, double pct3,
                         unsigned long long seed, int *grid, int *rects, int max_rects,
                         int *n_rects)
{
    if (n_grid < 7 || ratio < 0 || !grid || !n_rects)
        return mgfvm_fail(MGFVM_EINVAL, "random pattern: bad arguments");
    double s = pct1 + pct2 + pct3;
    if (s > 100.1 || s < 99.9) return mgfvm_fail(MGFVM_EINVAL, "random pattern: percentages must sum to 100");
    double p1 = pct1 / 100.0, p2 = pct2 / 100.0, p3 = pct3 / 100.0;
    double target = (double)n_grid * n_grid * ratio;
    double per = p1 * 1.0 + p2 * 4.0 + p3 * 9.0;
    int total = (int)(target / per + 0.5);
    int counts[3] = {(int)(total * p3 + 0.5), (int)(total * p2 + 0.5), (int)(total * p1 + 0.5)};
    const int sizes[3] = {3, 2, 1};
    rng_t g = {seed};
    memset(grid, 0, sizeof(int) * (size_t)n_grid * n_grid);
    int n = 0;
    for (int t = 0; t < 3; ++t) {
        int sz = sizes[t];
        for (int k = 0; k < counts[t]; ++k)
            for (int tries = 0; tries < 10000; ++tries) {
                int r = rng_below(&g, n_grid - sz + 1), c = rng_below(&g, n_grid - sz + 1);
                int clash = 0;
                for (int a = 0; a < sz && !clash; ++a)
                    for (int b = 0; b < sz; ++b)
                        if (grid[(r + a) * n_grid + c + b]) { clash = 1; break; }
                if (clash) continue;
                for (int a = 0; a < sz; ++a)
                    for (int b = 0; b < sz; ++b) grid[(r + a) * n_grid + c + b] = 1;
                if (rects && n < max_rects) {
                    rects[4 * n] = r + 1; rects[4 * n + 1] = r + sz;
                    rects[4 * n + 2] = c + 1; rects[4 * n + 3] = c + sz;
                }
                ++n;
                break;
            }
    }
    *n_rects = n;
    return MGFVM_OK;
}

/* One obstacle per occupied pixel, row-major, as `r+1 r+1 c+1 c+1` — the line
 * format of the staggered generator's pattern files (create_patterns_staggered.c:47-54). */
int mgfvm_pattern_pixels(const int *grid, int dim, int *obs, int max_obs, int *count)
{
    int n = 0;
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c)
            if (grid[r * dim + c]) {
                if (obs && n < max_obs) {
                    obs[4 * n] = r + 1; obs[4 * n + 1] = r + 1;
                    obs[4 * n + 2] = c + 1; obs[4 * n + 3] = c + 1;
                }
                ++n;
            }
    *count = n;
    return MGFVM_OK;
}
