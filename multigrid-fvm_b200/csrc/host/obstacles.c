/*
 * obstacles.c — the two sequential obstacle loops of the reference, turned into
 * data the GPU can apply in parallel with the same result bit for bit.
 *
 * 1. update()'s pressure copy (Version-6-26-04.c:1153-1177).  For every obstacle in
 *    list order the reference copies into its bottom row from the row below, its
 *    top row from the row above, its left column from the left and its right column
 *    from the right; later copies overwrite earlier ones and may read cells earlier
 *    copies wrote.  Replaying the copies on cell labels gives, for every written
 *    cell, the cell whose pre-copy value it ends up holding; the GPU then does
 *    p[dst] = p_before[src].  If some source is itself a destination the gather
 *    must read all sources before writing (flag `hazard`).
 *
 * 2. coefsc()'s obstacle-face diffusion (:939-963).  Every obstacle cell adds a
 *    diffusion term to the east coefficient of its west neighbour, the west
 *    coefficient of its east neighbour, the north coefficient of its south
 *    neighbour and the south coefficient of its north neighbour, and each time the
 *    same term to that neighbour's ap.  FP addition is order-dependent, so for every
 *    receiving cell the additions are recorded in loop order as 2-bit codes
 *    (0: from the east cell into ae, 1: from the west cell into aw, 2: from the
 *    north cell into an, 3: from the south cell into as), up to 14 per cell, count
 *    in the top 4 bits.  Cells on the boundary ring are dropped: no routine reads
 *    their coefficients.
 */
#include "mgfvm_host.h"

#include <stdlib.h>
#include <string.h>

#define SEQ_MAX 14

static int cmp_pair(const void *a, const void *b)
{
    const int *x = (const int *)a, *y = (const int *)b;
    return (x[0] > y[0]) - (x[0] < y[0]);
}

int mgfvm_build_obstacle_prog(const mgfvm_config *c, int ig, mgfvm_obstacle_prog *out)
{
    memset(out, 0, sizeof *out);
    if (c->nobs <= 0 || ig >= c->ig_obs) return MGFVM_OK;
    int nx = c->nfx / (1 << ig) + 2, ny = c->nfy / (1 << ig) + 2;
    size_t n = (size_t)nx * ny;
    int *origin = (int *)malloc(sizeof(int) * n);
    unsigned char *written = (unsigned char *)calloc(n, 1);
    unsigned *seq = (unsigned *)calloc(n, sizeof(unsigned));
    if (!origin || !written || !seq) {
        free(origin); free(written); free(seq);
        return mgfvm_fail(MGFVM_ENOMEM, "obstacle program: out of host memory");
    }
    for (size_t q = 0; q < n; ++q) origin[q] = (int)q;

    int overflow = 0;
    for (int k = 0; k < c->nobs; ++k) {
        int r[4];
        mgfvm_obstacle_range(c, k, ig, r);
        int is = r[0], ie = r[1], js = r[2], je = r[3];
        /* pressure copies, in the reference's order */
        for (int i = is; i <= ie; ++i) { int d = js * nx + i; origin[d] = origin[d - nx]; written[d] = 1; }
        for (int i = is; i <= ie; ++i) { int d = je * nx + i; origin[d] = origin[d + nx]; written[d] = 1; }
        for (int j = js; j <= je; ++j) { int d = j * nx + is; origin[d] = origin[d - 1]; written[d] = 1; }
        for (int j = js; j <= je; ++j) { int d = j * nx + ie; origin[d] = origin[d + 1]; written[d] = 1; }
        /* diffusion additions, i outer and j inner as in :941-962 */
        for (int i = is; i <= ie; ++i)
            for (int j = js; j <= je; ++j) {
                int q = j * nx + i;
                const int recv[4] = {q - 1, q + 1, q - nx, q + nx};
                for (int t = 0; t < 4; ++t) {
                    int x = recv[t], xi = x % nx, xj = x / nx;
                    if (xi < 1 || xi > nx - 2 || xj < 1 || xj > ny - 2) continue;
                    unsigned cnt = seq[x] >> 28;
                    if (cnt >= SEQ_MAX) { overflow = 1; continue; }
                    seq[x] = (seq[x] & 0x0FFFFFFFu) | ((unsigned)t << (2 * cnt)) | ((cnt + 1) << 28);
                }
            }
    }
    if (overflow) {
        free(origin); free(written); free(seq);
        return mgfvm_fail(MGFVM_EUNSUPPORTED,
                          "level %d: a cell receives more than %d obstacle-face additions "
                          "(overlapping obstacles)", ig, SEQ_MAX);
    }
    int ncopy = 0, nseq = 0, maxa = 0;
    for (size_t q = 0; q < n; ++q) {
        if (written[q] && origin[q] != (int)q) ++ncopy;
        if (seq[q]) { ++nseq; int a = (int)(seq[q] >> 28); if (a > maxa) maxa = a; }
    }
    int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(ncopy ? ncopy : 1));
    out->dst = (int *)malloc(sizeof(int) * (size_t)(ncopy ? ncopy : 1));
    out->src = (int *)malloc(sizeof(int) * (size_t)(ncopy ? ncopy : 1));
    out->cells = (int *)malloc(sizeof(int) * (size_t)(nseq ? nseq : 1));
    out->codes = (unsigned *)malloc(sizeof(unsigned) * (size_t)(nseq ? nseq : 1));
    if (!pairs || !out->dst || !out->src || !out->cells || !out->codes) {
        free(pairs); free(origin); free(written); free(seq);
        mgfvm_free_obstacle_prog(out);
        return mgfvm_fail(MGFVM_ENOMEM, "obstacle program: out of host memory");
    }
    int m = 0;
    for (size_t q = 0; q < n; ++q)
        if (written[q] && origin[q] != (int)q) { pairs[2 * m] = (int)q; pairs[2 * m + 1] = origin[q]; ++m; }
    qsort(pairs, (size_t)m, 2 * sizeof(int), cmp_pair);
    int hazard = 0, outlet = 0;
    for (int k = 0; k < m; ++k) {
        out->dst[k] = pairs[2 * k];
        out->src[k] = pairs[2 * k + 1];
        int s = out->src[k];
        if (written[s] && origin[s] != s) hazard = 1;
        if (out->dst[k] % nx >= nx - 2 || s % nx >= nx - 2) outlet = 1;
    }
    out->touches_outlet = outlet;
    out->ncopy = m;
    out->hazard = hazard;
    if (!hazard && m > 0) {
        /* group the copies by owner: the source when interior, else the interior cell
         * next to it (sources are at most one cell outside an interior obstacle) */
        int *tri = (int *)malloc(sizeof(int) * 3 * (size_t)m);
        out->owners = (int *)malloc(sizeof(int) * (size_t)m);
        out->fan = (int *)malloc(sizeof(int) * 2 * (size_t)m);
        if (!tri || !out->owners || !out->fan) {
            free(tri); free(pairs); free(origin); free(written); free(seq);
            mgfvm_free_obstacle_prog(out);
            return mgfvm_fail(MGFVM_ENOMEM, "obstacle program: out of host memory");
        }
        for (int k = 0; k < m; ++k) {
            const int s0 = out->src[k], si = s0 % nx, sj = s0 / nx;
            const int oi = si < 1 ? 1 : (si > nx - 2 ? nx - 2 : si);
            const int oj = sj < 1 ? 1 : (sj > ny - 2 ? ny - 2 : sj);
            tri[3 * k] = oj * nx + oi;
            tri[3 * k + 1] = out->dst[k];
            tri[3 * k + 2] = (oi == si && oj == sj) ? -1 : s0;
        }
        qsort(tri, (size_t)m, 3 * sizeof(int), cmp_pair);   /* by owner */
        for (int k = 0; k < m; ++k) {
            out->owners[k] = tri[3 * k];
            const int last = k == m - 1 || tri[3 * (k + 1)] != tri[3 * k];
            out->fan[2 * k] = tri[3 * k + 1] | (last ? PFAN_LAST : 0);
            out->fan[2 * k + 1] = tri[3 * k + 2];
        }
        free(tri);
    }
    m = 0;
    for (size_t q = 0; q < n; ++q)
        if (seq[q]) { out->cells[m] = (int)q; out->codes[m] = seq[q]; ++m; }
    out->nseq = m;
    out->max_adds = maxa;
    free(pairs); free(origin); free(written); free(seq);
    return MGFVM_OK;
}

void mgfvm_free_obstacle_prog(mgfvm_obstacle_prog *p)
{
    if (!p) return;
    free(p->dst); free(p->src); free(p->cells); free(p->codes); free(p->owners); free(p->fan);
    memset(p, 0, sizeof *p);
}
