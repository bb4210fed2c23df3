/*
 * mgfvm_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU parity checker of the CUDA
 * engine.  Never linked into the product library.
 *
 * A sequential restatement of one case of the reference solver, routine by routine,
 * in the reference's own loop order, so that every floating-point operation happens
 * in the same order as in Version-6-26-04.c compiled with gcc (no FMA contraction).
 * Each routine cites the reference lines it restates.  Where the reference's
 * behaviour is undefined, the oracle takes the rule the engine documents:
 *   - levels at or above ig_obs hold the empty obstacle range {1,0,1,0} (the
 *     reference leaves them uninitialised, :471, yet reads them at :939, :1153);
 *   - the mass-error history is unbounded (the reference keeps 3000 entries, :39).
 */
#include "mgfvm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int npx, npy;
    double dx, dy, amu;
    double *a[MGFVM_NFIELDS];
    int *tag;
    int *rng;          /* 4*nobs: is, ie, js, je */
    int *inl, *outl;   /* 2*ninlt / 2*noutlt: js, je */
} lvl_t;

struct orc_case {
    mgfvm_config cfg;
    int *obs;          /* owned copy of cfg.obs */
    int ng;
    lvl_t *L;
    double last_err;
    double *err, *delta;
    int nh, caph;
    double *prev[4];   /* level-0 u, v, p, sc after the previous cycle */
    int have_prev;
};

#define A(l, f) ((l)->a[MGFVM_F_##f])

static int ipow2(int e) { return 1 << e; }

/* ------------------------------------------------------------ allocation */
/* AllocateMemorySoA, Version-6-26-04.c:402-506: level sizes, spacing, and the
 * obstacle / inlet / outlet index mapping from level ig_* - 1 to finer levels. */
static int alloc_levels(orc_case *c)
{
    const mgfvm_config *g = &c->cfg;
    c->ng = g->ngrid;
    c->L = (lvl_t *)calloc((size_t)c->ng, sizeof(lvl_t));
    if (!c->L) return MGFVM_ENOMEM;
    for (int ig = 0; ig < c->ng; ++ig) {
        lvl_t *l = &c->L[ig];
        int fac = ipow2(ig);
        l->npx = g->nfx / fac + 2;
        l->npy = g->nfy / fac + 2;
        l->dx = g->xl / (l->npx - 2);
        l->dy = g->yl / (l->npy - 2);
        l->amu = g->amuf;
        size_t n = (size_t)l->npx * l->npy;
        for (int f = 0; f < MGFVM_NFIELDS; ++f) {
            l->a[f] = (double *)calloc(n, sizeof(double));
            if (!l->a[f]) return MGFVM_ENOMEM;
        }
        l->tag = (int *)calloc(n, sizeof(int));
        l->rng = (int *)calloc((size_t)(g->nobs > 0 ? g->nobs : 1) * 4, sizeof(int));
        l->inl = (int *)calloc(2 * MGFVM_MAX_PORTS, sizeof(int));
        l->outl = (int *)calloc(2 * MGFVM_MAX_PORTS, sizeof(int));
        if (!l->tag || !l->rng || !l->inl || !l->outl) return MGFVM_ENOMEM;
        for (int k = 0; k < g->nobs; ++k) {
            int *r = &l->rng[4 * k];
            if (ig < g->ig_obs) {            /* :470-476 */
                int f2 = ipow2(g->ig_obs - 1 - ig);
                r[0] = (c->obs[4 * k + 0] + g->ibeg_obs - 1) * f2 + 1;
                r[1] = (c->obs[4 * k + 1] + g->ibeg_obs) * f2;
                r[2] = (c->obs[4 * k + 2] - 1) * f2 + 1;
                r[3] = c->obs[4 * k + 3] * f2;
            } else {                          /* empty range on uninitialised levels */
                r[0] = 1; r[1] = 0; r[2] = 1; r[3] = 0;
            }
        }
        for (int k = 0; k < g->ninlt; ++k)   /* :481-489 */
            if (ig < g->ig_inlt) {
                int f2 = ipow2(g->ig_inlt - 1 - ig);
                l->inl[2 * k] = (g->jfinlt[k] - 1) * f2 + 1;
                l->inl[2 * k + 1] = g->jlinlt[k] * f2;
            }
        for (int k = 0; k < g->noutlt; ++k)  /* :492-501 */
            if (ig < g->ig_outlt) {
                int f2 = ipow2(g->ig_outlt - 1 - ig);
                l->outl[2 * k] = (g->jfoutlt[k] - 1) * f2 + 1;
                l->outl[2 * k + 1] = g->jloutlt[k] * f2;
            }
    }
    return MGFVM_OK;
}

/* ------------------------------------------------------------------ init */
/* init, Version-6-26-04.c:546-676. */
static void init_levels(orc_case *c)
{
    const mgfvm_config *g = &c->cfg;
    for (int ig = 0; ig < c->ng; ++ig) {          /* defaults :549-578 */
        lvl_t *l = &c->L[ig];
        int n = l->npx * l->npy;
        for (int k = 0; k < n; ++k) {
            A(l, U)[k] = g->u_guess;  A(l, V)[k] = g->v_guess;
            A(l, SC)[k] = g->sc_guess; A(l, P)[k] = g->p_guess;
            A(l, PP)[k] = 0.0; A(l, SU)[k] = 0.0; A(l, C)[k] = 0.0; A(l, AP)[k] = 0.0;
            A(l, RESU)[k] = 0.0; A(l, RESV)[k] = 0.0; A(l, RESSC)[k] = 0.0; A(l, RS)[k] = 0.0;
            l->tag[k] = 1;
            A(l, APU)[k] = 1.0e30; A(l, APV)[k] = 1.0e30;
            A(l, SPU)[k] = 0.0; A(l, SPV)[k] = 0.0; A(l, SPSC)[k] = 0.0;
            A(l, AREAX)[k] = l->dy; A(l, AREAY)[k] = l->dx;
            A(l, CX)[k] = 0.0; A(l, CY)[k] = 0.0;
        }
    }
    for (int ig = 0; ig < c->ng; ++ig) {          /* boundary values :581-612 */
        lvl_t *l = &c->L[ig];
        int nx = l->npx, ny = l->npy;
        for (int j = 0; j < ny; ++j) {
            int k = j * nx;
            A(l, U)[k] = g->u_xm; A(l, V)[k] = g->v_xm; A(l, P)[k] = g->p_xm; A(l, SC)[k] = g->sc_xm;
        }
        for (int j = 0; j < ny; ++j) {
            int k = j * nx + nx - 1;
            A(l, U)[k - 1] = g->u_xp; A(l, V)[k] = g->v_xp; A(l, P)[k] = g->p_xp; A(l, SC)[k] = g->sc_xp;
        }
        for (int i = 0; i < nx; ++i) {
            A(l, U)[i] = g->u_ym; A(l, V)[i] = g->v_ym; A(l, P)[i] = g->p_ym; A(l, SC)[i] = g->sc_ym;
        }
        for (int i = 0; i < nx; ++i) {
            int k = (ny - 1) * nx + i;
            A(l, U)[k] = g->u_yp; A(l, V)[k] = g->v_yp; A(l, P)[k] = g->p_yp; A(l, SC)[k] = g->sc_yp;
        }
    }
    if (g->nobs > 0)                              /* obstacles :616-641 */
        for (int ig = 0; ig < g->ig_obs && ig < c->ng; ++ig) {
            lvl_t *l = &c->L[ig];
            int nx = l->npx;
            for (int k = 0; k < g->nobs; ++k) {
                const int *r = &l->rng[4 * k];
                for (int j = r[2]; j <= r[3]; ++j)
                    for (int i = r[0]; i <= r[1]; ++i) {
                        int q = j * nx + i;
                        A(l, U)[q] = 0.0; A(l, V)[q] = 0.0;
                        A(l, U)[q - 1] = 0.0; A(l, V)[q - nx] = 0.0;
                        A(l, SPU)[q] = 1.0e30; A(l, SPV)[q] = 1.0e30;
                        A(l, SPU)[q - 1] = 1.0e30; A(l, SPV)[q - nx] = 1.0e30;
                        A(l, SPSC)[q] = 1.0e30;
                        l->tag[q] = 0;
                        A(l, SC)[q] = g->sc_obs;
                    }
            }
        }
    if (g->ninlt > 0)                             /* inlets :645-658 */
        for (int ig = 0; ig < g->ig_inlt && ig < c->ng; ++ig) {
            lvl_t *l = &c->L[ig];
            for (int k = 0; k < g->ninlt; ++k)
                for (int j = l->inl[2 * k]; j <= l->inl[2 * k + 1]; ++j) {
                    int q = j * l->npx;
                    A(l, U)[q] = g->uinlt[k]; A(l, V)[q] = g->vinlt[k]; A(l, SC)[q] = g->scinlt[k];
                }
        }
    if (g->noutlt > 0)                            /* outlets :661-674 */
        for (int ig = 0; ig < g->ig_outlt && ig < c->ng; ++ig) {
            lvl_t *l = &c->L[ig];
            for (int k = 0; k < g->noutlt; ++k)
                for (int j = l->outl[2 * k]; j <= l->outl[2 * k + 1]; ++j) {
                    int q = j * l->npx + l->npx - 2;
                    A(l, U)[q] = g->uoutlt[k]; A(l, V)[q] = g->voutlt[k]; A(l, SC)[q + 1] = g->scoutlt[k];
                }
        }
}

/* rest_geom, Version-6-26-04.c:1391-1473: coarse face areas, then coarse x-
 * boundary u, v as averages of the two fine faces (left column, then right). */
static void rest_geom(orc_case *c)
{
    for (int ig = 1; ig < c->ng; ++ig) {
        lvl_t *f = &c->L[ig - 1], *k = &c->L[ig];
        int nxf = f->npx, nxc = k->npx, nyc = k->npy;
        for (int jc = 1; jc < nyc - 1; ++jc)
            for (int ic = 0; ic < nxc - 1; ++ic) {
                int q = 2 * jc * nxf + 2 * ic;
                A(k, AREAX)[jc * nxc + ic] = A(f, AREAX)[q] + A(f, AREAX)[q - nxf];
            }
        for (int jc = 0; jc < nyc - 1; ++jc)
            for (int ic = 1; ic < nxc - 1; ++ic) {
                int q = 2 * jc * nxf + 2 * ic;
                A(k, AREAY)[jc * nxc + ic] = A(f, AREAY)[q] + A(f, AREAY)[q - 1];
            }
    }
    for (int ig = 1; ig < c->ng; ++ig) {
        lvl_t *f = &c->L[ig - 1], *k = &c->L[ig];
        int nxf = f->npx, nxc = k->npx, nyc = k->npy;
        for (int jc = 1; jc < nyc - 1; ++jc) {
            int q = 2 * jc * nxf;
            A(k, U)[jc * nxc] = 0.5 * (A(f, U)[q] + A(f, U)[q - nxf]);
            A(k, V)[jc * nxc] = 0.5 * (A(f, V)[q] + A(f, V)[q - 1]);
        }
    }
    for (int ig = 1; ig < c->ng; ++ig) {
        lvl_t *f = &c->L[ig - 1], *k = &c->L[ig];
        int nxf = f->npx, nxc = k->npx, nyc = k->npy;
        for (int jc = 1; jc < nyc - 1; ++jc) {
            int q = 2 * jc * nxf + 2 * (nxc - 2);
            A(k, U)[jc * nxc + nxc - 2] = 0.5 * (A(f, U)[q] + A(f, U)[q - nxf]);
            A(k, V)[jc * nxc + nxc - 2] = 0.5 * (A(f, V)[q] + A(f, V)[q - 1]);
        }
    }
}

/* ------------------------------------------------------ SIMPLE routines */
/* fluxes :678-694 */
static void fluxes(lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    for (int j = 0; j < ny - 1; ++j)
        for (int i = 0; i < nx - 1; ++i) {
            int q = j * nx + i;
            A(l, CX)[q] = 0.5 * A(l, U)[q] * A(l, AREAX)[q];
            A(l, CY)[q] = 0.5 * A(l, V)[q] * A(l, AREAY)[q];
        }
}

/* hybrid upwind/central neighbour coefficient: max(|c|, D) + c (Version-6-26-04.c:845-848) */
static inline double hyb(double c, double d, int sign) { return sign > 0 ? fmax(fabs(c), d) + c : fmax(fabs(c), d) - c; }

/* coefu :815-860 */
static void coefu(lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double *cx = A(l, CX), *cy = A(l, CY);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int q = j * nx + i, s = q - nx;
            double cxm = 0.5 * (cx[q] + cx[q - 1]);
            double cxp = 0.5 * (cx[q] + cx[q + 1]);
            double cym = 0.5 * (cy[s] + cy[s + 1]);
            double cyp = 0.5 * (cy[q] + cy[q + 1]);
            double dxm = l->amu * (A(l, AREAX)[q] / l->dx);
            double dym = l->amu * (A(l, AREAY)[q] / l->dy);
            A(l, AW)[q] = hyb(cxm, dxm, +1);
            A(l, AE)[q] = hyb(cxp, dxm, -1);
            A(l, AS)[q] = hyb(cym, dym, +1);
            A(l, AN)[q] = hyb(cyp, dym, -1);
            A(l, AP)[q] = A(l, AW)[q] + A(l, AE)[q] + A(l, AS)[q] + A(l, AN)[q];
        }
    for (int i = 1; i < nx - 2; ++i) {          /* wall shear :849-858 */
        int top = (ny - 2) * nx + i, bot = nx + i;
        double add = l->amu * (A(l, AREAY)[top] / l->dy);
        A(l, AN)[top] += add; A(l, AP)[top] += add;
        A(l, AS)[bot] += add; A(l, AP)[bot] += add;
    }
}

/* coefv :966-1016 */
static void coefv(lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double *cx = A(l, CX), *cy = A(l, CY);
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i, n = q + nx, s = q - nx;
            double cxm = 0.5 * (cx[q - 1] + cx[n - 1]);
            double cxp = 0.5 * (cx[q] + cx[n]);
            double cym = 0.5 * (cy[q] + cy[s]);
            double cyp = 0.5 * (cy[q] + cy[n]);
            double dx_ = l->amu * (A(l, AREAX)[q] / l->dx);
            double dy_ = l->amu * (A(l, AREAY)[q] / l->dy);
            A(l, AW)[q] = hyb(cxm, dx_, +1);
            A(l, AE)[q] = hyb(cxp, dx_, -1);
            A(l, AS)[q] = hyb(cym, dy_, +1);
            A(l, AN)[q] = hyb(cyp, dy_, -1);
            A(l, AP)[q] = A(l, AW)[q] + A(l, AE)[q] + A(l, AS)[q] + A(l, AN)[q];
        }
    for (int j = 1; j < ny - 2; ++j) {          /* side-wall shear :1005-1015 */
        int rgt = j * nx + (nx - 2), lft = j * nx + 1;
        double add = l->amu * (A(l, AREAY)[rgt] / l->dy);
        A(l, AE)[rgt] += add; A(l, AP)[rgt] += add;
        A(l, AW)[lft] += add; A(l, AP)[lft] += add;
    }
}

/* coefsc :861-964, including the host-side obstacle-face diffusion loop :939-963 */
static void coefsc(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double amusc = c->cfg.amuf / c->cfg.prsc;
    double *cx = A(l, CX), *cy = A(l, CY), *ax = A(l, AREAX), *ay = A(l, AREAY);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i, s = q - nx;
            double dxm = amusc * (ax[q - 1] / l->dx);
            double dym = amusc * (ay[s] / l->dy);
            double dxp = amusc * (ax[q] / l->dx);
            double dyp = amusc * (ay[q] / l->dy);
            A(l, AW)[q] = hyb(cx[q - 1], dxm, +1);
            A(l, AE)[q] = hyb(cx[q], dxp, -1);
            A(l, AS)[q] = hyb(cy[s], dym, +1);
            A(l, AN)[q] = hyb(cy[q], dyp, -1);
            A(l, AP)[q] = A(l, AW)[q] + A(l, AE)[q] + A(l, AS)[q] + A(l, AN)[q];
        }
    for (int k = 0; k < c->cfg.nobs; ++k) {
        const int *r = &l->rng[4 * k];
        for (int i = r[0]; i <= r[1]; ++i)
            for (int j = r[2]; j <= r[3]; ++j) {
                int q = j * nx + i;
                double add = amusc * (ax[q] / l->dx);
                A(l, AE)[q - 1] += add; A(l, AP)[q - 1] += add;
                A(l, AW)[q + 1] += add; A(l, AP)[q + 1] += add;
                add = amusc * (ay[q] / l->dy);
                A(l, AN)[q - nx] += add; A(l, AP)[q - nx] += add;
                A(l, AS)[q + nx] += add; A(l, AP)[q + nx] += add;
            }
    }
}

/* umom :741-767 */
static void umom(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double rm = c->cfg.relxm, rm1 = 1.0 - rm;
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int q = j * nx + i;
            double s = A(l, AREAX)[q] * (A(l, P)[q] - A(l, P)[q + 1]);
            double ap = A(l, AP)[q] / rm;
            s = s + rm1 * ap * A(l, U)[q] + A(l, RESU)[q]
                + c->cfg.dpdxm * A(l, AREAX)[q] * A(l, AREAY)[q];
            A(l, SU)[q] = s;
            ap = ap + A(l, SPU)[q];
            A(l, AP)[q] = ap;
            A(l, APU)[q] = ap;
        }
}

/* vmom :769-793 */
static void vmom(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double rm = c->cfg.relxm, rm1 = 1.0 - rm;
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i;
            double s = A(l, AREAY)[q] * (A(l, P)[q] - A(l, P)[q + nx]);
            double ap = A(l, AP)[q] / rm;
            s = s + rm1 * ap * A(l, V)[q] + A(l, RESV)[q]
                + c->cfg.dpdym * A(l, AREAX)[q] * A(l, AREAY)[q];
            A(l, SU)[q] = s;
            ap = ap + A(l, SPV)[q];
            A(l, AP)[q] = ap;
            A(l, APV)[q] = ap;
        }
}

/* scalar :795-812 */
static void scalar_src(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i;
            A(l, SU)[q] = A(l, SPSC)[q] * c->cfg.sc_obs + A(l, RESSC)[q];
            A(l, AP)[q] = A(l, AP)[q] + A(l, SPSC)[q];
        }
}

/* masserror :1096-1125 (sum in the reference's row-major order) */
static double masserror(lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double err = 0.0;
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i;
            double ax = A(l, AREAX)[q], ay = A(l, AREAY)[q];
            double div = ax * A(l, U)[q] - ax * A(l, U)[q - 1] + ay * A(l, V)[q] - ay * A(l, V)[q - nx];
            A(l, SU)[q] = -div;
            A(l, PP)[q] = 0.0;
            err += fabs(div);
        }
    return err;
}

/* coefp :1018-1092 */
static void coefp(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double *ax = A(l, AREAX), *ay = A(l, AREAY);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i, s = q - nx;
            A(l, AW)[q] = ax[q - 1] * ax[q - 1] / A(l, APU)[q - 1];
            A(l, AE)[q] = ax[q] * ax[q] / A(l, APU)[q];
            A(l, AS)[q] = ay[s] * ay[s] / A(l, APV)[s];
            A(l, AN)[q] = ay[q] * ay[q] / A(l, APV)[q];
            A(l, AP)[q] = A(l, AW)[q] + A(l, AE)[q] + A(l, AS)[q] + A(l, AN)[q]
                          + (1 - l->tag[q]) * 1.0e30;
        }
    const double diag = 1.0e30;       /* p' Dirichlet rows :1045-1090 */
    if (c->cfg.ibc_xm == 2)
        for (int j = 1; j < ny - 1; ++j) { int q = j * nx + 1; A(l, AP)[q] += diag; A(l, SU)[q] = 0.0; }
    if (c->cfg.ibc_xp == 2)
        for (int j = 1; j < ny - 1; ++j) { int q = j * nx + nx - 2; A(l, AP)[q] += diag; A(l, SU)[q] = 0.0; }
    if (c->cfg.ibc_ym == 2)
        for (int i = 1; i < nx - 1; ++i) { int q = nx + i; A(l, AP)[q] += diag; A(l, SU)[q] = 0.0; }
    if (c->cfg.ibc_yp == 2)
        for (int i = 1; i < nx - 1; ++i) { int q = (ny - 2) * nx + i; A(l, AP)[q] += diag; A(l, SU)[q] = 0.0; }
}

/* update :1127-1178, including the host-side obstacle pressure copy :1153-1177 */
static void update(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double *u = A(l, U), *v = A(l, V), *p = A(l, P), *pp = A(l, PP);
    const double ppref = 0.0;
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i;
            u[q] += A(l, AREAX)[q] * (pp[q] - pp[q + 1]) / A(l, APU)[q];
            v[q] += A(l, AREAY)[q] * (pp[q] - pp[q + nx]) / A(l, APV)[q];
            p[q] += c->cfg.relxp * (pp[q] - ppref);
        }
    for (int k = 0; k < c->cfg.nobs; ++k) {
        const int *r = &l->rng[4 * k];
        for (int i = r[0]; i <= r[1]; ++i) p[r[2] * nx + i] = p[(r[2] - 1) * nx + i];
        for (int i = r[0]; i <= r[1]; ++i) p[r[3] * nx + i] = p[(r[3] + 1) * nx + i];
        for (int j = r[2]; j <= r[3]; ++j) p[j * nx + r[0]] = p[j * nx + r[0] - 1];
        for (int j = r[2]; j <= r[3]; ++j) p[j * nx + r[1]] = p[j * nx + r[1] + 1];
    }
}

/* pbound :1179-1210 (periodic copies; the y loop keeps the reference's flat offsets) */
static void pbound(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    double *u = A(l, U), *v = A(l, V);
    if (c->cfg.ibc_xm == 3)
        for (int j = 1; j < ny - 1; ++j) {
            int q = j * nx, q1 = q + nx - 3;
            u[q] = u[q1]; u[q1 + 1] = u[q + 1];
            v[q] = v[q1]; v[q1 + 1] = v[q + 1];
        }
    if (c->cfg.ibc_ym == 3)
        for (int i = 1; i < nx - 1; ++i) {
            int q = i, q1 = q + ny - 3;
            u[q] = u[q1]; u[q1 + nx] = u[q + nx];
            v[q] = v[q1]; v[q1 + nx] = v[q + nx];
        }
}

/* outflow :1211-1228 */
static void outflow(orc_case *c, lvl_t *l)
{
    int nx = l->npx, ny = l->npy;
    if (c->cfg.ibc_xp != 4) return;
    for (int j = 0; j < ny; ++j) {
        int q = j * nx + nx - 1;
        A(l, U)[q - 1] = A(l, U)[q - 2];
        A(l, V)[q] = A(l, V)[q - 1];
        A(l, P)[q] = A(l, P)[q - 1];
        A(l, SC)[q] = A(l, SC)[q - 1];
    }
}

/* ------------------------------------------------------------ smoothers */
/* solver (Jacobi, wj = 1) :1231-1296: ping-pong between phi and a copy. */
static void jacobi(orc_case *c, lvl_t *l, double *phi, int nx, int ny, int nsw)
{
    (void)c;
    int npx = l->npx, n = l->npx * l->npy;
    const double wj = 1.0;             /* :1241 (the 0.67 ternary after it is dead code) */
    double *work = (double *)malloc(sizeof(double) * n);
    memcpy(work, phi, sizeof(double) * n);
    double *cur = phi, *nxt = work;
    const double *aw = A(l, AW), *ae = A(l, AE), *as = A(l, AS), *an = A(l, AN), *ap = A(l, AP), *su = A(l, SU);
    for (int it = 0; it < nsw; ++it) {
        for (int j = 1; j < ny; ++j)
            for (int i = 1; i < nx; ++i) {
                int q = j * npx + i;
                double nb = aw[q] * cur[q - 1] + ae[q] * cur[q + 1] + as[q] * cur[q - npx] + an[q] * cur[q + npx];
                double g = (nb + su[q]) / (ap[q] + 1.0e-30);
                nxt[q] = (1.0 - wj) * cur[q] + wj * g;
            }
        double *t = cur; cur = nxt; nxt = t;
    }
    if (cur != phi) memcpy(phi, work, sizeof(double) * n);
    free(work);
}

/* solvergs (red-black Gauss-Seidel) :1297-1351 */
static void rbgs(lvl_t *l, double *phi, int nx, int ny, int nsw)
{
    int npx = l->npx;
    const double *aw = A(l, AW), *ae = A(l, AE), *as = A(l, AS), *an = A(l, AN), *ap = A(l, AP), *su = A(l, SU);
    for (int it = 0; it < nsw; ++it)
        for (int colour = 0; colour < 2; ++colour)
            for (int j = 1; j < ny; ++j)
                for (int i = 1; i < nx; ++i) {
                    if ((i + j) % 2 != colour) continue;
                    int q = j * npx + i;
                    double nb = aw[q] * phi[q - 1] + ae[q] * phi[q + 1] + as[q] * phi[q - npx] + an[q] * phi[q + npx];
                    phi[q] = (nb + su[q]) / ap[q];
                }
}

/* field, extent and sweep count of each equation (:701, :710, :725, :735, :1238) */
static void smooth(orc_case *c, lvl_t *l, int which)
{
    double *phi; int nx, ny, nsw;
    switch (which) {
    case 0: phi = A(l, U); nx = l->npx - 2; ny = l->npy - 1; nsw = c->cfg.nswpm; break;
    case 1: phi = A(l, V); nx = l->npx - 1; ny = l->npy - 2; nsw = c->cfg.nswpm; break;
    case 2: phi = A(l, PP); nx = l->npx - 1; ny = l->npy - 1; nsw = c->cfg.nswpp; break;
    default: phi = A(l, SC); nx = l->npx - 1; ny = l->npy - 1; nsw = c->cfg.nswpm; break;
    }
    if (c->cfg.isolve == 1) jacobi(c, l, phi, nx, ny, nsw);
    else if (c->cfg.isolve == 2) rbgs(l, phi, nx, ny, nsw);
}

/* solve_u / solve_v / solve_pprime / solve_sc :696-737 */
static void solve_u(orc_case *c, lvl_t *l) { coefu(l); umom(c, l); smooth(c, l, 0); }
static void solve_v(orc_case *c, lvl_t *l) { coefv(l); vmom(c, l); smooth(c, l, 1); }
static double solve_pp(orc_case *c, lvl_t *l)
{
    double e = masserror(l);
    c->last_err = e;
    coefp(c, l);
    smooth(c, l, 2);
    update(c, l);
    return e;
}
static void solve_sc(orc_case *c, lvl_t *l) { coefsc(c, l); scalar_src(c, l); smooth(c, l, 3); }

/* ---------------------------------------------------------- restriction */
/* restv :1354-1389 */
static void restv(lvl_t *f, lvl_t *k)
{
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic, qw = q - 1, qs = q - nxf;
            A(k, U)[qc] = (A(f, U)[q] * A(f, AREAX)[q] + A(f, U)[qs] * A(f, AREAX)[qs]) / (A(k, AREAX)[qc] + 1.0e-30);
            A(k, V)[qc] = (A(f, V)[q] * A(f, AREAY)[q] + A(f, V)[qw] * A(f, AREAY)[qw]) / (A(k, AREAY)[qc] + 1.0e-30);
            A(k, P)[qc] = 0.25 * (A(f, P)[q] + A(f, P)[qw] + A(f, P)[qs] + A(f, P)[qs - 1]);
            A(k, SC)[qc] = 0.25 * (A(f, SC)[q] + A(f, SC)[qw] + A(f, SC)[qs] + A(f, SC)[qs - 1]);
        }
}

static void zero(double *x, int n) { memset(x, 0, sizeof(double) * (size_t)n); }

/* residual of the u equation on one level: restru :1474-1564 */
static void resid_u(orc_case *c, lvl_t *l, int with_defect)
{
    int nx = l->npx, ny = l->npy;
    double *rs = A(l, RS), *u = A(l, U), *p = A(l, P);
    zero(rs, nx * ny);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 2; ++i) {
            int q = j * nx + i;
            double r = A(l, AW)[q] * u[q - 1] + A(l, AE)[q] * u[q + 1] + A(l, AS)[q] * u[q - nx]
                     + A(l, AN)[q] * u[q + nx] - A(l, AP)[q] * u[q]
                     + A(l, AREAX)[q] * (p[q] - p[q + 1]);
            if (with_defect)
                r = r + A(l, RESU)[q] + c->cfg.dpdxm * A(l, AREAX)[q] * A(l, AREAY)[q];
            else
                r = r + c->cfg.dpdxm * A(l, AREAX)[q] * A(l, AREAY)[q];
            if (with_defect && A(l, AREAX)[q] == 0.0) r = 0.0;
            rs[q] = r;
        }
}

static void restru(orc_case *c, lvl_t *f, lvl_t *k)
{
    coefu(f); resid_u(c, f, 1);
    coefu(k); resid_u(c, k, 0);
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    double *rf = A(f, RS), *rc = A(k, RS);
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 2; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            A(k, RESU)[qc] = (rf[q] + rf[q - nxf])
                           + 0.5 * (rf[q - 1] + rf[q - 1 - nxf] + rf[q + 1] + rf[q + 1 - nxf])
                           - rc[qc];
        }
}

/* restrv :1650-1740 */
static void resid_v(orc_case *c, lvl_t *l, int with_defect)
{
    int nx = l->npx, ny = l->npy;
    double *rs = A(l, RS), *v = A(l, V), *p = A(l, P);
    zero(rs, nx * ny);
    for (int j = 1; j < ny - 2; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i;
            double r = A(l, AW)[q] * v[q - 1] + A(l, AE)[q] * v[q + 1] + A(l, AS)[q] * v[q - nx]
                     + A(l, AN)[q] * v[q + nx] - A(l, AP)[q] * v[q]
                     + A(l, AREAY)[q] * (p[q] - p[q + nx]);
            if (with_defect)
                r = r + A(l, RESV)[q] + c->cfg.dpdym * A(l, AREAX)[q] * A(l, AREAY)[q];
            else
                r = r + c->cfg.dpdym * A(l, AREAX)[q] * A(l, AREAY)[q];
            if (with_defect && A(l, AREAY)[q] == 0.0) r = 0.0;
            rs[q] = r;
        }
}

static void restrv(orc_case *c, lvl_t *f, lvl_t *k)
{
    coefv(f); resid_v(c, f, 1);
    coefv(k); resid_v(c, k, 0);
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    double *rf = A(f, RS), *rc = A(k, RS);
    for (int jc = 1; jc < nyc - 2; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            A(k, RESV)[qc] = (rf[q] + rf[q - 1])
                           + 0.5 * (rf[q - nxf] + rf[q - nxf - 1] + rf[q + nxf] + rf[q + nxf - 1])
                           - rc[qc];
        }
}

/* restrsc :1565-1648 */
static void resid_sc(lvl_t *l, int with_defect)
{
    int nx = l->npx, ny = l->npy;
    double *rs = A(l, RS), *s = A(l, SC);
    zero(rs, nx * ny);
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int q = j * nx + i;
            double r = A(l, AW)[q] * s[q - 1] + A(l, AE)[q] * s[q + 1] + A(l, AS)[q] * s[q - nx]
                     + A(l, AN)[q] * s[q + nx] - A(l, AP)[q] * s[q];
            if (with_defect) r = r + A(l, RESSC)[q];
            rs[q] = r;
        }
}

static void restrsc(orc_case *c, lvl_t *f, lvl_t *k)
{
    coefsc(c, f); resid_sc(f, 1);
    coefsc(c, k); resid_sc(k, 0);
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    double *rf = A(f, RS), *rc = A(k, RS);
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            A(k, RESSC)[qc] = (rf[q] + rf[q - nxf] + rf[q - 1] + rf[q - 1 - nxf]) - rc[qc];
        }
}

/* ---------------------------------------------------------- prolongation */
/* prolu :1745-1819 (sequential scatter) */
static void prolu(lvl_t *f, lvl_t *k)
{
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    double *cc = A(k, C), *u = A(f, U);
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) cc[jc * nxc + ic] = 0.0;
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 2; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            double r = (u[q] * A(f, AREAX)[q] + u[q - nxf] * A(f, AREAX)[q - nxf]) / (A(k, AREAX)[qc] + 1.0E-30);
            cc[qc] = A(k, U)[qc] - r;
        }
    const double f1 = 3. / 4., f2 = 1. / 4.;
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 2; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            double c1 = f1 * cc[qc] + f2 * cc[qc + nxc];
            double c2 = f1 * cc[qc] + f2 * cc[qc - nxc];
            if (A(f, SPU)[q] > 1.0e10) { c1 = 0.0; c2 = 0.0; }
            u[q] += c1;            u[q - nxf] += c2;
            u[q - 1] += 0.5 * c1;  u[q - nxf - 1] += 0.5 * c2;
            u[q + 1] += 0.5 * c1;  u[q - nxf + 1] += 0.5 * c2;
        }
}

/* prolv :1821-1892 */
static void prolv(lvl_t *f, lvl_t *k)
{
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    double *cc = A(k, C), *v = A(f, V);
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) cc[jc * nxc + ic] = 0.0;
    for (int jc = 1; jc < nyc - 2; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            double r = (v[q] * A(f, AREAY)[q] + v[q - 1] * A(f, AREAY)[q - 1]) / (A(k, AREAY)[qc] + 1.0E-30);
            cc[qc] = A(k, V)[qc] - r;
        }
    const double f1 = 3. / 4., f2 = 1. / 4.;
    for (int jc = 1; jc < nyc - 2; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            double c1 = f1 * cc[qc] + f2 * cc[qc + 1];
            double c2 = f1 * cc[qc] + f2 * cc[qc - 1];
            if (A(f, SPV)[q] > 1.0e10) { c1 = 0.0; c2 = 0.0; }
            v[q] += c1;              v[q - 1] += c2;
            v[q - nxf] += 0.5 * c1;  v[q - 1 - nxf] += 0.5 * c2;
            v[q + nxf] += 0.5 * c1;  v[q - 1 + nxf] += 0.5 * c2;
        }
}

/* prolp :1894-1961 and prolsc :1962-2028 (bilinear 9/16, 3/16, 3/16, 1/16) */
static void prol_cell(lvl_t *f, lvl_t *k, int fld, int mask_by_spu)
{
    int nxf = f->npx, nxc = k->npx, nyc = k->npy;
    double *cc = A(k, C), *x = f->a[fld], *xc = k->a[fld];
    zero(cc, nxc * nyc);
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic, qs = q - nxf;
            double r = 0.25 * (x[q] + x[q - 1] + x[qs] + x[qs - 1]);
            cc[qc] = xc[qc] - r;
            if (mask_by_spu && A(f, SPU)[q] > 1.0e10) cc[qc] = 0.0;
        }
    const double f1 = 9. / 16., f2 = 3. / 16., f3 = 3. / 16., f4 = 1. / 16.;
    for (int jc = 1; jc < nyc - 1; ++jc)
        for (int ic = 1; ic < nxc - 1; ++ic) {
            int qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic;
            x[q]           += f1 * cc[qc] + f2 * cc[qc + 1] + f3 * cc[qc + nxc] + f4 * cc[qc + 1 + nxc];
            x[q - 1]       += f1 * cc[qc] + f2 * cc[qc - 1] + f3 * cc[qc + nxc] + f4 * cc[qc - 1 + nxc];
            x[q - nxf]     += f1 * cc[qc] + f2 * cc[qc + 1] + f3 * cc[qc - nxc] + f4 * cc[qc + 1 - nxc];
            x[q - nxf - 1] += f1 * cc[qc] + f2 * cc[qc - 1] + f3 * cc[qc - nxc] + f4 * cc[qc - 1 - nxc];
        }
}

/* -------------------------------------------------------- level routines */
static void step_down(orc_case *c, int ig)    /* :201-207 */
{
    lvl_t *l = &c->L[ig];
    fluxes(l);
    solve_u(c, l);
    solve_v(c, l);
    double e = solve_pp(c, l);
    if (ig == 0) {
        if (c->nh == c->caph) {
            c->caph = c->caph ? 2 * c->caph : 1024;
            c->err = (double *)realloc(c->err, sizeof(double) * c->caph);
            c->delta = (double *)realloc(c->delta, sizeof(double) * c->caph);
        }
        c->err[c->nh] = e;
        c->delta[c->nh] = 0.0;
    }
    pbound(c, l);
    outflow(c, l);
    solve_sc(c, l);
}

static void step_up(orc_case *c, int ig)      /* :235-244 */
{
    lvl_t *l = &c->L[ig];
    fluxes(l);
    solve_u(c, l);
    solve_v(c, l);
    solve_pp(c, l);
    pbound(c, l);
    solve_sc(c, l);
    outflow(c, l);
}

static void restrict_to(orc_case *c, int ig)  /* :211-220 */
{
    lvl_t *f = &c->L[ig], *k = &c->L[ig + 1];
    restv(f, k);
    fluxes(k);
    fluxes(f);
    restru(c, f, k);
    restrv(c, f, k);
    restrsc(c, f, k);
}

static void prolong_from(orc_case *c, int ig) /* :230-233, coarse ig+1 -> fine ig */
{
    lvl_t *f = &c->L[ig], *k = &c->L[ig + 1];
    prolu(f, k);
    prolv(f, k);
    prol_cell(f, k, MGFVM_F_P, 1);
    prol_cell(f, k, MGFVM_F_SC, 0);
}

/* Fixed-point change between this cycle's and the previous cycle's level-0 state:
 * relative L2 change of u, v, sc and of p with its interior mean removed (shifted
 * sums so a uniform pressure drift does not cancel catastrophically). */
static double fixed_point_delta(orc_case *c)
{
    lvl_t *l = &c->L[0];
    int nx = l->npx, ny = l->npy;
    const int flds[4] = {MGFVM_F_U, MGFVM_F_V, MGFVM_F_SC, MGFVM_F_P};
    double worst = 0.0;
    double N = (double)(nx - 2) * (double)(ny - 2);
    for (int t = 0; t < 4; ++t) {
        const double *x = l->a[flds[t]], *y = c->prev[t];
        double num = 0.0, den = 0.0;
        if (t < 3) {
            for (int j = 1; j < ny - 1; ++j)
                for (int i = 1; i < nx - 1; ++i) {
                    int q = j * nx + i;
                    double d = x[q] - y[q];
                    num += d * d;
                    den += x[q] * x[q];
                }
        } else {
            int q0 = nx + 1;
            double kd = x[q0] - y[q0], kp = x[q0];
            double s1 = 0, s2 = 0, t1 = 0, t2 = 0;
            for (int j = 1; j < ny - 1; ++j)
                for (int i = 1; i < nx - 1; ++i) {
                    int q = j * nx + i;
                    double d = (x[q] - y[q]) - kd, e = x[q] - kp;
                    s1 += d; s2 += d * d; t1 += e; t2 += e * e;
                }
            num = s2 - s1 * s1 / N;
            den = t2 - t1 * t1 / N;
            if (num < 0) num = 0;
        }
        double r;
        if (num == 0.0) r = 0.0;
        else if (den <= 0.0) r = INFINITY;
        else r = sqrt(num / den);
        if (r > worst || r != r) worst = r;
    }
    return worst;
}

static void snapshot_prev(orc_case *c)
{
    lvl_t *l = &c->L[0];
    size_t n = (size_t)l->npx * l->npy;
    const int flds[4] = {MGFVM_F_U, MGFVM_F_V, MGFVM_F_SC, MGFVM_F_P};
    for (int t = 0; t < 4; ++t) memcpy(c->prev[t], l->a[flds[t]], sizeof(double) * n);
    c->have_prev = 1;
}

void orc_cycle(orc_case *c)                   /* :195-249 */
{
    for (int ig = 0; ig < c->ng; ++ig) {
        step_down(c, ig);
        if (ig != c->ng - 1) restrict_to(c, ig);
    }
    for (int ig = c->ng - 1; ig > 0; ig--) {
        prolong_from(c, ig - 1);
        if (ig != 1) step_up(c, ig - 1);
    }
    c->delta[c->nh] = c->have_prev ? fixed_point_delta(c) : 0.0;
    snapshot_prev(c);
    c->nh++;
}

int orc_solve(orc_case *c, int max_cycles, double fp_tol)
{
    int n = 0;
    while (n < max_cycles) {
        orc_cycle(c);
        ++n;
        double e = c->err[c->nh - 1], d = c->delta[c->nh - 1];
        if (e < c->cfg.convergence) break;
        if (fp_tol > 0.0 && c->nh >= 2 && d < fp_tol) break;
    }
    return n;
}

int orc_op(orc_case *c, int op, int level)
{
    if (level < 0 || level >= c->ng) return MGFVM_EINVAL;
    lvl_t *l = &c->L[level];
    switch (op) {
    case MGFVM_OP_FLUXES: fluxes(l); break;
    case MGFVM_OP_SOLVE_U: solve_u(c, l); break;
    case MGFVM_OP_SOLVE_V: solve_v(c, l); break;
    case MGFVM_OP_SOLVE_PP: solve_pp(c, l); break;
    case MGFVM_OP_PBOUND: pbound(c, l); break;
    case MGFVM_OP_OUTFLOW: outflow(c, l); break;
    case MGFVM_OP_SOLVE_SC: solve_sc(c, l); break;
    case MGFVM_OP_RESTRICT: if (level + 1 >= c->ng) return MGFVM_EINVAL; restrict_to(c, level); break;
    case MGFVM_OP_PROLONG: if (level + 1 >= c->ng) return MGFVM_EINVAL; prolong_from(c, level); break;
    case MGFVM_OP_SMOOTH_U: smooth(c, l, 0); break;
    case MGFVM_OP_SMOOTH_V: smooth(c, l, 1); break;
    case MGFVM_OP_SMOOTH_PP: smooth(c, l, 2); break;
    case MGFVM_OP_SMOOTH_SC: smooth(c, l, 3); break;
    default: return MGFVM_EINVAL;
    }
    return MGFVM_OK;
}

/* ------------------------------------------------------------ public */
int orc_create(const mgfvm_config *cfg, const double *inlet_u, int n_inlet, orc_case **out)
{
    *out = NULL;
    if (cfg->ngrid < 1 || cfg->nfx < 1 || cfg->nfy < 1) return MGFVM_EINVAL;
    orc_case *c = (orc_case *)calloc(1, sizeof(orc_case));
    if (!c) return MGFVM_ENOMEM;
    c->cfg = *cfg;
    c->obs = (int *)malloc(sizeof(int) * 4 * (size_t)(cfg->nobs > 0 ? cfg->nobs : 1));
    if (cfg->nobs > 0) memcpy(c->obs, cfg->obs, sizeof(int) * 4 * (size_t)cfg->nobs);
    c->cfg.obs = c->obs;
    int rc = alloc_levels(c);
    if (rc) { orc_destroy(c); return rc; }
    init_levels(c);
    if (inlet_u && n_inlet > 0) {
        lvl_t *l = &c->L[0];
        for (int j = 1; j <= n_inlet && j < l->npy - 1; ++j) A(l, U)[j * l->npx] = inlet_u[j - 1];
    }
    rest_geom(c);
    size_t n0 = (size_t)c->L[0].npx * c->L[0].npy;
    for (int t = 0; t < 4; ++t) c->prev[t] = (double *)calloc(n0, sizeof(double));
    c->caph = 1024;
    c->err = (double *)malloc(sizeof(double) * c->caph);
    c->delta = (double *)malloc(sizeof(double) * c->caph);
    *out = c;
    return MGFVM_OK;
}

void orc_destroy(orc_case *c)
{
    if (!c) return;
    if (c->L) {
        for (int ig = 0; ig < c->ng; ++ig) {
            lvl_t *l = &c->L[ig];
            for (int f = 0; f < MGFVM_NFIELDS; ++f) free(l->a[f]);
            free(l->tag); free(l->rng); free(l->inl); free(l->outl);
        }
        free(c->L);
    }
    for (int t = 0; t < 4; ++t) free(c->prev[t]);
    free(c->err); free(c->delta); free(c->obs);
    free(c);
}

int orc_ngrid(const orc_case *c) { return c->ng; }

int orc_dims(const orc_case *c, int level, int *npx, int *npy)
{
    if (level < 0 || level >= c->ng) return MGFVM_EINVAL;
    *npx = c->L[level].npx; *npy = c->L[level].npy;
    return MGFVM_OK;
}

int orc_get(const orc_case *c, int level, int field, double *out)
{
    if (level < 0 || level >= c->ng || field < 0 || field >= MGFVM_NFIELDS) return MGFVM_EINVAL;
    const lvl_t *l = &c->L[level];
    memcpy(out, l->a[field], sizeof(double) * (size_t)l->npx * l->npy);
    return MGFVM_OK;
}

int orc_set(orc_case *c, int level, int field, const double *in)
{
    if (level < 0 || level >= c->ng || field < 0 || field >= MGFVM_NFIELDS) return MGFVM_EINVAL;
    lvl_t *l = &c->L[level];
    memcpy(l->a[field], in, sizeof(double) * (size_t)l->npx * l->npy);
    return MGFVM_OK;
}

int orc_get_tag(const orc_case *c, int level, int *out)
{
    if (level < 0 || level >= c->ng) return MGFVM_EINVAL;
    const lvl_t *l = &c->L[level];
    memcpy(out, l->tag, sizeof(int) * (size_t)l->npx * l->npy);
    return MGFVM_OK;
}

int orc_get_obstacle_ranges(const orc_case *c, int level, int *out)
{
    if (level < 0 || level >= c->ng) return MGFVM_EINVAL;
    memcpy(out, c->L[level].rng, sizeof(int) * 4 * (size_t)c->cfg.nobs);
    return MGFVM_OK;
}

int orc_history(const orc_case *c, double *err, double *delta, int cap)
{
    int n = c->nh < cap ? c->nh : cap;
    if (err) memcpy(err, c->err, sizeof(double) * (size_t)n);
    if (delta) memcpy(delta, c->delta, sizeof(double) * (size_t)n);
    return c->nh;
}

double orc_last_err(const orc_case *c) { return c->last_err; }
