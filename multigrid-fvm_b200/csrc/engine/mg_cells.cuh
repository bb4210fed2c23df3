// mg_cells.cuh — the per-cell arithmetic of every V-cycle routine, shared by the
// grid-wide kernels (one thread per cell, all cases of a batch in one launch), the
// shared-memory tile smoothers and the coarse-level kernel (one CTA per case).
//
// Every function restates one loop body of Version-6-26-04.c with the operations in
// the reference's order; this code is compiled with --fmad=false so the FP64 results
// are bit-identical to the reference built with gcc.  Where the reference runs a
// second loop over boundary rows or obstacle cells after the main loop, the
// function applies that loop's additions to the cell in the same order.
#pragma once

#include "mg_common.cuh"

namespace mg {

#define MGF(L, s) ((L).f[(s)])

// max(|c|, D) +/- c: the hybrid upwind/central coefficient (:845-848)
__device__ __forceinline__ double hyb_p(double c, double d) { return fmax(fabs(c), d) + c; }
__device__ __forceinline__ double hyb_m(double c, double d) { return fmax(fabs(c), d) - c; }

struct Coef { double aw, ae, as, an, ap; };

// Face mass fluxes cx = 0.5 u A_x, cy = 0.5 v A_y (fluxes :678-694), either read from
// the arrays fluxes() filled or recomputed from u, v: identical bits either way, so a
// kernel that runs right after the fluxes would be computed may skip the round trip.
struct FluxArrays {
    const double *cx, *cy;
    __device__ __forceinline__ FluxArrays(const LevelDev &L) : cx(MGF(L, S_CX)), cy(MGF(L, S_CY)) {}
    __device__ __forceinline__ double x(int q) const { return cx[q]; }
    __device__ __forceinline__ double y(int q) const { return cy[q]; }
};
struct FluxLive {
    const double *u, *v, *ax, *ay;
    __device__ __forceinline__ FluxLive(const LevelDev &L)
        : u(MGF(L, S_U)), v(MGF(L, S_V)), ax(MGF(L, S_AREAX)), ay(MGF(L, S_AREAY)) {}
    __device__ __forceinline__ double x(int q) const { return 0.5 * u[q] * ax[q]; }
    __device__ __forceinline__ double y(int q) const { return 0.5 * v[q] * ay[q]; }
};

// ------------------------------------------------------------------ fluxes
// fluxes :678-694, domain i in [0, npx-2], j in [0, npy-2]
__device__ __forceinline__ void cell_fluxes(const LevelDev &L, int q)
{
    MGF(L, S_CX)[q] = 0.5 * MGF(L, S_U)[q] * MGF(L, S_AREAX)[q];
    MGF(L, S_CY)[q] = 0.5 * MGF(L, S_V)[q] * MGF(L, S_AREAY)[q];
}

// ------------------------------------------------------------ coefficients
// coefu :815-860 at u face (i, j), i in [1, npx-3], j in [1, npy-2], including the
// wall-shear rows j = npy-2 then j = 1 (:849-858; both use areay of row npy-2).
template <class F>
__device__ __forceinline__ Coef coef_u(const LevelDev &L, const F &fl, int i, int j)
{
    const int nx = L.npx, q = j * nx + i, s = q - nx;
    const double cq = fl.x(q);
    double cxm = 0.5 * (cq + fl.x(q - 1));
    double cxp = 0.5 * (cq + fl.x(q + 1));
    double cym = 0.5 * (fl.y(s) + fl.y(s + 1));
    double cyp = 0.5 * (fl.y(q) + fl.y(q + 1));
    double dxm = L.amu * (MGF(L, S_AREAX)[q] / L.dx);
    double dym = L.amu * (MGF(L, S_AREAY)[q] / L.dy);
    Coef k;
    k.aw = hyb_p(cxm, dxm);
    k.ae = hyb_m(cxp, dxm);
    k.as = hyb_p(cym, dym);
    k.an = hyb_m(cyp, dym);
    k.ap = k.aw + k.ae + k.as + k.an;
    const int top = L.npy - 2;
    if (j == top) {
        double add = L.amu * (MGF(L, S_AREAY)[q] / L.dy);
        k.an += add; k.ap += add;
    }
    if (j == 1) {
        double add = L.amu * (MGF(L, S_AREAY)[top * nx + i] / L.dy);
        k.as += add; k.ap += add;
    }
    return k;
}

// coefv :966-1016 at v face (i, j), i in [1, npx-2], j in [1, npy-3], including the
// side-wall columns i = npx-2 then i = 1 (:1005-1015; both use areay of column npx-2).
template <class F>
__device__ __forceinline__ Coef coef_v(const LevelDev &L, const F &fl, int i, int j)
{
    const int nx = L.npx, q = j * nx + i, n = q + nx, s = q - nx;
    double cxm = 0.5 * (fl.x(q - 1) + fl.x(n - 1));
    double cxp = 0.5 * (fl.x(q) + fl.x(n));
    const double cyq = fl.y(q);
    double cym = 0.5 * (cyq + fl.y(s));
    double cyp = 0.5 * (cyq + fl.y(n));
    double dx_ = L.amu * (MGF(L, S_AREAX)[q] / L.dx);
    double dy_ = L.amu * (MGF(L, S_AREAY)[q] / L.dy);
    Coef k;
    k.aw = hyb_p(cxm, dx_);
    k.ae = hyb_m(cxp, dx_);
    k.as = hyb_p(cym, dy_);
    k.an = hyb_m(cyp, dy_);
    k.ap = k.aw + k.ae + k.as + k.an;
    const int rgt = nx - 2;
    if (i == rgt) {
        double add = L.amu * (MGF(L, S_AREAY)[q] / L.dy);
        k.ae += add; k.ap += add;
    }
    if (i == 1) {
        double add = L.amu * (MGF(L, S_AREAY)[j * nx + rgt] / L.dy);
        k.aw += add; k.ap += add;
    }
    return k;
}

// coefsc :861-964 at cell (i, j) interior, then the obstacle-face additions this cell
// receives from the host-only loop :939-963, in that loop's order (codes built by
// mgfvm_build_obstacle_prog: 0 ae from the east cell, 1 aw from the west cell,
// 2 an from the north cell, 3 as from the south cell; count in bits 28-31).
template <class F>
__device__ __forceinline__ Coef coef_sc(const LevelDev &L, const F &fl, int i, int j)
{
    const int nx = L.npx, q = j * nx + i, s = q - nx;
    const double *ax = MGF(L, S_AREAX), *ay = MGF(L, S_AREAY);
    const double amusc = L.amusc;
    double dxm = amusc * (ax[q - 1] / L.dx);
    double dym = amusc * (ay[s] / L.dy);
    double dxp = amusc * (ax[q] / L.dx);
    double dyp = amusc * (ay[q] / L.dy);
    Coef k;
    k.aw = hyb_p(fl.x(q - 1), dxm);
    k.ae = hyb_m(fl.x(q), dxp);
    k.as = hyb_p(fl.y(s), dym);
    k.an = hyb_m(fl.y(q), dyp);
    k.ap = k.aw + k.ae + k.as + k.an;
    if (L.seq) {
        unsigned code = L.seq[q];
        int cnt = (int)(code >> 28);
        for (int t = 0; t < cnt; ++t) {
            int d = (int)((code >> (2 * t)) & 3u);
            double add;
            if (d == 0)      { add = amusc * (ax[q + 1] / L.dx);  k.ae += add; }
            else if (d == 1) { add = amusc * (ax[q - 1] / L.dx);  k.aw += add; }
            else if (d == 2) { add = amusc * (ay[q + nx] / L.dy); k.an += add; }
            else             { add = amusc * (ay[q - nx] / L.dy); k.as += add; }
            k.ap += add;
        }
    }
    return k;
}

__device__ __forceinline__ void store_coef(const LevelDev &L, int eq, int q, const Coef &k, double su)
{
    MGF(L, co_slot(eq, CK_AW))[q] = k.aw; MGF(L, co_slot(eq, CK_AE))[q] = k.ae;
    MGF(L, co_slot(eq, CK_AS))[q] = k.as; MGF(L, co_slot(eq, CK_AN))[q] = k.an;
    MGF(L, co_slot(eq, CK_AP))[q] = k.ap; MGF(L, co_slot(eq, CK_SU))[q] = su;
}

// ---------------------------------------------------------- assembly ops
// solve_u's assembly: coefu :815-860 then umom :741-767 at one u face
template <class F>
__device__ __forceinline__ void cell_mom_u(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j)
{
    const int q = j * L.npx + i;
    Coef k = coef_u(L, fl, i, j);
    const double ax = MGF(L, S_AREAX)[q];
    const double rm = C.relxm, rm1 = 1.0 - C.relxm;
    double su = ax * (MGF(L, S_P)[q] - MGF(L, S_P)[q + 1]);
    double ap = k.ap / rm;
    su = su + rm1 * ap * MGF(L, S_U)[q] + MGF(L, S_RESU)[q] + C.dpdxm * ax * MGF(L, S_AREAY)[q];
    ap = ap + MGF(L, S_SPU)[q];
    k.ap = ap;
    store_coef(L, EQ_U, q, k, su);
    MGF(L, S_APU)[q] = ap;
}

// solve_v's assembly: coefv :966-1016 then vmom :769-793 at one v face
template <class F>
__device__ __forceinline__ void cell_mom_v(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j)
{
    const int q = j * L.npx + i;
    Coef k = coef_v(L, fl, i, j);
    const double ay = MGF(L, S_AREAY)[q];
    const double rm = C.relxm, rm1 = 1.0 - C.relxm;
    double su = ay * (MGF(L, S_P)[q] - MGF(L, S_P)[q + L.npx]);
    double ap = k.ap / rm;
    su = su + rm1 * ap * MGF(L, S_V)[q] + MGF(L, S_RESV)[q] + C.dpdym * MGF(L, S_AREAX)[q] * ay;
    ap = ap + MGF(L, S_SPV)[q];
    k.ap = ap;
    store_coef(L, EQ_V, q, k, su);
    MGF(L, S_APV)[q] = ap;
}

// solve_sc's assembly: coefsc :861-964 (+ obstacle faces) then scalar :795-812
template <class F>
__device__ __forceinline__ void cell_sc(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j)
{
    const int q = j * L.npx + i;
    Coef k = coef_sc(L, fl, i, j);
    const double spsc = MGF(L, S_SPSC)[q];
    double su = spsc * C.sc_obs + MGF(L, S_RESSC)[q];
    k.ap = k.ap + spsc;
    store_coef(L, EQ_SC, q, k, su);
}

// The three assemblies that depend only on the fluxes at the start of a level
// visit, plus those fluxes, at cell (i, j) of the full padded array.
enum AsmBits { A_FLUX = 1, A_U = 2, A_V = 4, A_SC = 8, A_SC_OUTFLOW = 16 };

// The part of `what` thread slice z of 3 does when a launch spreads the assemblies
// over blockIdx.z (slice 0: fluxes and u, 1: v, 2: scalar and its outflow ghost).
__host__ __device__ __forceinline__ unsigned asm_slice(unsigned what, int z, int nz)
{
    if (nz <= 1) return what;
    const unsigned part[3] = {A_FLUX | A_U, A_V, A_SC | A_SC_OUTFLOW};
    return what & part[z];
}
template <class F>
__device__ __forceinline__ void cell_asm(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j,
                                         unsigned what)
{
    const int nx = L.npx, ny = L.npy;
    if ((what & A_FLUX) && i <= nx - 2 && j <= ny - 2) cell_fluxes(L, j * nx + i);
    const bool in = i >= 1 && j >= 1 && i <= nx - 2 && j <= ny - 2;
    if ((what & A_U) && in && i <= nx - 3) cell_mom_u(L, C, fl, i, j);
    if ((what & A_V) && in && j <= ny - 3) cell_mom_v(L, C, fl, i, j);
    if ((what & A_SC) && in) cell_sc(L, C, fl, i, j);
    // the scalar part of outflow (:1226), which the down leg applies before solve_sc
    if ((what & A_SC_OUTFLOW) && i == nx - 1 && C.ibc_xp == 4) MGF(L, S_SC)[j * nx + i] = MGF(L, S_SC)[j * nx + i - 1];
}

// solve_pprime's assembly: masserror :1096-1125 then coefp :1018-1092 (with the
// p' Dirichlet rows in the order x-, x+, y-, y+) at one interior cell; returns |div|.
// u, v: the velocity arrays to read (the fields, or the smoother's buffers holding them)
__device__ __forceinline__ double mass_coefp_values(const LevelDev &L, const CaseDev &C, int i, int j, Coef &k,
                                                    double &su_out, const double *u, const double *v)
{
    const int nx = L.npx, ny = L.npy, q = j * nx + i, s = q - nx;
    const double *ax = MGF(L, S_AREAX), *ay = MGF(L, S_AREAY);
    const double *apu = MGF(L, S_APU), *apv = MGF(L, S_APV);
    const double axq = ax[q], ayq = ay[q];
    double div = axq * u[q] - axq * u[q - 1] + ayq * v[q] - ayq * v[s];
    double su = -div;
    k.aw = ax[q - 1] * ax[q - 1] / apu[q - 1];
    k.ae = axq * axq / apu[q];
    k.as = ay[s] * ay[s] / apv[s];
    k.an = ayq * ayq / apv[q];
    k.ap = k.aw + k.ae + k.as + k.an + (double)(1 - L.tag[q]) * 1.0e30;
    const double diag = 1.0e30;
    if (C.ibc_xm == 2 && i == 1) { k.ap = k.ap + diag; su = 0.0; }
    if (C.ibc_xp == 2 && i == nx - 2) { k.ap = k.ap + diag; su = 0.0; }
    if (C.ibc_ym == 2 && j == 1) { k.ap = k.ap + diag; su = 0.0; }
    if (C.ibc_yp == 2 && j == ny - 2) { k.ap = k.ap + diag; su = 0.0; }
    su_out = su;
    return fabs(div);
}

// `from_tmp`: the u, v, sc smoothing left its results in the ping-pong buffers; they
// are read from there and this cell's values are copied back to the fields.
__device__ __forceinline__ double cell_mass_coefp(const LevelDev &L, const CaseDev &C, int i, int j,
                                                  bool from_tmp = false)
{
    Coef k;
    double su;
    const double *u = MGF(L, from_tmp ? S_TMP0 : S_U), *v = MGF(L, from_tmp ? S_TMP1 : S_V);
    const double ad = mass_coefp_values(L, C, i, j, k, su, u, v);
    if (from_tmp) {
        const int q = j * L.npx + i;
        if (i <= L.npx - 3) MGF(L, S_U)[q] = u[q];
        if (j <= L.npy - 3) MGF(L, S_V)[q] = v[q];
        MGF(L, S_SC)[q] = MGF(L, S_TMP2)[q];
    }
    const int q = j * L.npx + i;
    MGF(L, S_PP)[q] = 0.0;
    store_coef(L, EQ_PP, q, k, su);
    return ad;
}

// update :1127-1152 (the obstacle pressure copy :1153-1177 is a separate gather)
__device__ __forceinline__ void cell_update(const LevelDev &L, const CaseDev &C, int q)
{
    double *u = MGF(L, S_U), *v = MGF(L, S_V), *p = MGF(L, S_P);
    const double *pp = MGF(L, S_PP);
    const double ppref = 0.0;
    const double ppq = pp[q];
    u[q] += MGF(L, S_AREAX)[q] * (ppq - pp[q + 1]) / MGF(L, S_APU)[q];
    v[q] += MGF(L, S_AREAY)[q] * (ppq - pp[q + L.npx]) / MGF(L, S_APV)[q];
    p[q] += C.relxp * (ppq - ppref);
}

// --------------------------------------------------------------- smoothers
__device__ __forceinline__ int eq_field(int e) { return e == EQ_U ? S_U : e == EQ_V ? S_V : e == EQ_PP ? S_PP : S_SC; }
__device__ __forceinline__ int eq_tmp(int e) { return e == EQ_V ? S_TMP1 : e == EQ_SC ? S_TMP2 : S_TMP0; }

// Jacobi point update with wj = 1 (solver :1259-1286) from neighbour values
__device__ __forceinline__ double jacobi_value(double aw, double ae, double as, double an, double ap, double su,
                                               double pw, double pe, double ps, double pn, double pc)
{
    const double wj = 1.0;
    double nb = aw * pw + ae * pe + as * ps + an * pn;
    double g = (nb + su) / (ap + 1.0e-30);
    return (1.0 - wj) * pc + wj * g;
}

// red-black Gauss-Seidel point update (solvergs :1308-1350)
__device__ __forceinline__ double gs_value(double aw, double ae, double as, double an, double ap, double su,
                                           double pw, double pe, double ps, double pn)
{
    double nb = aw * pw + ae * pe + as * ps + an * pn;
    return (nb + su) / ap;
}

// ------------------------------------------------------------ division by a fixed divisor
// A smoother divides by the same ap in every unit of a launch.  The reciprocal y =
// RN(1/b) is taken once with the IEEE division; each quotient is then finished with
// Markstein's correction steps (P. Markstein, IBM J. Res. Develop. 34(1):111-119, 1990;
// J.-M. Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., sec. 4.7):
// q0 = RN(a y); r0 = a - b q0 and q1 = RN(q0 + r0 y) make q1 faithful (|q1 - a/b| <
// ulp), so r1 = a - b q1 is exact and q2 = RN(q1 + r1 y) = RN(a/b).  The theorem needs
// no underflow or overflow anywhere: operands outside [2^-450, 2^450] in magnitude
// (which keeps the quotient within [2^-900, 2^900]), zero, Inf and NaN take the IEEE
// division.  Results are therefore the bits of a / b in every case.
struct Recip {
    double b, y;
    bool ok;
};

__device__ __forceinline__ Recip make_recip(double b)
{
    const double m = fabs(b);
    return {b, 1.0 / b, m >= 0x1p-450 && m <= 0x1p450};
}

__device__ __forceinline__ double ieee_div(double a, double b) { return a / b; }

__device__ __forceinline__ double div_by(double a, const Recip &R)
{
    const double m = fabs(a);
    if (R.ok && m >= 0x1p-450 && m <= 0x1p450) {
        const double q0 = a * R.y;
        const double r0 = fma(-R.b, q0, a);
        const double q1 = fma(r0, R.y, q0);
        const double r1 = fma(-R.b, q1, a);
        return fma(r1, R.y, q1);
    }
    return ieee_div(a, R.b);
}

// gs_value with the divisor's reciprocal precomputed (R = make_recip(ap))
__device__ __forceinline__ double gs_value_r(double aw, double ae, double as, double an, const Recip &R, double su,
                                             double pw, double pe, double ps, double pn)
{
    double nb = aw * pw + ae * pe + as * ps + an * pn;
    return div_by(nb + su, R);
}

// jacobi_value with R = make_recip(ap + 1.0e-30)
__device__ __forceinline__ double jacobi_value_r(double aw, double ae, double as, double an, const Recip &R,
                                                 double su, double pw, double pe, double ps, double pn, double pc)
{
    const double wj = 1.0;
    double nb = aw * pw + ae * pe + as * ps + an * pn;
    double g = div_by(nb + su, R);
    return (1.0 - wj) * pc + wj * g;
}

__device__ __forceinline__ void cell_jacobi(const LevelDev &L, int e, const double *cur, double *nxt, int q)
{
    const int nx = L.npx;
    nxt[q] = jacobi_value(MGF(L, co_slot(e, CK_AW))[q], MGF(L, co_slot(e, CK_AE))[q],
                          MGF(L, co_slot(e, CK_AS))[q], MGF(L, co_slot(e, CK_AN))[q],
                          MGF(L, co_slot(e, CK_AP))[q], MGF(L, co_slot(e, CK_SU))[q],
                          cur[q - 1], cur[q + 1], cur[q - nx], cur[q + nx], cur[q]);
}

__device__ __forceinline__ void cell_gs(const LevelDev &L, int e, double *phi, int q)
{
    const int nx = L.npx;
    phi[q] = gs_value(MGF(L, co_slot(e, CK_AW))[q], MGF(L, co_slot(e, CK_AE))[q],
                      MGF(L, co_slot(e, CK_AS))[q], MGF(L, co_slot(e, CK_AN))[q],
                      MGF(L, co_slot(e, CK_AP))[q], MGF(L, co_slot(e, CK_SU))[q],
                      phi[q - 1], phi[q + 1], phi[q - nx], phi[q + nx]);
}

// ------------------------------------------------------------ restriction
// restv :1354-1389 at coarse interior cell (ic, jc)
__device__ __forceinline__ void cell_restv(const LevelDev &F, const LevelDev &K, int ic, int jc)
{
    const int nxf = F.npx, qc = jc * K.npx + ic, q = 2 * jc * nxf + 2 * ic, qw = q - 1, qs = q - nxf;
    const double *uf = MGF(F, S_U), *vf = MGF(F, S_V), *pf = MGF(F, S_P), *sf = MGF(F, S_SC);
    const double *axf = MGF(F, S_AREAX), *ayf = MGF(F, S_AREAY);
    MGF(K, S_U)[qc] = (uf[q] * axf[q] + uf[qs] * axf[qs]) / (MGF(K, S_AREAX)[qc] + 1.0e-30);
    MGF(K, S_V)[qc] = (vf[q] * ayf[q] + vf[qw] * ayf[qw]) / (MGF(K, S_AREAY)[qc] + 1.0e-30);
    MGF(K, S_P)[qc] = 0.25 * (pf[q] + pf[qw] + pf[qs] + pf[qs - 1]);
    MGF(K, S_SC)[qc] = 0.25 * (sf[q] + sf[qw] + sf[qs] + sf[qs - 1]);
}

// residual of the u equation at face (i, j) (restru :1494-1512 fine, :1528-1541 coarse)
template <class F>
__device__ __forceinline__ double resid_u(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j, bool fine)
{
    const int nx = L.npx, q = j * nx + i;
    Coef k = coef_u(L, fl, i, j);
    const double *u = MGF(L, S_U), *p = MGF(L, S_P);
    const double ax = MGF(L, S_AREAX)[q], ay = MGF(L, S_AREAY)[q];
    double r = k.aw * u[q - 1] + k.ae * u[q + 1] + k.as * u[q - nx] + k.an * u[q + nx]
             - k.ap * u[q] + ax * (p[q] - p[q + 1]);
    if (fine) {
        r = r + MGF(L, S_RESU)[q] + C.dpdxm * ax * ay;
        if (ax == 0.0) r = 0.0;
    } else {
        r = r + C.dpdxm * ax * ay;
    }
    return r;
}

// residual of the v equation (restrv :1670-1688 fine, :1704-1718 coarse)
template <class F>
__device__ __forceinline__ double resid_v(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j, bool fine)
{
    const int nx = L.npx, q = j * nx + i;
    Coef k = coef_v(L, fl, i, j);
    const double *v = MGF(L, S_V), *p = MGF(L, S_P);
    const double ax = MGF(L, S_AREAX)[q], ay = MGF(L, S_AREAY)[q];
    double r = k.aw * v[q - 1] + k.ae * v[q + 1] + k.as * v[q - nx] + k.an * v[q + nx]
             - k.ap * v[q] + ay * (p[q] - p[q + nx]);
    if (fine) {
        r = r + MGF(L, S_RESV)[q] + C.dpdym * ax * ay;
        if (ay == 0.0) r = 0.0;
    } else {
        r = r + C.dpdym * ax * ay;
    }
    return r;
}

// residual of the scalar equation (restrsc :1585-1600 fine, :1618-1630 coarse)
template <class F>
__device__ __forceinline__ double resid_sc(const LevelDev &L, const F &fl, int i, int j, bool fine)
{
    const int nx = L.npx, q = j * nx + i;
    Coef k = coef_sc(L, fl, i, j);
    const double *s = MGF(L, S_SC);
    double r = k.aw * s[q - 1] + k.ae * s[q + 1] + k.as * s[q - nx] + k.an * s[q + nx] - k.ap * s[q];
    if (fine) r = r + MGF(L, S_RESSC)[q];
    return r;
}

// Fine-level residuals of the three transported equations at fine cell (i, j) where
// each is defined (restru :1494-1512, restrv :1670-1688, restrsc :1585-1600), stored
// in the level's ping-pong buffers (free between smoothing calls): u in TMP0, v in
// TMP1, sc in TMP2.  Fluxes are recomputed from the fine u, v (fluxes(fine) :216).
__device__ __forceinline__ void cell_fine_residuals(const LevelDev &F, const CaseDev &C, int i, int j, int which)
{
    const FluxLive ff(F);
    const int nx = F.npx, ny = F.npy, q = j * nx + i;
    const bool in = i >= 1 && j >= 1 && i <= nx - 2 && j <= ny - 2;
    if (!in) return;
    if (which == 0 && i <= nx - 3) MGF(F, S_TMP0)[q] = resid_u(F, C, ff, i, j, true);
    if (which == 1 && j <= ny - 3) MGF(F, S_TMP1)[q] = resid_v(F, C, ff, i, j, true);
    if (which == 2) MGF(F, S_TMP2)[q] = resid_sc(F, ff, i, j, true);
}

// FAS defects at coarse cell (ic, jc): restru :1546-1563 (which 0), restrv :1722-1738
// (1), restrsc :1634-1647 (2), from the fine residuals above and the coarse
// residual of the restricted state (coarse fluxes recomputed from the coarse u, v).
__device__ __forceinline__ void cell_restrict(const LevelDev &F, const LevelDev &K, const CaseDev &C,
                                              int ic, int jc, int which)
{
    const FluxLive fk(K);
    const int nxf = F.npx, nxc = K.npx, nyc = K.npy, qc = jc * nxc + ic;
    const int q = 2 * jc * nxf + 2 * ic;
    if (which == 0 && ic <= nxc - 3) {
        const double *rf = MGF(F, S_TMP0);
        double rc = resid_u(K, C, fk, ic, jc, false);
        MGF(K, S_RESU)[qc] = (rf[q] + rf[q - nxf]) + 0.5 * (rf[q - 1] + rf[q - 1 - nxf] + rf[q + 1] + rf[q + 1 - nxf]) - rc;
    }
    if (which == 1 && jc <= nyc - 3) {
        const double *rf = MGF(F, S_TMP1);
        double rc = resid_v(K, C, fk, ic, jc, false);
        MGF(K, S_RESV)[qc] = (rf[q] + rf[q - 1]) + 0.5 * (rf[q - nxf] + rf[q - nxf - 1] + rf[q + nxf] + rf[q + nxf - 1]) - rc;
    }
    if (which == 2) {
        const double *rf = MGF(F, S_TMP2);
        double rc = resid_sc(K, fk, ic, jc, false);
        MGF(K, S_RESSC)[qc] = (rf[q] + rf[q - nxf] + rf[q - 1] + rf[q - 1 - nxf]) - rc;
    }
}

// ---------------------------------------------------------- prolongation
// coarse corrections c = x_c - R(x_f) at coarse interior cell (ic, jc):
// prolu :1760-1777, prolv :1840-1856, prolp :1914-1928, prolsc :1981-1994
__device__ __forceinline__ void cell_prol_corr(const LevelDev &F, const LevelDev &K, int ic, int jc)
{
    const int nxf = F.npx, nxc = K.npx, nyc = K.npy, qc = jc * nxc + ic;
    const int q = 2 * jc * nxf + 2 * ic, qs = q - nxf;
    if (ic <= nxc - 3) {
        const double *u = MGF(F, S_U), *ax = MGF(F, S_AREAX);
        double r = (u[q] * ax[q] + u[qs] * ax[qs]) / (MGF(K, S_AREAX)[qc] + 1.0E-30);
        MGF(K, S_CU)[qc] = MGF(K, S_U)[qc] - r;
    }
    if (jc <= nyc - 3) {
        const double *v = MGF(F, S_V), *ay = MGF(F, S_AREAY);
        double r = (v[q] * ay[q] + v[q - 1] * ay[q - 1]) / (MGF(K, S_AREAY)[qc] + 1.0E-30);
        MGF(K, S_CV)[qc] = MGF(K, S_V)[qc] - r;
    }
    {
        const double *p = MGF(F, S_P);
        double r = 0.25 * (p[q] + p[q - 1] + p[qs] + p[qs - 1]);
        double c = MGF(K, S_P)[qc] - r;
        if (MGF(F, S_SPU)[q] > 1.0e10) c = 0.0;
        MGF(K, S_CP)[qc] = c;
    }
    {
        const double *s = MGF(F, S_SC);
        double r = 0.25 * (s[q] + s[q - 1] + s[qs] + s[qs - 1]);
        MGF(K, S_C)[qc] = MGF(K, S_SC)[qc] - r;
    }
}

// Fine-cell gather of the reference's scatter-add prolongation (same additions in
// the same order as its sequential loops): fine interior cell (i, j).
__device__ __forceinline__ void cell_prol_apply(const LevelDev &F, const LevelDev &K, int i, int j)
{
    const int nxf = F.npx, nyf = F.npy, nxc = K.npx, nyc = K.npy, q = j * nxf + i;
    const double f1 = 3. / 4., f2 = 1. / 4.;
    // u faces, i in [1, nxf-3]: prolu :1782-1814
    if (i <= nxf - 3) {
        const double *cu = MGF(K, S_CU);
        const double *spu = MGF(F, S_SPU);
        const bool up = (j & 1) == 0;                  // even row: corr1 of jc = j/2
        const int jc = up ? j / 2 : (j + 1) / 2;       // odd row: corr2 of jc = (j+1)/2
        const int dj = up ? nxc : -nxc;
        double u = MGF(F, S_U)[q];
        if ((i & 1) == 0) {
            const int ic = i / 2, qc = jc * nxc + ic;
            double corr = f1 * cu[qc] + f2 * cu[qc + dj];
            if (spu[2 * jc * nxf + 2 * ic] > 1.0e10) corr = 0.0;
            u += corr;
        } else {
            const int ia = (i - 1) / 2, ib = (i + 1) / 2;
            if (ia >= 1) {
                const int qc = jc * nxc + ia;
                double corr = f1 * cu[qc] + f2 * cu[qc + dj];
                if (spu[2 * jc * nxf + 2 * ia] > 1.0e10) corr = 0.0;
                u += 0.5 * corr;
            }
            if (ib <= nxc - 3) {
                const int qc = jc * nxc + ib;
                double corr = f1 * cu[qc] + f2 * cu[qc + dj];
                if (spu[2 * jc * nxf + 2 * ib] > 1.0e10) corr = 0.0;
                u += 0.5 * corr;
            }
        }
        MGF(F, S_U)[q] = u;
    }
    // v faces, j in [1, nyf-3]: prolv :1861-1888
    if (j <= nyf - 3) {
        const double *cv = MGF(K, S_CV);
        const double *spv = MGF(F, S_SPV);
        const bool right = (i & 1) == 0;               // even column: corr1 of ic = i/2
        const int ic = right ? i / 2 : (i + 1) / 2;
        const int di = right ? 1 : -1;
        double v = MGF(F, S_V)[q];
        if ((j & 1) == 0) {
            const int jc = j / 2, qc = jc * nxc + ic;
            double corr = f1 * cv[qc] + f2 * cv[qc + di];
            if (spv[2 * jc * nxf + 2 * ic] > 1.0e10) corr = 0.0;
            v += corr;
        } else {
            const int ja = (j - 1) / 2, jb = (j + 1) / 2;
            if (ja >= 1) {
                const int qc = ja * nxc + ic;
                double corr = f1 * cv[qc] + f2 * cv[qc + di];
                if (spv[2 * ja * nxf + 2 * ic] > 1.0e10) corr = 0.0;
                v += 0.5 * corr;
            }
            if (jb <= nyc - 3) {
                const int qc = jb * nxc + ic;
                double corr = f1 * cv[qc] + f2 * cv[qc + di];
                if (spv[2 * jb * nxf + 2 * ic] > 1.0e10) corr = 0.0;
                v += 0.5 * corr;
            }
        }
        MGF(F, S_V)[q] = v;
    }
    // p and sc cells: prolp :1933-1958, prolsc :1999-2025
    {
        const double g1 = 9. / 16., g2 = 3. / 16., g3 = 3. / 16., g4 = 1. / 16.;
        const int ic = (i + 1) / 2, jc = (j + 1) / 2, qc = jc * nxc + ic;
        const int di = (i & 1) == 0 ? 1 : -1;
        const int dj = (j & 1) == 0 ? nxc : -nxc;
        const double *cp = MGF(K, S_CP), *cs = MGF(K, S_C);
        MGF(F, S_P)[q] += g1 * cp[qc] + g2 * cp[qc + di] + g3 * cp[qc + dj] + g4 * cp[qc + di + dj];
        MGF(F, S_SC)[q] += g1 * cs[qc] + g2 * cs[qc + di] + g3 * cs[qc + dj] + g4 * cs[qc + di + dj];
    }
}

// ---------------------------------------------------------- boundary lines
// outflow :1211-1228 at row j; `with_sc` also copies the scalar ghost
__device__ __forceinline__ void row_outflow(const LevelDev &L, int j, bool with_sc)
{
    const int q = j * L.npx + L.npx - 1;
    MGF(L, S_U)[q - 1] = MGF(L, S_U)[q - 2];
    MGF(L, S_V)[q] = MGF(L, S_V)[q - 1];
    MGF(L, S_P)[q] = MGF(L, S_P)[q - 1];
    if (with_sc) MGF(L, S_SC)[q] = MGF(L, S_SC)[q - 1];
}

// pbound x-periodic :1185-1195, row j in [1, npy-2]
__device__ __forceinline__ void row_periodic_x(const LevelDev &L, int j)
{
    double *u = MGF(L, S_U), *v = MGF(L, S_V);
    const int q = j * L.npx, q1 = q + L.npx - 3;
    u[q] = u[q1]; u[q1 + 1] = u[q + 1];
    v[q] = v[q1]; v[q1 + 1] = v[q + 1];
}

// pbound y-periodic :1197-1208; sequential: later iterations read cells earlier
// iterations wrote (the reference's flat offset i + npy - 3), so one thread runs it.
__device__ __forceinline__ void line_periodic_y(const LevelDev &L)
{
    double *u = MGF(L, S_U), *v = MGF(L, S_V);
    const int nx = L.npx, ny = L.npy;
    for (int i = 1; i < nx - 1; ++i) {
        const int q = i, q1 = q + ny - 3;
        u[q] = u[q1]; u[q1 + nx] = u[q + nx];
        v[q] = v[q1]; v[q1 + nx] = v[q + nx];
    }
}

}  // namespace mg
