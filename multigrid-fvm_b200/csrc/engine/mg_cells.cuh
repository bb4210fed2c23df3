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

// ------------------------------------------------------------- value access
// Every routine below is written once over an access type IO that says how it reads
// and writes a level's arrays.  Prim (here) reads and writes the FP64 fields; the
// engine's kernels use it through the plain-LevelDev wrappers at the end of each
// section.  The tangent kernel (mg_tangent.cu) passes a type whose values are
// (value, derivative) pairs: the same operations in the same order give the same
// value bits and, by the chain rule, the derivative.  IO::T is the value type; `g`
// reads an array that no differentiated parameter changes (face areas, obstacle
// sources), always as plain FP64.
struct Prim {
    using T = double;
    const LevelDev &L;
    __device__ __forceinline__ double ld(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ void st(int s, int q, double v) const { L.f[s][q] = v; }
    __device__ __forceinline__ double g(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ double amu() const { return L.amu; }
    __device__ __forceinline__ double amusc() const { return L.amusc; }
    __device__ __forceinline__ double pb(int k) const { return L.pbuf[k]; }      // pressure-copy buffer
    __device__ __forceinline__ void set_pb(int k, double v) const { L.pbuf[k] = v; }
};

// the value part (comparisons and branches look at values only)
__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double gabs(double x) { return fabs(x); }
__device__ __forceinline__ double gmax(double a, double b) { return fmax(a, b); }

// max(|c|, D) +/- c: the hybrid upwind/central coefficient (:845-848)
template <class T, class D>
__device__ __forceinline__ T hyb_p(const T &c, const D &d) { return gmax(gabs(c), d) + c; }
template <class T, class D>
__device__ __forceinline__ T hyb_m(const T &c, const D &d) { return gmax(gabs(c), d) - c; }

template <class T> struct CoefT { T aw, ae, as, an, ap; };
using Coef = CoefT<double>;

// Face mass fluxes cx = 0.5 u A_x, cy = 0.5 v A_y (fluxes :678-694), either read from
// the arrays fluxes() filled or recomputed from u, v: identical bits either way, so a
// kernel that runs right after the fluxes would be computed may skip the round trip.
template <class IO>
struct FluxArraysT {
    IO io;
    __device__ __forceinline__ typename IO::T x(int q) const { return io.ld(S_CX, q); }
    __device__ __forceinline__ typename IO::T y(int q) const { return io.ld(S_CY, q); }
};
template <class IO>
struct FluxLiveT {
    IO io;
    __device__ __forceinline__ typename IO::T x(int q) const { return 0.5 * io.ld(S_U, q) * io.g(S_AREAX, q); }
    __device__ __forceinline__ typename IO::T y(int q) const { return 0.5 * io.ld(S_V, q) * io.g(S_AREAY, q); }
};
struct FluxArrays : FluxArraysT<Prim> {
    __device__ __forceinline__ FluxArrays(const LevelDev &L) : FluxArraysT<Prim>{Prim{L}} {}
};
struct FluxLive : FluxLiveT<Prim> {
    __device__ __forceinline__ FluxLive(const LevelDev &L) : FluxLiveT<Prim>{Prim{L}} {}
};

// ------------------------------------------------------------------ fluxes
// fluxes :678-694, domain i in [0, npx-2], j in [0, npy-2]
template <class IO>
__device__ __forceinline__ void cell_fluxes_io(const IO &io, int q)
{
    io.st(S_CX, q, 0.5 * io.ld(S_U, q) * io.g(S_AREAX, q));
    io.st(S_CY, q, 0.5 * io.ld(S_V, q) * io.g(S_AREAY, q));
}
__device__ __forceinline__ void cell_fluxes(const LevelDev &L, int q) { cell_fluxes_io(Prim{L}, q); }

// ------------------------------------------------------------ coefficients
// coefu :815-860 at u face (i, j), i in [1, npx-3], j in [1, npy-2], including the
// wall-shear rows j = npy-2 then j = 1 (:849-858; both use areay of row npy-2).
template <class IO, class F>
__device__ __forceinline__ CoefT<typename IO::T> coef_u(const IO &io, const F &fl, int i, int j)
{
    using T = typename IO::T;
    const LevelDev &L = io.L;
    const int nx = L.npx, q = j * nx + i, s = q - nx;
    const T cq = fl.x(q);
    T cxm = 0.5 * (cq + fl.x(q - 1));
    T cxp = 0.5 * (cq + fl.x(q + 1));
    T cym = 0.5 * (fl.y(s) + fl.y(s + 1));
    T cyp = 0.5 * (fl.y(q) + fl.y(q + 1));
    T dxm = io.amu() * (io.g(S_AREAX, q) / L.dx);
    T dym = io.amu() * (io.g(S_AREAY, q) / L.dy);
    CoefT<T> k;
    k.aw = hyb_p(cxm, dxm);
    k.ae = hyb_m(cxp, dxm);
    k.as = hyb_p(cym, dym);
    k.an = hyb_m(cyp, dym);
    k.ap = k.aw + k.ae + k.as + k.an;
    const int top = L.npy - 2;
    if (j == top) {
        T add = io.amu() * (io.g(S_AREAY, q) / L.dy);
        k.an = k.an + add; k.ap = k.ap + add;
    }
    if (j == 1) {
        T add = io.amu() * (io.g(S_AREAY, top * nx + i) / L.dy);
        k.as = k.as + add; k.ap = k.ap + add;
    }
    return k;
}

// coefv :966-1016 at v face (i, j), i in [1, npx-2], j in [1, npy-3], including the
// side-wall columns i = npx-2 then i = 1 (:1005-1015; both use areay of column npx-2).
template <class IO, class F>
__device__ __forceinline__ CoefT<typename IO::T> coef_v(const IO &io, const F &fl, int i, int j)
{
    using T = typename IO::T;
    const LevelDev &L = io.L;
    const int nx = L.npx, q = j * nx + i, n = q + nx, s = q - nx;
    T cxm = 0.5 * (fl.x(q - 1) + fl.x(n - 1));
    T cxp = 0.5 * (fl.x(q) + fl.x(n));
    const T cyq = fl.y(q);
    T cym = 0.5 * (cyq + fl.y(s));
    T cyp = 0.5 * (cyq + fl.y(n));
    T dx_ = io.amu() * (io.g(S_AREAX, q) / L.dx);
    T dy_ = io.amu() * (io.g(S_AREAY, q) / L.dy);
    CoefT<T> k;
    k.aw = hyb_p(cxm, dx_);
    k.ae = hyb_m(cxp, dx_);
    k.as = hyb_p(cym, dy_);
    k.an = hyb_m(cyp, dy_);
    k.ap = k.aw + k.ae + k.as + k.an;
    const int rgt = nx - 2;
    if (i == rgt) {
        T add = io.amu() * (io.g(S_AREAY, q) / L.dy);
        k.ae = k.ae + add; k.ap = k.ap + add;
    }
    if (i == 1) {
        T add = io.amu() * (io.g(S_AREAY, j * nx + rgt) / L.dy);
        k.aw = k.aw + add; k.ap = k.ap + add;
    }
    return k;
}

// coefsc :861-964 at cell (i, j) interior, then the obstacle-face additions this cell
// receives from the host-only loop :939-963, in that loop's order (codes built by
// mgfvm_build_obstacle_prog: 0 ae from the east cell, 1 aw from the west cell,
// 2 an from the north cell, 3 as from the south cell; count in bits 28-31).
template <class IO, class F>
__device__ __forceinline__ CoefT<typename IO::T> coef_sc(const IO &io, const F &fl, int i, int j)
{
    using T = typename IO::T;
    const LevelDev &L = io.L;
    const int nx = L.npx, q = j * nx + i, s = q - nx;
    const T amusc = io.amusc();
    T dxm = amusc * (io.g(S_AREAX, q - 1) / L.dx);
    T dym = amusc * (io.g(S_AREAY, s) / L.dy);
    T dxp = amusc * (io.g(S_AREAX, q) / L.dx);
    T dyp = amusc * (io.g(S_AREAY, q) / L.dy);
    CoefT<T> k;
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
            T add;
            if (d == 0)      { add = amusc * (io.g(S_AREAX, q + 1) / L.dx);  k.ae = k.ae + add; }
            else if (d == 1) { add = amusc * (io.g(S_AREAX, q - 1) / L.dx);  k.aw = k.aw + add; }
            else if (d == 2) { add = amusc * (io.g(S_AREAY, q + nx) / L.dy); k.an = k.an + add; }
            else             { add = amusc * (io.g(S_AREAY, q - nx) / L.dy); k.as = k.as + add; }
            k.ap = k.ap + add;
        }
    }
    return k;
}

template <class IO, class T>
__device__ __forceinline__ void store_coef(const IO &io, int eq, int q, const CoefT<T> &k, const T &su)
{
    io.st(co_slot(eq, CK_AW), q, k.aw); io.st(co_slot(eq, CK_AE), q, k.ae);
    io.st(co_slot(eq, CK_AS), q, k.as); io.st(co_slot(eq, CK_AN), q, k.an);
    io.st(co_slot(eq, CK_AP), q, k.ap); io.st(co_slot(eq, CK_SU), q, su);
}

// ---------------------------------------------------------- assembly ops
// solve_u's assembly: coefu :815-860 then umom :741-767 at one u face
template <class IO, class F>
__device__ __forceinline__ void cell_mom_u(const IO &io, const CaseDev &C, const F &fl, int i, int j)
{
    using T = typename IO::T;
    const int q = j * io.L.npx + i;
    CoefT<T> k = coef_u(io, fl, i, j);
    const double ax = io.g(S_AREAX, q);
    const double rm = C.relxm, rm1 = 1.0 - C.relxm;
    T su = ax * (io.ld(S_P, q) - io.ld(S_P, q + 1));
    T ap = k.ap / rm;
    su = su + rm1 * ap * io.ld(S_U, q) + io.ld(S_RESU, q) + C.dpdxm * ax * io.g(S_AREAY, q);
    ap = ap + io.g(S_SPU, q);
    k.ap = ap;
    store_coef(io, EQ_U, q, k, su);
    io.st(S_APU, q, ap);
}

// solve_v's assembly: coefv :966-1016 then vmom :769-793 at one v face
template <class IO, class F>
__device__ __forceinline__ void cell_mom_v(const IO &io, const CaseDev &C, const F &fl, int i, int j)
{
    using T = typename IO::T;
    const int q = j * io.L.npx + i;
    CoefT<T> k = coef_v(io, fl, i, j);
    const double ay = io.g(S_AREAY, q);
    const double rm = C.relxm, rm1 = 1.0 - C.relxm;
    T su = ay * (io.ld(S_P, q) - io.ld(S_P, q + io.L.npx));
    T ap = k.ap / rm;
    su = su + rm1 * ap * io.ld(S_V, q) + io.ld(S_RESV, q) + C.dpdym * io.g(S_AREAX, q) * ay;
    ap = ap + io.g(S_SPV, q);
    k.ap = ap;
    store_coef(io, EQ_V, q, k, su);
    io.st(S_APV, q, ap);
}

// solve_sc's assembly: coefsc :861-964 (+ obstacle faces) then scalar :795-812
template <class IO, class F>
__device__ __forceinline__ void cell_sc(const IO &io, const CaseDev &C, const F &fl, int i, int j)
{
    using T = typename IO::T;
    const int q = j * io.L.npx + i;
    CoefT<T> k = coef_sc(io, fl, i, j);
    const double spsc = io.g(S_SPSC, q);
    T su = spsc * C.sc_obs + io.ld(S_RESSC, q);
    k.ap = k.ap + spsc;
    store_coef(io, EQ_SC, q, k, su);
}

// The three assemblies that depend only on the fluxes at the start of a level
// visit, plus those fluxes, at cell (i, j) of the full padded array.
enum AsmBits { A_FLUX = 1, A_U = 2, A_V = 4, A_SC = 8, A_SC_OUTFLOW = 16,
               A_F32 = 32,    // mixed precision: store the equations' FP32 smoother operands (mg_kernels.cu)
               A_JAC = 64 };  // with A_F32: the smoother is Jacobi (divisor ap + 1e-30)

// The part of `what` thread slice z of 3 does when a launch spreads the assemblies
// over blockIdx.z (slice 0: fluxes and u, 1: v, 2: scalar and its outflow ghost).
__host__ __device__ __forceinline__ unsigned asm_slice(unsigned what, int z, int nz)
{
    if (nz <= 1) return what;
    const unsigned part[3] = {A_FLUX | A_U, A_V, A_SC | A_SC_OUTFLOW};
    return (what & part[z]) | (what & (unsigned)(A_F32 | A_JAC));
}
template <class IO, class F>
__device__ __forceinline__ void cell_asm_io(const IO &io, const CaseDev &C, const F &fl, int i, int j, unsigned what)
{
    const int nx = io.L.npx, ny = io.L.npy;
    if ((what & A_FLUX) && i <= nx - 2 && j <= ny - 2) cell_fluxes_io(io, j * nx + i);
    const bool in = i >= 1 && j >= 1 && i <= nx - 2 && j <= ny - 2;
    if ((what & A_U) && in && i <= nx - 3) cell_mom_u(io, C, fl, i, j);
    if ((what & A_V) && in && j <= ny - 3) cell_mom_v(io, C, fl, i, j);
    if ((what & A_SC) && in) cell_sc(io, C, fl, i, j);
    // the scalar part of outflow (:1226), which the down leg applies before solve_sc
    if ((what & A_SC_OUTFLOW) && i == nx - 1 && C.ibc_xp == 4) io.st(S_SC, j * nx + i, io.ld(S_SC, j * nx + i - 1));
}
template <class F>
__device__ __forceinline__ void cell_asm(const LevelDev &L, const CaseDev &C, const F &fl, int i, int j,
                                         unsigned what)
{
    cell_asm_io(Prim{L}, C, fl, i, j, what);
}

// solve_pprime's assembly: masserror :1096-1125 then coefp :1018-1092 (with the
// p' Dirichlet rows in the order x-, x+, y-, y+) at one interior cell; returns |div|.
// us, vs: the slots of the velocities to read (the fields, or the smoother's buffers
// holding them).  `parts` (MC_*) selects what is formed: the coefficients, the
// source su (and |div|), or both; each part reads only its own operands.
enum MassParts { MC_COEF = 1, MC_SU = 2, MC_ALL = 3 };
template <class IO>
__device__ __forceinline__ typename IO::T mass_coefp_io(const IO &io, const CaseDev &C, int i, int j,
                                                        CoefT<typename IO::T> &k, typename IO::T &su_out, int us,
                                                        int vs, int parts = MC_ALL)
{
    using T = typename IO::T;
    const LevelDev &L = io.L;
    const int nx = L.npx, ny = L.npy, q = j * nx + i, s = q - nx;
    const double axq = io.g(S_AREAX, q), ayq = io.g(S_AREAY, q);
    T div = T(0.0), su = T(0.0);
    if (parts & MC_SU) {
        div = axq * io.ld(us, q) - axq * io.ld(us, q - 1) + ayq * io.ld(vs, q) - ayq * io.ld(vs, s);
        su = -div;
    }
    if (parts & MC_COEF) {
        const double axw = io.g(S_AREAX, q - 1), ays = io.g(S_AREAY, s);
        k.aw = axw * axw / io.ld(S_APU, q - 1);
        k.ae = axq * axq / io.ld(S_APU, q);
        k.as = ays * ays / io.ld(S_APV, s);
        k.an = ayq * ayq / io.ld(S_APV, q);
        k.ap = k.aw + k.ae + k.as + k.an + (double)(1 - L.tag[q]) * 1.0e30;
    }
    const double diag = 1.0e30;
    const bool cf = (parts & MC_COEF) != 0;
    if (C.ibc_xm == 2 && i == 1) { if (cf) k.ap = k.ap + diag; su = 0.0; }
    if (C.ibc_xp == 2 && i == nx - 2) { if (cf) k.ap = k.ap + diag; su = 0.0; }
    if (C.ibc_ym == 2 && j == 1) { if (cf) k.ap = k.ap + diag; su = 0.0; }
    if (C.ibc_yp == 2 && j == ny - 2) { if (cf) k.ap = k.ap + diag; su = 0.0; }
    su_out = su;
    return gabs(div);
}
__device__ __forceinline__ double mass_coefp_values(const LevelDev &L, const CaseDev &C, int i, int j, Coef &k,
                                                    double &su_out, int us, int vs)
{
    return mass_coefp_io(Prim{L}, C, i, j, k, su_out, us, vs);
}

// `from_tmp`: the u, v, sc smoothing left its results in the ping-pong buffers; they
// are read from there and this cell's values are copied back to the fields.
template <class IO>
__device__ __forceinline__ typename IO::T cell_mass_coefp_io(const IO &io, const CaseDev &C, int i, int j,
                                                             bool from_tmp = false, int parts = MC_ALL)
{
    using T = typename IO::T;
    CoefT<T> k;
    T su;
    const int us = from_tmp ? S_TMP0 : S_U, vs = from_tmp ? S_TMP1 : S_V;
    const T ad = mass_coefp_io(io, C, i, j, k, su, us, vs, parts);
    const int q = j * io.L.npx + i;
    if (from_tmp) {
        if (i <= io.L.npx - 3) io.st(S_U, q, io.ld(us, q));
        if (j <= io.L.npy - 3) io.st(S_V, q, io.ld(vs, q));
        io.st(S_SC, q, io.ld(S_TMP2, q));
    }
    if (parts == MC_ALL) {
        io.st(S_PP, q, T(0.0));
        store_coef(io, EQ_PP, q, k, su);
    } else if (parts == MC_COEF) {
        io.st(S_PP, q, T(0.0));
        io.st(co_slot(EQ_PP, CK_AW), q, k.aw); io.st(co_slot(EQ_PP, CK_AE), q, k.ae);
        io.st(co_slot(EQ_PP, CK_AS), q, k.as); io.st(co_slot(EQ_PP, CK_AN), q, k.an);
        io.st(co_slot(EQ_PP, CK_AP), q, k.ap);
    } else if (parts == MC_SU) {
        io.st(co_slot(EQ_PP, CK_SU), q, su);
    }
    return ad;
}
__device__ __forceinline__ double cell_mass_coefp(const LevelDev &L, const CaseDev &C, int i, int j,
                                                  bool from_tmp = false)
{
    return cell_mass_coefp_io(Prim{L}, C, i, j, from_tmp);
}

// update :1127-1152 (the obstacle pressure copy :1153-1177 is a separate gather);
// `parts` bits 1, 2, 4 select the u, v, p updates (each reads only its own operands)
template <class IO>
__device__ __forceinline__ void cell_update_io(const IO &io, const CaseDev &C, int q, int parts = 7)
{
    using T = typename IO::T;
    const double ppref = 0.0;
    const T ppq = io.ld(S_PP, q);
    if (parts & 1) io.st(S_U, q, io.ld(S_U, q) + io.g(S_AREAX, q) * (ppq - io.ld(S_PP, q + 1)) / io.ld(S_APU, q));
    if (parts & 2)
        io.st(S_V, q, io.ld(S_V, q) + io.g(S_AREAY, q) * (ppq - io.ld(S_PP, q + io.L.npx)) / io.ld(S_APV, q));
    if (parts & 4) io.st(S_P, q, io.ld(S_P, q) + C.relxp * (ppq - ppref));
}
__device__ __forceinline__ void cell_update(const LevelDev &L, const CaseDev &C, int q) { cell_update_io(Prim{L}, C, q); }

// --------------------------------------------------------------- smoothers
__device__ __forceinline__ int eq_field(int e) { return e == EQ_U ? S_U : e == EQ_V ? S_V : e == EQ_PP ? S_PP : S_SC; }
__device__ __forceinline__ int eq_tmp(int e) { return e == EQ_V ? S_TMP1 : e == EQ_SC ? S_TMP2 : S_TMP0; }

// Jacobi point update with wj = 1 (solver :1259-1286) from neighbour values
template <class T>
__device__ __forceinline__ T jacobi_value(const T &aw, const T &ae, const T &as, const T &an, const T &ap,
                                          const T &su, const T &pw, const T &pe, const T &ps, const T &pn,
                                          const T &pc)
{
    const double wj = 1.0;
    T nb = aw * pw + ae * pe + as * ps + an * pn;
    T g = (nb + su) / (ap + 1.0e-30);
    return (1.0 - wj) * pc + wj * g;
}

// red-black Gauss-Seidel point update (solvergs :1308-1350)
template <class T>
__device__ __forceinline__ T gs_value(const T &aw, const T &ae, const T &as, const T &an, const T &ap, const T &su,
                                      const T &pw, const T &pe, const T &ps, const T &pn)
{
    T nb = aw * pw + ae * pe + as * ps + an * pn;
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

template <class IO>
__device__ __forceinline__ void cell_jacobi_io(const IO &io, int e, int cur, int nxt, int q)
{
    const int nx = io.L.npx;
    io.st(nxt, q,
          jacobi_value(io.ld(co_slot(e, CK_AW), q), io.ld(co_slot(e, CK_AE), q), io.ld(co_slot(e, CK_AS), q),
                       io.ld(co_slot(e, CK_AN), q), io.ld(co_slot(e, CK_AP), q), io.ld(co_slot(e, CK_SU), q),
                       io.ld(cur, q - 1), io.ld(cur, q + 1), io.ld(cur, q - nx), io.ld(cur, q + nx), io.ld(cur, q)));
}
template <class IO>
__device__ __forceinline__ void cell_gs_io(const IO &io, int e, int phi, int q)
{
    const int nx = io.L.npx;
    io.st(phi, q,
          gs_value(io.ld(co_slot(e, CK_AW), q), io.ld(co_slot(e, CK_AE), q), io.ld(co_slot(e, CK_AS), q),
                   io.ld(co_slot(e, CK_AN), q), io.ld(co_slot(e, CK_AP), q), io.ld(co_slot(e, CK_SU), q),
                   io.ld(phi, q - 1), io.ld(phi, q + 1), io.ld(phi, q - nx), io.ld(phi, q + nx)));
}
__device__ __forceinline__ void cell_jacobi(const LevelDev &L, int e, int cur, int nxt, int q)
{
    cell_jacobi_io(Prim{L}, e, cur, nxt, q);
}
__device__ __forceinline__ void cell_gs(const LevelDev &L, int e, int phi, int q) { cell_gs_io(Prim{L}, e, phi, q); }

// ------------------------------------------------------------ restriction
// restv :1354-1389 at coarse interior cell (ic, jc); `parts` bits 1, 2, 4, 8 select
// u, v, p, sc (each reads only its own fine values)
template <class IO>
__device__ __forceinline__ void cell_restv_io(const IO &F, const IO &K, int ic, int jc, int parts = 15)
{
    using T = typename IO::T;
    const int nxf = F.L.npx, qc = jc * K.L.npx + ic, q = 2 * jc * nxf + 2 * ic, qw = q - 1, qs = q - nxf;
    T u = T(0.0), v = T(0.0), p = T(0.0), sc = T(0.0);
    if (parts & 1)
        u = (F.ld(S_U, q) * F.g(S_AREAX, q) + F.ld(S_U, qs) * F.g(S_AREAX, qs)) / (K.g(S_AREAX, qc) + 1.0e-30);
    if (parts & 2)
        v = (F.ld(S_V, q) * F.g(S_AREAY, q) + F.ld(S_V, qw) * F.g(S_AREAY, qw)) / (K.g(S_AREAY, qc) + 1.0e-30);
    if (parts & 4) p = 0.25 * (F.ld(S_P, q) + F.ld(S_P, qw) + F.ld(S_P, qs) + F.ld(S_P, qs - 1));
    if (parts & 8) sc = 0.25 * (F.ld(S_SC, q) + F.ld(S_SC, qw) + F.ld(S_SC, qs) + F.ld(S_SC, qs - 1));
    if (parts & 1) K.st(S_U, qc, u);
    if (parts & 2) K.st(S_V, qc, v);
    if (parts & 4) K.st(S_P, qc, p);
    if (parts & 8) K.st(S_SC, qc, sc);
    // the fine level does not change until the prolongation back into it, so these are
    // the R(x_f) the corrections subtract (prol_corr's r, same operations)
    if (parts & 1) K.st(S_RU, qc, u);
    if (parts & 2) K.st(S_RV, qc, v);
    if (parts & 4) K.st(S_RP, qc, p);
    if (parts & 8) K.st(S_RSC, qc, sc);
}
__device__ __forceinline__ void cell_restv(const LevelDev &F, const LevelDev &K, int ic, int jc)
{
    cell_restv_io(Prim{F}, Prim{K}, ic, jc);
}

// residual of the u equation at face (i, j) (restru :1494-1512 fine, :1528-1541 coarse)
template <class IO, class F>
__device__ __forceinline__ typename IO::T resid_u(const IO &io, const CaseDev &C, const F &fl, int i, int j, bool fine)
{
    using T = typename IO::T;
    const int nx = io.L.npx, q = j * nx + i;
    CoefT<T> k = coef_u(io, fl, i, j);
    const double ax = io.g(S_AREAX, q), ay = io.g(S_AREAY, q);
    T r = k.aw * io.ld(S_U, q - 1) + k.ae * io.ld(S_U, q + 1) + k.as * io.ld(S_U, q - nx) + k.an * io.ld(S_U, q + nx)
        - k.ap * io.ld(S_U, q) + ax * (io.ld(S_P, q) - io.ld(S_P, q + 1));
    if (fine) {
        r = r + io.ld(S_RESU, q) + C.dpdxm * ax * ay;
        if (ax == 0.0) r = 0.0;
    } else {
        r = r + C.dpdxm * ax * ay;
    }
    return r;
}

// residual of the v equation (restrv :1670-1688 fine, :1704-1718 coarse)
template <class IO, class F>
__device__ __forceinline__ typename IO::T resid_v(const IO &io, const CaseDev &C, const F &fl, int i, int j, bool fine)
{
    using T = typename IO::T;
    const int nx = io.L.npx, q = j * nx + i;
    CoefT<T> k = coef_v(io, fl, i, j);
    const double ax = io.g(S_AREAX, q), ay = io.g(S_AREAY, q);
    T r = k.aw * io.ld(S_V, q - 1) + k.ae * io.ld(S_V, q + 1) + k.as * io.ld(S_V, q - nx) + k.an * io.ld(S_V, q + nx)
        - k.ap * io.ld(S_V, q) + ay * (io.ld(S_P, q) - io.ld(S_P, q + nx));
    if (fine) {
        r = r + io.ld(S_RESV, q) + C.dpdym * ax * ay;
        if (ay == 0.0) r = 0.0;
    } else {
        r = r + C.dpdym * ax * ay;
    }
    return r;
}

// residual of the scalar equation (restrsc :1585-1600 fine, :1618-1630 coarse)
template <class IO, class F>
__device__ __forceinline__ typename IO::T resid_sc(const IO &io, const F &fl, int i, int j, bool fine)
{
    using T = typename IO::T;
    const int nx = io.L.npx, q = j * nx + i;
    CoefT<T> k = coef_sc(io, fl, i, j);
    T r = k.aw * io.ld(S_SC, q - 1) + k.ae * io.ld(S_SC, q + 1) + k.as * io.ld(S_SC, q - nx)
        + k.an * io.ld(S_SC, q + nx) - k.ap * io.ld(S_SC, q);
    if (fine) r = r + io.ld(S_RESSC, q);
    return r;
}

// Fine-level residuals of the three transported equations at fine cell (i, j) where
// each is defined (restru :1494-1512, restrv :1670-1688, restrsc :1585-1600), stored
// in the level's ping-pong buffers (free between smoothing calls): u in TMP0, v in
// TMP1, sc in TMP2.  Fluxes are recomputed from the fine u, v (fluxes(fine) :216).
template <class IO>
__device__ __forceinline__ void cell_fine_residuals_io(const IO &F, const CaseDev &C, int i, int j, int which)
{
    const FluxLiveT<IO> ff{F};
    const int nx = F.L.npx, ny = F.L.npy, q = j * nx + i;
    const bool in = i >= 1 && j >= 1 && i <= nx - 2 && j <= ny - 2;
    if (!in) return;
    if (which == 0 && i <= nx - 3) F.st(S_TMP0, q, resid_u(F, C, ff, i, j, true));
    if (which == 1 && j <= ny - 3) F.st(S_TMP1, q, resid_v(F, C, ff, i, j, true));
    if (which == 2) F.st(S_TMP2, q, resid_sc(F, ff, i, j, true));
}
__device__ __forceinline__ void cell_fine_residuals(const LevelDev &F, const CaseDev &C, int i, int j, int which)
{
    cell_fine_residuals_io(Prim{F}, C, i, j, which);
}

// FAS defects at coarse cell (ic, jc): restru :1546-1563 (which 0), restrv :1722-1738
// (1), restrsc :1634-1647 (2), from the fine residuals above and the coarse
// residual of the restricted state (coarse fluxes recomputed from the coarse u, v).
template <class IO>
__device__ __forceinline__ void cell_restrict_io(const IO &F, const IO &K, const CaseDev &C, int ic, int jc,
                                                 int which)
{
    using T = typename IO::T;
    const FluxLiveT<IO> fk{K};
    const int nxf = F.L.npx, nxc = K.L.npx, nyc = K.L.npy, qc = jc * nxc + ic;
    const int q = 2 * jc * nxf + 2 * ic;
    if (which == 0 && ic <= nxc - 3) {
        const int r = S_TMP0;
        T rc = resid_u(K, C, fk, ic, jc, false);
        K.st(S_RESU, qc, (F.ld(r, q) + F.ld(r, q - nxf))
                             + 0.5 * (F.ld(r, q - 1) + F.ld(r, q - 1 - nxf) + F.ld(r, q + 1) + F.ld(r, q + 1 - nxf))
                             - rc);
    }
    if (which == 1 && jc <= nyc - 3) {
        const int r = S_TMP1;
        T rc = resid_v(K, C, fk, ic, jc, false);
        K.st(S_RESV, qc, (F.ld(r, q) + F.ld(r, q - 1))
                             + 0.5 * (F.ld(r, q - nxf) + F.ld(r, q - nxf - 1) + F.ld(r, q + nxf) + F.ld(r, q + nxf - 1))
                             - rc);
    }
    if (which == 2) {
        const int r = S_TMP2;
        T rc = resid_sc(K, fk, ic, jc, false);
        K.st(S_RESSC, qc, (F.ld(r, q) + F.ld(r, q - nxf) + F.ld(r, q - 1) + F.ld(r, q - 1 - nxf)) - rc);
    }
}
__device__ __forceinline__ void cell_restrict(const LevelDev &F, const LevelDev &K, const CaseDev &C, int ic, int jc,
                                              int which)
{
    cell_restrict_io(Prim{F}, Prim{K}, C, ic, jc, which);
}

// ---------------------------------------------------------- prolongation
// coarse corrections c = x_c - R(x_f) at coarse interior cell (ic, jc):
// prolu :1760-1777, prolv :1840-1856, prolp :1914-1928, prolsc :1981-1994
template <class IO>
__device__ __forceinline__ void cell_prol_corr_io(const IO &F, const IO &K, int ic, int jc, int parts = 15)
{
    using T = typename IO::T;
    const int nxf = F.L.npx, nxc = K.L.npx, nyc = K.L.npy, qc = jc * nxc + ic;
    const int q = 2 * jc * nxf + 2 * ic, qs = q - nxf;
    if ((parts & 1) && ic <= nxc - 3) {
        T r = (F.ld(S_U, q) * F.g(S_AREAX, q) + F.ld(S_U, qs) * F.g(S_AREAX, qs)) / (K.g(S_AREAX, qc) + 1.0E-30);
        K.st(S_CU, qc, K.ld(S_U, qc) - r);
    }
    if ((parts & 2) && jc <= nyc - 3) {
        T r = (F.ld(S_V, q) * F.g(S_AREAY, q) + F.ld(S_V, q - 1) * F.g(S_AREAY, q - 1)) / (K.g(S_AREAY, qc) + 1.0E-30);
        K.st(S_CV, qc, K.ld(S_V, qc) - r);
    }
    if (parts & 4) {
        T r = 0.25 * (F.ld(S_P, q) + F.ld(S_P, q - 1) + F.ld(S_P, qs) + F.ld(S_P, qs - 1));
        T c = K.ld(S_P, qc) - r;
        if (F.g(S_SPU, q) > 1.0e10) c = 0.0;
        K.st(S_CP, qc, c);
    }
    if (parts & 8) {
        T r = 0.25 * (F.ld(S_SC, q) + F.ld(S_SC, q - 1) + F.ld(S_SC, qs) + F.ld(S_SC, qs - 1));
        K.st(S_C, qc, K.ld(S_SC, qc) - r);
    }
}
__device__ __forceinline__ void cell_prol_corr(const LevelDev &F, const LevelDev &K, int ic, int jc)
{
    cell_prol_corr_io(Prim{F}, Prim{K}, ic, jc);
}

// The coarse corrections a prolongation gathers, either read from the arrays
// cell_prol_corr filled (FUSED = false) or formed where they are needed from the coarse
// state and the R(x_f) restv saved (FUSED = true): the same subtraction on the same
// operands (and the same zeroing of p's correction under solid cells), so the same
// bits.  Outside a correction's domain both read the array (nothing writes it there).
template <class IO, bool FUSED>
struct ProlCorr {
    const IO &F, &K;
    using T = typename IO::T;
    __device__ __forceinline__ T u(int ic, int jc) const
    {
        const int nxc = K.L.npx, qc = jc * nxc + ic;
        if (FUSED && ic >= 1 && ic <= nxc - 3 && jc >= 1 && jc <= K.L.npy - 2) return K.ld(S_U, qc) - K.ld(S_RU, qc);
        return K.ld(S_CU, qc);
    }
    __device__ __forceinline__ T v(int ic, int jc) const
    {
        const int nxc = K.L.npx, qc = jc * nxc + ic;
        if (FUSED && ic >= 1 && ic <= nxc - 2 && jc >= 1 && jc <= K.L.npy - 3) return K.ld(S_V, qc) - K.ld(S_RV, qc);
        return K.ld(S_CV, qc);
    }
    __device__ __forceinline__ T p(int ic, int jc) const
    {
        const int nxc = K.L.npx, qc = jc * nxc + ic;
        if (FUSED && ic >= 1 && ic <= nxc - 2 && jc >= 1 && jc <= K.L.npy - 2) {
            T c = K.ld(S_P, qc) - K.ld(S_RP, qc);
            if (F.g(S_SPU, 2 * jc * F.L.npx + 2 * ic) > 1.0e10) c = 0.0;
            return c;
        }
        return K.ld(S_CP, qc);
    }
    __device__ __forceinline__ T sc(int ic, int jc) const
    {
        const int nxc = K.L.npx, qc = jc * nxc + ic;
        if (FUSED && ic >= 1 && ic <= nxc - 2 && jc >= 1 && jc <= K.L.npy - 2) return K.ld(S_SC, qc) - K.ld(S_RSC, qc);
        return K.ld(S_C, qc);
    }
};

// Fine-cell gather of the reference's scatter-add prolongation (same additions in
// the same order as its sequential loops): fine interior cell (i, j).  FUSED: the
// corrections are formed here (ProlCorr), and the fine cell (2 ic, 2 jc) also writes
// coarse cell (ic, jc)'s corrections to the arrays, as cell_prol_corr would have.
template <class IO, bool FUSED = false>
__device__ __forceinline__ void cell_prol_apply_io(const IO &F, const IO &K, int i, int j, int parts = 15)
{
    using T = typename IO::T;
    const int nxf = F.L.npx, nyf = F.L.npy, nxc = K.L.npx, nyc = K.L.npy, q = j * nxf + i;
    const double f1 = 3. / 4., f2 = 1. / 4.;
    const ProlCorr<IO, FUSED> cr{F, K};
    if (FUSED && ((i | j) & 1) == 0) {
        const int ic = i / 2, jc = j / 2, qc = jc * nxc + ic;
        if (ic <= nxc - 3) K.st(S_CU, qc, cr.u(ic, jc));
        if (jc <= nyc - 3) K.st(S_CV, qc, cr.v(ic, jc));
        K.st(S_CP, qc, cr.p(ic, jc));
        K.st(S_C, qc, cr.sc(ic, jc));
    }
    // u faces, i in [1, nxf-3]: prolu :1782-1814
    if ((parts & 1) && i <= nxf - 3) {
        const bool up = (j & 1) == 0;                  // even row: corr1 of jc = j/2
        const int jc = up ? j / 2 : (j + 1) / 2;       // odd row: corr2 of jc = (j+1)/2
        const int jn = up ? jc + 1 : jc - 1;           // the other row of the pair
        T u = F.ld(S_U, q);
        if ((i & 1) == 0) {
            const int ic = i / 2;
            T corr = f1 * cr.u(ic, jc) + f2 * cr.u(ic, jn);
            if (F.g(S_SPU, 2 * jc * nxf + 2 * ic) > 1.0e10) corr = 0.0;
            u = u + corr;
        } else {
            const int ia = (i - 1) / 2, ib = (i + 1) / 2;
            if (ia >= 1) {
                T corr = f1 * cr.u(ia, jc) + f2 * cr.u(ia, jn);
                if (F.g(S_SPU, 2 * jc * nxf + 2 * ia) > 1.0e10) corr = 0.0;
                u = u + 0.5 * corr;
            }
            if (ib <= nxc - 3) {
                T corr = f1 * cr.u(ib, jc) + f2 * cr.u(ib, jn);
                if (F.g(S_SPU, 2 * jc * nxf + 2 * ib) > 1.0e10) corr = 0.0;
                u = u + 0.5 * corr;
            }
        }
        F.st(S_U, q, u);
    }
    // v faces, j in [1, nyf-3]: prolv :1861-1888
    if ((parts & 2) && j <= nyf - 3) {
        const bool right = (i & 1) == 0;               // even column: corr1 of ic = i/2
        const int ic = right ? i / 2 : (i + 1) / 2;
        const int in = right ? ic + 1 : ic - 1;        // the other column of the pair
        T v = F.ld(S_V, q);
        if ((j & 1) == 0) {
            const int jc = j / 2;
            T corr = f1 * cr.v(ic, jc) + f2 * cr.v(in, jc);
            if (F.g(S_SPV, 2 * jc * nxf + 2 * ic) > 1.0e10) corr = 0.0;
            v = v + corr;
        } else {
            const int ja = (j - 1) / 2, jb = (j + 1) / 2;
            if (ja >= 1) {
                T corr = f1 * cr.v(ic, ja) + f2 * cr.v(in, ja);
                if (F.g(S_SPV, 2 * ja * nxf + 2 * ic) > 1.0e10) corr = 0.0;
                v = v + 0.5 * corr;
            }
            if (jb <= nyc - 3) {
                T corr = f1 * cr.v(ic, jb) + f2 * cr.v(in, jb);
                if (F.g(S_SPV, 2 * jb * nxf + 2 * ic) > 1.0e10) corr = 0.0;
                v = v + 0.5 * corr;
            }
        }
        F.st(S_V, q, v);
    }
    // p and sc cells: prolp :1933-1958, prolsc :1999-2025
    {
        const double g1 = 9. / 16., g2 = 3. / 16., g3 = 3. / 16., g4 = 1. / 16.;
        const int ic = (i + 1) / 2, jc = (j + 1) / 2;
        const int in = (i & 1) == 0 ? ic + 1 : ic - 1;
        const int jn = (j & 1) == 0 ? jc + 1 : jc - 1;
        if (parts & 4)
            F.st(S_P, q, F.ld(S_P, q) + (g1 * cr.p(ic, jc) + g2 * cr.p(in, jc) + g3 * cr.p(ic, jn)
                                         + g4 * cr.p(in, jn)));
        if (parts & 8)
            F.st(S_SC, q, F.ld(S_SC, q) + (g1 * cr.sc(ic, jc) + g2 * cr.sc(in, jc) + g3 * cr.sc(ic, jn)
                                           + g4 * cr.sc(in, jn)));
    }
}
template <bool FUSED = false>
__device__ __forceinline__ void cell_prol_apply(const LevelDev &F, const LevelDev &K, int i, int j)
{
    cell_prol_apply_io<Prim, FUSED>(Prim{F}, Prim{K}, i, j);
}

// ---------------------------------------------------------- boundary lines
// outflow :1211-1228 at row j; `with_sc` also copies the scalar ghost
template <class IO>
__device__ __forceinline__ void row_outflow_io(const IO &io, int j, bool with_sc)
{
    const int q = j * io.L.npx + io.L.npx - 1;
    io.st(S_U, q - 1, io.ld(S_U, q - 2));
    io.st(S_V, q, io.ld(S_V, q - 1));
    io.st(S_P, q, io.ld(S_P, q - 1));
    if (with_sc) io.st(S_SC, q, io.ld(S_SC, q - 1));
}
__device__ __forceinline__ void row_outflow(const LevelDev &L, int j, bool with_sc) { row_outflow_io(Prim{L}, j, with_sc); }

// pbound x-periodic :1185-1195, row j in [1, npy-2]
template <class IO>
__device__ __forceinline__ void row_periodic_x_io(const IO &io, int j)
{
    const int q = j * io.L.npx, q1 = q + io.L.npx - 3;
    io.st(S_U, q, io.ld(S_U, q1)); io.st(S_U, q1 + 1, io.ld(S_U, q + 1));
    io.st(S_V, q, io.ld(S_V, q1)); io.st(S_V, q1 + 1, io.ld(S_V, q + 1));
}
__device__ __forceinline__ void row_periodic_x(const LevelDev &L, int j) { row_periodic_x_io(Prim{L}, j); }

// pbound y-periodic :1197-1208; sequential: later iterations read cells earlier
// iterations wrote (the reference's flat offset i + npy - 3), so one thread runs it.
template <class IO>
__device__ __forceinline__ void line_periodic_y_io(const IO &io)
{
    const int nx = io.L.npx, ny = io.L.npy;
    for (int i = 1; i < nx - 1; ++i) {
        const int q = i, q1 = q + ny - 3;
        io.st(S_U, q, io.ld(S_U, q1)); io.st(S_U, q1 + nx, io.ld(S_U, q + nx));
        io.st(S_V, q, io.ld(S_V, q1)); io.st(S_V, q1 + nx, io.ld(S_V, q + nx));
    }
}
__device__ __forceinline__ void line_periodic_y(const LevelDev &L) { line_periodic_y_io(Prim{L}); }

}  // namespace mg
