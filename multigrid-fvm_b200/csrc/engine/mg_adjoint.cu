// mg_adjoint.cu — the taped V-cycle and its transpose (see mg_adjoint.cuh).
#include <climits>

#include "mg_adjoint.cuh"

namespace mg {
namespace {

// ------------------------------------------------------------------ phases
struct Box { int i0, j0, wi, wj; };

__host__ __device__ inline Box box_eq(int npx, int npy, int e)
{
    if (e == EQ_U) return {1, 1, npx - 3, npy - 2};
    if (e == EQ_V) return {1, 1, npx - 2, npy - 3};
    return {1, 1, npx - 2, npy - 2};
}
__host__ __device__ inline int res_eq(int which) { return which == 0 ? EQ_U : which == 1 ? EQ_V : EQ_SC; }
__host__ __device__ inline int field_of(int e) { return e == EQ_U ? S_U : e == EQ_V ? S_V : e == EQ_PP ? S_PP : S_SC; }
__host__ __device__ inline int tmp_of(int e) { return e == EQ_V ? S_TMP1 : e == EQ_SC ? S_TMP2 : S_TMP0; }
__host__ __device__ inline unsigned long long bit(int s) { return 1ULL << s; }
__host__ __device__ inline unsigned long long coef_bits(int e)
{
    unsigned long long m = 0;
    for (int k = 0; k < NCOEF; ++k) m |= bit(co_slot(e, k));
    return m;
}

// The level a phase writes, and the slots it overwrites there.
__host__ __device__ inline int write_level(const Phase &P)
{
    return (P.kind == P_RESTV || P.kind == P_RESTRICT || P.kind == P_PROL_CORR) ? P.ig + 1 : P.ig;
}
__host__ __device__ inline unsigned long long write_mask(const Phase &P)
{
    switch (P.kind) {
    case P_ASM_U: return coef_bits(EQ_U) | bit(S_APU);
    case P_ASM_V: return coef_bits(EQ_V) | bit(S_APV);
    case P_ASM_SC: return coef_bits(EQ_SC);
    case P_SC_OUTFLOW: return bit(S_SC);
    case P_GS: return bit(field_of(P.a));
    case P_JAC_RING: return bit(tmp_of(P.a));
    case P_JAC_SWEEP: return bit(P.b == 0 ? tmp_of(P.a) : field_of(P.a));
    case P_JAC_COPY: return bit(field_of(P.a));
    case P_MASS_COEFP:
        return (P.a & MC_COEF ? bit(S_PP) | (coef_bits(EQ_PP) & ~bit(co_slot(EQ_PP, CK_SU))) : 0ULL) |
               (P.a & MC_SU ? bit(co_slot(EQ_PP, CK_SU)) : 0ULL);
    case P_UPDATE: return (P.a & 1 ? bit(S_U) : 0ULL) | (P.a & 2 ? bit(S_V) : 0ULL) | (P.a & 4 ? bit(S_P) : 0ULL);
    case P_PFIX: case P_PFIX_SCATTER: return bit(S_P);
    case P_PFIX_GATHER: return bit(PB_BIT);
    case P_OUTFLOW: return bit(S_U) | bit(S_V) | bit(S_P) | (P.b ? bit(S_SC) : 0ULL);
    case P_RESTV:
        return (P.a & 1 ? bit(S_U) | bit(S_RU) : 0ULL) | (P.a & 2 ? bit(S_V) | bit(S_RV) : 0ULL) |
               (P.a & 4 ? bit(S_P) | bit(S_RP) : 0ULL) | (P.a & 8 ? bit(S_SC) | bit(S_RSC) : 0ULL);
    case P_FINE_RES: return bit(tmp_of(res_eq(P.a)));
    case P_RESTRICT: return bit(P.a == 0 ? S_RESU : P.a == 1 ? S_RESV : S_RESSC);
    case P_PROL_CORR:
        return (P.a & 1 ? bit(S_CU) : 0ULL) | (P.a & 2 ? bit(S_CV) : 0ULL) | (P.a & 4 ? bit(S_CP) : 0ULL) |
               (P.a & 8 ? bit(S_C) : 0ULL);
    case P_PROL_APPLY:
        return (P.a & 1 ? bit(S_U) : 0ULL) | (P.a & 2 ? bit(S_V) : 0ULL) | (P.a & 4 ? bit(S_P) : 0ULL) |
               (P.a & 8 ? bit(S_SC) : 0ULL);
    default: return 0;
    }
}

// The cells (i, j) a phase visits: a box of the level it runs over (for the pressure
// copy: i = copy index; for outflow: j = row), with the half-sweep's colour filter and
// the Jacobi ring filter applied by the caller.
__host__ __device__ inline Box phase_box(const Phase &P, const LevelDev &F, const LevelDev *K)
{
    const int nx = F.npx, ny = F.npy;
    switch (P.kind) {
    case P_ASM_U: return box_eq(nx, ny, EQ_U);
    case P_ASM_V: return box_eq(nx, ny, EQ_V);
    case P_ASM_SC: case P_MASS_COEFP: case P_UPDATE: case P_PROL_APPLY: return {1, 1, nx - 2, ny - 2};
    case P_SC_OUTFLOW: return {nx - 1, 0, 1, ny};
    case P_GS: case P_JAC_SWEEP: case P_JAC_COPY: return box_eq(nx, ny, P.a);
    case P_JAC_RING: {
        const Box d = box_eq(nx, ny, P.a);
        return {d.i0 - 1, d.j0 - 1, d.wi + 2, d.wj + 2};
    }
    case P_PFIX: case P_PFIX_GATHER: case P_PFIX_SCATTER: return {0, 0, F.ncopy, 1};
    case P_OUTFLOW: return {0, 0, 1, ny};
    case P_FINE_RES: return box_eq(nx, ny, res_eq(P.a));
    case P_RESTV: case P_PROL_CORR: return {1, 1, K->npx - 2, K->npy - 2};
    case P_RESTRICT: return box_eq(K->npx, K->npy, res_eq(P.a));
    default: return {0, 0, 0, 0};
    }
}

// One cell of a phase through the access type of the case view X (X::io(level)).
template <class X>
__device__ __forceinline__ void phase_cell(const X &x, const Phase &P, int i, int j)
{
    const CaseDev &C = x.C;
    const auto F = x.io(P.ig);
    using IO = typename std::remove_cv<decltype(F)>::type;
    const int nx = F.L.npx, q = j * nx + i;
    switch (P.kind) {
    case P_ASM_U: cell_mom_u(F, C, FluxLiveT<IO>{F}, i, j); break;
    case P_ASM_V: cell_mom_v(F, C, FluxLiveT<IO>{F}, i, j); break;
    case P_ASM_SC: cell_sc(F, C, FluxLiveT<IO>{F}, i, j); break;
    case P_SC_OUTFLOW: F.st(S_SC, q, F.ld(S_SC, q - 1)); break;
    case P_GS: cell_gs_io(F, P.a, field_of(P.a), q); break;
    case P_JAC_RING: F.st(tmp_of(P.a), q, F.ld(field_of(P.a), q)); break;
    case P_JAC_SWEEP: {
        const int phi = field_of(P.a), tmp = tmp_of(P.a);
        cell_jacobi_io(F, P.a, P.b == 0 ? phi : tmp, P.b == 0 ? tmp : phi, q);
        break;
    }
    case P_JAC_COPY: F.st(field_of(P.a), q, F.ld(tmp_of(P.a), q)); break;
    case P_MASS_COEFP: cell_mass_coefp_io(F, C, i, j, false, P.a); break;
    case P_UPDATE: cell_update_io(F, C, q, P.a); break;
    case P_PFIX: F.st(S_P, F.L.pdst[i], F.ld(S_P, F.L.psrc[i])); break;
    case P_PFIX_GATHER: F.set_pb(i, F.ld(S_P, F.L.psrc[i])); break;
    case P_PFIX_SCATTER: F.st(S_P, F.L.pdst[i], F.pb(i)); break;
    case P_OUTFLOW: row_outflow_io(F, j, P.b != 0); break;
    case P_RESTV: cell_restv_io(F, x.io(P.ig + 1), i, j, P.a); break;
    case P_FINE_RES: cell_fine_residuals_io(F, C, i, j, P.a); break;
    case P_RESTRICT: cell_restrict_io(F, x.io(P.ig + 1), C, i, j, P.a); break;
    case P_PROL_CORR: cell_prol_corr_io(F, x.io(P.ig + 1), i, j, P.a); break;
    case P_PROL_APPLY: cell_prol_apply_io<IO, false>(F, x.io(P.ig + 1), i, j, P.a); break;
    default: break;
    }
}

// A case runs on a cluster of CTAs (the kernel's cluster rank picks a CTA's share of
// every phase); worker index and count over the cluster's threads.
__device__ __forceinline__ unsigned cl_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cl_size()
{
    unsigned n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return n;
}
__device__ __forceinline__ int wk_id() { return (int)(cl_rank() * blockDim.x + threadIdx.x); }
__device__ __forceinline__ int wk_n() { return (int)(cl_size() * blockDim.x); }
// Every thread of the case's cluster arrives; memory written before (global included)
// is visible to every thread of the cluster after.
__device__ __forceinline__ void case_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Every cell of a phase, spread over the case's cluster.
template <class Fn>
__device__ __forceinline__ void phase_cells(const CaseDev &C, const Phase &P, Fn f)
{
    const LevelDev &L = C.lv[P.ig];
    const LevelDev *K = P.ig + 1 < C.ngrid ? &C.lv[P.ig + 1] : nullptr;
    const Box d = phase_box(P, L, K);
    if (d.wi <= 0 || d.wj <= 0) return;
    if (P.kind == P_GS) {
        // cells of colour b: (i + j) & 1 == b
        const int wr = (d.wi + 1) >> 1, n = wr * d.wj;
        for (int t = wk_id(); t < n; t += wk_n()) {
            const int j = d.j0 + t / wr;
            const int i = d.i0 + (((d.i0 + j) & 1) != P.b ? 1 : 0) + 2 * (t % wr);
            if (i <= d.i0 + d.wi - 1) f(i, j);
        }
        return;
    }
    const int n = d.wi * d.wj;
    for (int t = wk_id(); t < n; t += wk_n()) {
        const int i = d.i0 + t % d.wi, j = d.j0 + t / d.wi;
        if (P.kind == P_JAC_RING && i != d.i0 && i != d.i0 + d.wi - 1 && j != d.j0 && j != d.j0 + d.wj - 1) continue;
        f(i, j);
    }
}

// ------------------------------------------------------- forward (taped)
// Plain FP64 access (the bits of the engine's kernels) that checks every store against
// the phase's write mask: a store outside it would escape the tape, so the case is
// flagged and the call fails.
struct Rec {
    using T = double;
    const LevelDev &L;
    unsigned long long mask;   // the phase's mask if this is its written level, else 0
    int *bad;
    __device__ __forceinline__ double ld(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ void st(int s, int q, double v) const
    {
        if (!((mask >> s) & 1ULL)) *bad = 1;
        L.f[s][q] = v;
    }
    __device__ __forceinline__ double g(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ double amu() const { return L.amu; }
    __device__ __forceinline__ double amusc() const { return L.amusc; }
    __device__ __forceinline__ double pb(int k) const { return L.pbuf[k]; }
    __device__ __forceinline__ void set_pb(int k, double v) const
    {
        if (!((mask >> PB_BIT) & 1ULL)) *bad = 1;
        L.pbuf[k] = v;
    }
};
struct RecCase {
    const CaseDev &C;
    int wlev;
    unsigned long long mask;
    int *bad;
    __device__ __forceinline__ Rec io(int ig) const { return Rec{C.lv[ig], ig == wlev ? mask : 0ULL, bad}; }
};

// Copy the arrays phase P overwrites between the level and the tape (save: to the tape).
// A half-sweep overwrites the cells of its colour only: those alone are kept, in the
// order phase_cells visits them.
__device__ void tape_copy(const CaseDev &C, const CaseAdj &A, const Phase &P, bool save)
{
    const LevelDev &L = C.lv[write_level(P)];
    double *t = A.tape + P.off;
    if (P.kind == P_GS) {
        const Box d = box_eq(L.npx, L.npy, P.a);
        double *a = L.f[field_of(P.a)];
        const int wr = (d.wi + 1) >> 1, n = wr * d.wj;
        for (int k = wk_id(); k < n; k += wk_n()) {
            const int j = d.j0 + k / wr;
            const int i = d.i0 + (((d.i0 + j) & 1) != P.b ? 1 : 0) + 2 * (k % wr);
            if (i > d.i0 + d.wi - 1) continue;
            if (save) t[k] = a[j * L.npx + i];
            else a[j * L.npx + i] = t[k];
        }
        return;
    }
    const long long n = (long long)L.npx * L.npy;
    const unsigned long long m = write_mask(P);
    for (int s = 0; s < NSLOTS; ++s) {
        if (!((m >> s) & 1ULL)) continue;
        double *a = L.f[s];
        if (save)
            for (long long k = wk_id(); k < n; k += wk_n()) t[k] = a[k];
        else
            for (long long k = wk_id(); k < n; k += wk_n()) a[k] = t[k];
        t += n;
    }
    if ((m >> PB_BIT) & 1ULL) {
        if (save)
            for (int k = wk_id(); k < L.ncopy; k += wk_n()) t[k] = L.pbuf[k];
        else
            for (int k = wk_id(); k < L.ncopy; k += wk_n()) L.pbuf[k] = t[k];
    }
}

// ------------------------------------------------------------- reverse
constexpr int MAXW = 8;   // most values one cell of a phase writes (restv: 8)
enum { KS_NONE = INT_MIN, KS_AMU = -1, KS_AMUSC = -2, KS_PB = -3 };

// The state of one cell's evaluation: collect (mode 0) or probe read k (mode 1).  The
// adjoints of the outputs sit in named fields, reached only at constant offsets, so
// that after inlining the whole state lives in registers and the read and write
// counters fold to constants at every access site.
struct Probe {
    int mode, k, nr, nw, ks, kq, klev, ovf;
    double acc;
    double y0, y1, y2, y3, y4, y5, y6, y7;
    __device__ __forceinline__ double yb(int w) const
    {
        switch (w) {
        case 0: return y0; case 1: return y1; case 2: return y2; case 3: return y3;
        case 4: return y4; case 5: return y5; case 6: return y6; default: return y7;
        }
    }
    __device__ __forceinline__ void set_yb(int w, double v)
    {
        switch (w) {
        case 0: y0 = v; break; case 1: y1 = v; break; case 2: y2 = v; break; case 3: y3 = v; break;
        case 4: y4 = v; break; case 5: y5 = v; break; case 6: y6 = v; break; default: y7 = v; break;
        }
    }
};
static_assert(MAXW == 8, "Probe holds MAXW output adjoints");

// Dual-number access whose reads are numbered: in a probe, read k carries derivative
// 1 and every other read 0, so each value written carries d(value)/d(read k); the
// collect pass takes (and clears) the adjoints of the values written.
struct AdjIO {
    using T = Dual;
    const LevelDev &L;
    const LevelTan &B;
    Probe *P;
    int lev;
    __device__ __forceinline__ Dual rd(double v, int s, int q) const
    {
        const int r = P->nr++;
        if (P->mode == 1 && r == P->k) {
            P->ks = s;
            P->kq = q;
            P->klev = lev;
            return {v, 1.0};
        }
        return {v, 0.0};
    }
    __device__ __forceinline__ void wr(double *b, const Dual &x) const
    {
        const int w = P->nw++;
        if (w >= MAXW) {
            P->ovf = 1;
            return;
        }
        if (P->mode == 0) {
            P->set_yb(w, *b);
            *b = 0.0;
        } else {
            P->acc += P->yb(w) * x.d;
        }
    }
    __device__ __forceinline__ Dual ld(int s, int q) const { return rd(L.f[s][q], s, q); }
    __device__ __forceinline__ void st(int s, int q, const Dual &x) const { wr(B.t[s] + q, x); }
    __device__ __forceinline__ double g(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ Dual amu() const { return rd(L.amu, KS_AMU, 0); }
    __device__ __forceinline__ Dual amusc() const { return rd(L.amusc, KS_AMUSC, 0); }
    __device__ __forceinline__ Dual pb(int k) const { return rd(L.pbuf[k], KS_PB, k); }
    __device__ __forceinline__ void set_pb(int k, const Dual &x) const { wr(B.pbuf_t + k, x); }
};
struct AdjCase {
    const CaseDev &C;
    const CaseTan &B;
    Probe *P;
    __device__ __forceinline__ AdjIO io(int ig) const { return AdjIO{C.lv[ig], B.lv[ig], P, ig}; }
};

// Adjoints of amu and amusc gathered by one thread during one phase: a phase reads the
// parameters of its own level (f) and of the level below (k) at most.
struct ParAcc {
    double amu_f, amusc_f, amu_k, amusc_k;
};

// The transpose of one cell of phase P: adjoints of its reads += adjoint(out) *
// d(out)/d(read); adjoints of its outputs cleared.  amu/amusc go to the thread's
// accumulators of the phase.
__device__ __forceinline__ void adj_cell(const CaseDev &C, const CaseTan &B, const Phase &P, int i, int j,
                                         ParAcc &pa, int *bad)
{
    Probe S;
    S.mode = 0;
    S.nr = S.nw = 0;
    S.ovf = 0;
    const AdjCase X{C, B, &S};
    phase_cell(X, P, i, j);
    if (S.ovf) {
        *bad = 1;
        return;
    }
    const int K = S.nr, W = S.nw;
    bool any = false;
    for (int w = 0; w < W; ++w) any |= S.yb(w) != 0.0;
    if (!any) return;
    for (int k = 0; k < K; ++k) {
        S.mode = 1;
        S.k = k;
        S.nr = S.nw = 0;
        S.acc = 0.0;
        S.ks = KS_NONE;
        phase_cell(X, P, i, j);
        if (S.acc == 0.0) continue;
        if (S.ks >= 0) {
            atomicAdd(B.lv[S.klev].t[S.ks] + S.kq, S.acc);
        } else if (S.ks == KS_AMU) {
            if (S.klev == P.ig) pa.amu_f += S.acc;
            else pa.amu_k += S.acc;
        } else if (S.ks == KS_AMUSC) {
            if (S.klev == P.ig) pa.amusc_f += S.acc;
            else pa.amusc_k += S.acc;
        } else if (S.ks == KS_PB) {
            atomicAdd(B.lv[S.klev].pbuf_t + S.kq, S.acc);
        }
    }
}

// The cells of a half-sweep phase with their index in its colour-only tape.
template <class Fn>
__device__ __forceinline__ void gs_cells(const LevelDev &L, const Phase &P, Fn f)
{
    const Box d = box_eq(L.npx, L.npy, P.a);
    if (d.wi <= 0 || d.wj <= 0) return;
    const int wr = (d.wi + 1) >> 1, n = wr * d.wj;
    for (int t = wk_id(); t < n; t += wk_n()) {
        const int j = d.j0 + t / wr;
        const int i = d.i0 + (((d.i0 + j) & 1) != P.b ? 1 : 0) + 2 * (t % wr);
        if (i <= d.i0 + d.wi - 1) f(i, j, t);
    }
}

// A half-sweep, taped, in one pass: each cell's old value to the tape, then its update
// (its neighbours are of the other colour, which the half-sweep does not write).
__device__ __forceinline__ void fwd_gs_cell(const LevelDev &L, int e, int i, int j, double *tape, int t)
{
    const int q = j * L.npx + i;
    double *f = L.f[field_of(e)];
    tape[t] = f[q];
    cell_gs_io(Prim{L}, e, field_of(e), q);
}

// The transpose of one red-black half-sweep cell, phi_c = (sum a_nb phi_nb + su) / ap
// (gs_value), in closed form: d/da_nb = phi_nb / ap, d/dphi_nb = a_nb / ap, d/dsu =
// 1 / ap, d/dap = -phi_c / ap, the partial derivatives the dual arithmetic of adj_cell
// forms, here with the adjoint divided by ap once (the same numbers to rounding).  The
// cell's new value phi_c is read from the field before the tape restores the old one
// (its neighbours are unchanged by the half-sweep).  The cell's coefficients are read
// by no other cell of the half-sweep, so their adjoints take plain additions; the
// neighbours' take atomics.
__device__ __forceinline__ void adj_gs_cell(const LevelDev &L, const LevelTan &B, int e, int i, int j,
                                            const double *tape, int t)
{
    const int nx = L.npx, q = j * nx + i, phi = field_of(e);
    double *f = L.f[phi];
    const double val = f[q];
    f[q] = tape[t];
    double *yp = B.t[phi] + q;
    const double yb = *yp;
    *yp = 0.0;
    if (yb == 0.0) return;
    const double aw = L.f[co_slot(e, CK_AW)][q], ae = L.f[co_slot(e, CK_AE)][q], as = L.f[co_slot(e, CK_AS)][q],
                 an = L.f[co_slot(e, CK_AN)][q], ap = L.f[co_slot(e, CK_AP)][q];
    const double pw = f[q - 1], pe = f[q + 1], ps = f[q - nx], pn = f[q + nx];
    const double ya = yb / ap;
    B.t[co_slot(e, CK_AW)][q] += ya * pw;
    B.t[co_slot(e, CK_AE)][q] += ya * pe;
    B.t[co_slot(e, CK_AS)][q] += ya * ps;
    B.t[co_slot(e, CK_AN)][q] += ya * pn;
    B.t[co_slot(e, CK_AP)][q] += -(ya * val);
    B.t[co_slot(e, CK_SU)][q] += ya;
    double *b = B.t[phi];
    atomicAdd(b + q - 1, ya * aw);
    atomicAdd(b + q + 1, ya * ae);
    atomicAdd(b + q - nx, ya * as);
    atomicAdd(b + q + nx, ya * an);
}

// ------------------------------- closed-form transposes: the assembly family
// coef_u, coef_v and coef_sc (the hybrid-scheme coefficients from the live fluxes) and
// their users — the assemblies (coefu + umom, coefv + vmom, coefsc + scalar), the
// fine residuals and the FAS defects — transposed by hand with the partial derivatives
// the dual arithmetic forms (so the same numbers as the probes, to rounding): at a
// non-smooth point max(|c|, d) takes the mean of both sides, |c| at 0 the derivative 0.
// The forward values are recomputed with the engine's own routines (Prim).

// adjoints of a level's arrays: take (and clear) an output's, add to an input's
struct Bars {
    const LevelTan &B;
    __device__ __forceinline__ double take(int s, int q) const
    {
        double *b = B.t[s] + q;
        const double y = *b;
        *b = 0.0;
        return y;
    }
    __device__ __forceinline__ void add(int s, int q, double v) const
    {
        if (v != 0.0) atomicAdd(B.t[s] + q, v);
    }
};

// d/dc and d/dd of max(|c|, d) + sg c (sg = +1: hyb_p, -1: hyb_m)
__device__ __forceinline__ void hyb_partials(double c, double d, double sg, double &dc, double &dd)
{
    const double ac = fabs(c), sc = c > 0.0 ? 1.0 : c < 0.0 ? -1.0 : 0.0;
    if (ac > d) { dc = sc; dd = 0.0; }
    else if (d > ac) { dc = 0.0; dd = 1.0; }
    else { dc = 0.5 * sc; dd = 0.5; }
    dc += sg;
}

// the live fluxes' inputs: cx(q) = 0.5 u(q) Ax(q), cy(q) = 0.5 v(q) Ay(q)
__device__ __forceinline__ void flux_x_adj(const LevelDev &L, const Bars &b, int q, double bc)
{
    b.add(S_U, q, (0.5 * bc) * L.f[S_AREAX][q]);
}
__device__ __forceinline__ void flux_y_adj(const LevelDev &L, const Bars &b, int q, double bc)
{
    b.add(S_V, q, (0.5 * bc) * L.f[S_AREAY][q]);
}

// Transpose of coef_u at u face (i, j): output adjoints (aw .. ap) -> u, v adjoints;
// returns the adjoint of amu.
__device__ double coef_u_adj(const LevelDev &L, const Bars &b, int i, int j, double baw, double bae, double bas,
                             double ban, double bap)
{
    const int nx = L.npx, q = j * nx + i, s = q - nx, top = L.npy - 2;
    const FluxLive fl(L);
    const double cq = fl.x(q);
    const double cxm = 0.5 * (cq + fl.x(q - 1)), cxp = 0.5 * (cq + fl.x(q + 1));
    const double cym = 0.5 * (fl.y(s) + fl.y(s + 1)), cyp = 0.5 * (fl.y(q) + fl.y(q + 1));
    const double gx = L.f[S_AREAX][q] / L.dx, gy = L.f[S_AREAY][q] / L.dy;
    const double dxm = L.amu * gx, dym = L.amu * gy;
    double bamu = 0.0;
    // the wall-shear additions to an / as and ap (rows npy-2 and 1)
    if (j == 1) bamu += (bas + bap) * (L.f[S_AREAY][top * nx + i] / L.dy);
    if (j == top) bamu += (ban + bap) * gy;
    baw += bap; bae += bap; bas += bap; ban += bap;      // ap = aw + ae + as + an
    double dc, dd, bdx = 0.0, bdy = 0.0;
    hyb_partials(cxm, dxm, 1.0, dc, dd);  const double bcxm = baw * dc; bdx += baw * dd;
    hyb_partials(cxp, dxm, -1.0, dc, dd); const double bcxp = bae * dc; bdx += bae * dd;
    hyb_partials(cym, dym, 1.0, dc, dd);  const double bcym = bas * dc; bdy += bas * dd;
    hyb_partials(cyp, dym, -1.0, dc, dd); const double bcyp = ban * dc; bdy += ban * dd;
    bamu += bdx * gx + bdy * gy;
    flux_x_adj(L, b, q, 0.5 * bcxm + 0.5 * bcxp);
    flux_x_adj(L, b, q - 1, 0.5 * bcxm);
    flux_x_adj(L, b, q + 1, 0.5 * bcxp);
    flux_y_adj(L, b, s, 0.5 * bcym);
    flux_y_adj(L, b, s + 1, 0.5 * bcym);
    flux_y_adj(L, b, q, 0.5 * bcyp);
    flux_y_adj(L, b, q + 1, 0.5 * bcyp);
    return bamu;
}

// Transpose of coef_v at v face (i, j); returns the adjoint of amu.
__device__ double coef_v_adj(const LevelDev &L, const Bars &b, int i, int j, double baw, double bae, double bas,
                             double ban, double bap)
{
    const int nx = L.npx, q = j * nx + i, n = q + nx, s = q - nx, rgt = nx - 2;
    const FluxLive fl(L);
    const double cxm = 0.5 * (fl.x(q - 1) + fl.x(n - 1)), cxp = 0.5 * (fl.x(q) + fl.x(n));
    const double cyq = fl.y(q);
    const double cym = 0.5 * (cyq + fl.y(s)), cyp = 0.5 * (cyq + fl.y(n));
    const double gx = L.f[S_AREAX][q] / L.dx, gy = L.f[S_AREAY][q] / L.dy;
    const double dx_ = L.amu * gx, dy_ = L.amu * gy;
    double bamu = 0.0;
    // the side-wall additions to aw / ae and ap (columns 1 and npx-2)
    if (i == 1) bamu += (baw + bap) * (L.f[S_AREAY][j * nx + rgt] / L.dy);
    if (i == rgt) bamu += (bae + bap) * gy;
    baw += bap; bae += bap; bas += bap; ban += bap;
    double dc, dd, bdx = 0.0, bdy = 0.0;
    hyb_partials(cxm, dx_, 1.0, dc, dd);  const double bcxm = baw * dc; bdx += baw * dd;
    hyb_partials(cxp, dx_, -1.0, dc, dd); const double bcxp = bae * dc; bdx += bae * dd;
    hyb_partials(cym, dy_, 1.0, dc, dd);  const double bcym = bas * dc; bdy += bas * dd;
    hyb_partials(cyp, dy_, -1.0, dc, dd); const double bcyp = ban * dc; bdy += ban * dd;
    bamu += bdx * gx + bdy * gy;
    flux_x_adj(L, b, q - 1, 0.5 * bcxm);
    flux_x_adj(L, b, n - 1, 0.5 * bcxm);
    flux_x_adj(L, b, q, 0.5 * bcxp);
    flux_x_adj(L, b, n, 0.5 * bcxp);
    flux_y_adj(L, b, q, 0.5 * bcym + 0.5 * bcyp);
    flux_y_adj(L, b, s, 0.5 * bcym);
    flux_y_adj(L, b, n, 0.5 * bcyp);
    return bamu;
}

// Transpose of coef_sc at cell (i, j), obstacle-face additions included; returns the
// adjoint of amusc.
__device__ double coef_sc_adj(const LevelDev &L, const Bars &b, int i, int j, double baw, double bae, double bas,
                              double ban, double bap)
{
    const int nx = L.npx, q = j * nx + i, s = q - nx;
    const FluxLive fl(L);
    const double *AX = L.f[S_AREAX], *AY = L.f[S_AREAY];
    const double gxm = AX[q - 1] / L.dx, gym = AY[s] / L.dy, gxp = AX[q] / L.dx, gyp = AY[q] / L.dy;
    const double a = L.amusc;
    const double dxm = a * gxm, dym = a * gym, dxp = a * gxp, dyp = a * gyp;
    double bamusc = 0.0;
    if (L.seq) {
        const unsigned code = L.seq[q];
        const int cnt = (int)(code >> 28);
        for (int t = 0; t < cnt; ++t) {
            const int d = (int)((code >> (2 * t)) & 3u);
            if (d == 0) bamusc += (bae + bap) * (AX[q + 1] / L.dx);
            else if (d == 1) bamusc += (baw + bap) * (AX[q - 1] / L.dx);
            else if (d == 2) bamusc += (ban + bap) * (AY[q + nx] / L.dy);
            else bamusc += (bas + bap) * (AY[q - nx] / L.dy);
        }
    }
    baw += bap; bae += bap; bas += bap; ban += bap;
    double dc, dd;
    hyb_partials(fl.x(q - 1), dxm, 1.0, dc, dd); const double bw = baw * dc; bamusc += baw * dd * gxm;
    hyb_partials(fl.x(q), dxp, -1.0, dc, dd);    const double be = bae * dc; bamusc += bae * dd * gxp;
    hyb_partials(fl.y(s), dym, 1.0, dc, dd);     const double bs = bas * dc; bamusc += bas * dd * gym;
    hyb_partials(fl.y(q), dyp, -1.0, dc, dd);    const double bn = ban * dc; bamusc += ban * dd * gyp;
    flux_x_adj(L, b, q - 1, bw);
    flux_x_adj(L, b, q, be);
    flux_y_adj(L, b, s, bs);
    flux_y_adj(L, b, q, bn);
    return bamusc;
}

// Transposes of the assemblies at one cell (P_ASM_U / V / SC); the parameter adjoint
// goes to `pa`.
__device__ void asm_u_adj(const CaseDev &C, const LevelDev &L, const Bars &b, int i, int j, ParAcc &pa)
{
    const int q = j * L.npx + i;
    const double baw = b.take(co_slot(EQ_U, CK_AW), q), bae = b.take(co_slot(EQ_U, CK_AE), q),
                 bas = b.take(co_slot(EQ_U, CK_AS), q), ban = b.take(co_slot(EQ_U, CK_AN), q);
    const double bapo = b.take(co_slot(EQ_U, CK_AP), q) + b.take(S_APU, q), bsu = b.take(co_slot(EQ_U, CK_SU), q);
    if (baw == 0.0 && bae == 0.0 && bas == 0.0 && ban == 0.0 && bapo == 0.0 && bsu == 0.0) return;
    const Coef k = coef_u(Prim{L}, FluxLive(L), i, j);
    const double ax = L.f[S_AREAX][q], rm = C.relxm, rm1 = 1.0 - C.relxm;
    const double apr = k.ap / rm;
    // su = ax (p_P - p_E) + rm1 (ap / rm) u + resu + ...; ap_out = ap / rm + spu
    b.add(S_P, q, bsu * ax);
    b.add(S_P, q + 1, -(bsu * ax));
    b.add(S_U, q, bsu * (rm1 * apr));
    b.add(S_RESU, q, bsu);
    const double bap = (bapo + bsu * (rm1 * L.f[S_U][q])) / rm;
    pa.amu_f += coef_u_adj(L, b, i, j, baw, bae, bas, ban, bap);
}
__device__ void asm_v_adj(const CaseDev &C, const LevelDev &L, const Bars &b, int i, int j, ParAcc &pa)
{
    const int q = j * L.npx + i;
    const double baw = b.take(co_slot(EQ_V, CK_AW), q), bae = b.take(co_slot(EQ_V, CK_AE), q),
                 bas = b.take(co_slot(EQ_V, CK_AS), q), ban = b.take(co_slot(EQ_V, CK_AN), q);
    const double bapo = b.take(co_slot(EQ_V, CK_AP), q) + b.take(S_APV, q), bsu = b.take(co_slot(EQ_V, CK_SU), q);
    if (baw == 0.0 && bae == 0.0 && bas == 0.0 && ban == 0.0 && bapo == 0.0 && bsu == 0.0) return;
    const Coef k = coef_v(Prim{L}, FluxLive(L), i, j);
    const double ay = L.f[S_AREAY][q], rm = C.relxm, rm1 = 1.0 - C.relxm;
    const double apr = k.ap / rm;
    b.add(S_P, q, bsu * ay);
    b.add(S_P, q + L.npx, -(bsu * ay));
    b.add(S_V, q, bsu * (rm1 * apr));
    b.add(S_RESV, q, bsu);
    const double bap = (bapo + bsu * (rm1 * L.f[S_V][q])) / rm;
    pa.amu_f += coef_v_adj(L, b, i, j, baw, bae, bas, ban, bap);
}
__device__ void asm_sc_adj(const LevelDev &L, const Bars &b, int i, int j, ParAcc &pa)
{
    const int q = j * L.npx + i;
    const double baw = b.take(co_slot(EQ_SC, CK_AW), q), bae = b.take(co_slot(EQ_SC, CK_AE), q),
                 bas = b.take(co_slot(EQ_SC, CK_AS), q), ban = b.take(co_slot(EQ_SC, CK_AN), q);
    const double bap = b.take(co_slot(EQ_SC, CK_AP), q), bsu = b.take(co_slot(EQ_SC, CK_SU), q);
    if (baw == 0.0 && bae == 0.0 && bas == 0.0 && ban == 0.0 && bap == 0.0 && bsu == 0.0) return;
    b.add(S_RESSC, q, bsu);                          // su = spsc sc_obs + ressc; ap += spsc
    pa.amusc_f += coef_sc_adj(L, b, i, j, baw, bae, bas, ban, bap);
}

// Transposes of the residuals resid_u / resid_v / resid_sc at (i, j) of level L given
// the adjoint br of the residual; `fine`: the fine-level form (with the defect term
// and the zero where the face area is 0).  Returns the parameter adjoint (amu, or
// amusc for the scalar).
__device__ double resid_u_adj(const LevelDev &L, const Bars &b, int i, int j, bool fine, double br)
{
    const int nx = L.npx, q = j * nx + i;
    const double ax = L.f[S_AREAX][q];
    if (br == 0.0 || (fine && ax == 0.0)) return 0.0;
    const Coef k = coef_u(Prim{L}, FluxLive(L), i, j);
    const double *u = L.f[S_U];
    b.add(S_U, q - 1, br * k.aw);
    b.add(S_U, q + 1, br * k.ae);
    b.add(S_U, q - nx, br * k.as);
    b.add(S_U, q + nx, br * k.an);
    b.add(S_U, q, -(br * k.ap));
    b.add(S_P, q, br * ax);
    b.add(S_P, q + 1, -(br * ax));
    if (fine) b.add(S_RESU, q, br);
    return coef_u_adj(L, b, i, j, br * u[q - 1], br * u[q + 1], br * u[q - nx], br * u[q + nx], -(br * u[q]));
}
__device__ double resid_v_adj(const LevelDev &L, const Bars &b, int i, int j, bool fine, double br)
{
    const int nx = L.npx, q = j * nx + i;
    const double ay = L.f[S_AREAY][q];
    if (br == 0.0 || (fine && ay == 0.0)) return 0.0;
    const Coef k = coef_v(Prim{L}, FluxLive(L), i, j);
    const double *v = L.f[S_V];
    b.add(S_V, q - 1, br * k.aw);
    b.add(S_V, q + 1, br * k.ae);
    b.add(S_V, q - nx, br * k.as);
    b.add(S_V, q + nx, br * k.an);
    b.add(S_V, q, -(br * k.ap));
    b.add(S_P, q, br * ay);
    b.add(S_P, q + nx, -(br * ay));
    if (fine) b.add(S_RESV, q, br);
    return coef_v_adj(L, b, i, j, br * v[q - 1], br * v[q + 1], br * v[q - nx], br * v[q + nx], -(br * v[q]));
}
__device__ double resid_sc_adj(const LevelDev &L, const Bars &b, int i, int j, bool fine, double br)
{
    const int nx = L.npx, q = j * nx + i;
    if (br == 0.0) return 0.0;
    const Coef k = coef_sc(Prim{L}, FluxLive(L), i, j);
    const double *c = L.f[S_SC];
    b.add(S_SC, q - 1, br * k.aw);
    b.add(S_SC, q + 1, br * k.ae);
    b.add(S_SC, q - nx, br * k.as);
    b.add(S_SC, q + nx, br * k.an);
    b.add(S_SC, q, -(br * k.ap));
    if (fine) b.add(S_RESSC, q, br);
    return coef_sc_adj(L, b, i, j, br * c[q - 1], br * c[q + 1], br * c[q - nx], br * c[q + nx], -(br * c[q]));
}

// P_FINE_RES at fine cell (i, j): the residual of equation `which` into its buffer.
__device__ void fine_res_adj(const LevelDev &F, const Bars &b, int i, int j, int which, ParAcc &pa)
{
    const int q = j * F.npx + i;
    if (which == 0) pa.amu_f += resid_u_adj(F, b, i, j, true, b.take(S_TMP0, q));
    else if (which == 1) pa.amu_f += resid_v_adj(F, b, i, j, true, b.take(S_TMP1, q));
    else pa.amusc_f += resid_sc_adj(F, b, i, j, true, b.take(S_TMP2, q));
}

// P_RESTRICT at coarse cell (ic, jc): the FAS defect = restricted fine residuals
// (cell_restrict_io's weights) - the coarse residual of the restricted state.
__device__ void restrict_adj(const LevelDev &F, const LevelDev &K, const Bars &bf, const Bars &bk, int ic, int jc,
                             int which, ParAcc &pa)
{
    const int nxf = F.npx, qc = jc * K.npx + ic, q = 2 * jc * nxf + 2 * ic;
    if (which == 0) {
        const double y = bk.take(S_RESU, qc);
        if (y == 0.0) return;
        bf.add(S_TMP0, q, y); bf.add(S_TMP0, q - nxf, y);
        bf.add(S_TMP0, q - 1, 0.5 * y); bf.add(S_TMP0, q - 1 - nxf, 0.5 * y);
        bf.add(S_TMP0, q + 1, 0.5 * y); bf.add(S_TMP0, q + 1 - nxf, 0.5 * y);
        pa.amu_k += resid_u_adj(K, bk, ic, jc, false, -y);
    } else if (which == 1) {
        const double y = bk.take(S_RESV, qc);
        if (y == 0.0) return;
        bf.add(S_TMP1, q, y); bf.add(S_TMP1, q - 1, y);
        bf.add(S_TMP1, q - nxf, 0.5 * y); bf.add(S_TMP1, q - nxf - 1, 0.5 * y);
        bf.add(S_TMP1, q + nxf, 0.5 * y); bf.add(S_TMP1, q + nxf - 1, 0.5 * y);
        pa.amu_k += resid_v_adj(K, bk, ic, jc, false, -y);
    } else {
        const double y = bk.take(S_RESSC, qc);
        if (y == 0.0) return;
        bf.add(S_TMP2, q, y); bf.add(S_TMP2, q - nxf, y);
        bf.add(S_TMP2, q - 1, y); bf.add(S_TMP2, q - 1 - nxf, y);
        pa.amusc_k += resid_sc_adj(K, bk, ic, jc, false, -y);
    }
}

// P_MASS_COEFP at interior cell (i, j).  MC_COEF: p' = 0 and aw = A_w^2 / apu_W ...,
// ap = their sum + constants (d(a / x)/dx = -(a / x) / x, the dual division's);
// MC_SU: su = -div, or 0 on a p' Dirichlet row.
__device__ void mass_coefp_adj(const CaseDev &C, const LevelDev &L, const Bars &b, int i, int j, int parts)
{
    const int nx = L.npx, ny = L.npy, q = j * nx + i, s = q - nx;
    const double *AX = L.f[S_AREAX], *AY = L.f[S_AREAY];
    if (parts & MC_COEF) {
        b.take(S_PP, q);
        const double bap = b.take(co_slot(EQ_PP, CK_AP), q);
        const double baw = b.take(co_slot(EQ_PP, CK_AW), q) + bap, bae = b.take(co_slot(EQ_PP, CK_AE), q) + bap,
                     bas = b.take(co_slot(EQ_PP, CK_AS), q) + bap, ban = b.take(co_slot(EQ_PP, CK_AN), q) + bap;
        const double axw = AX[q - 1], axq = AX[q], ays = AY[s], ayq = AY[q];
        const double *apu = L.f[S_APU], *apv = L.f[S_APV];
        const double qw = axw * axw / apu[q - 1], qe = axq * axq / apu[q];
        const double qs = ays * ays / apv[s], qn = ayq * ayq / apv[q];
        b.add(S_APU, q - 1, baw * (-(qw * 1.0) / apu[q - 1]));
        b.add(S_APU, q, bae * (-(qe * 1.0) / apu[q]));
        b.add(S_APV, s, bas * (-(qs * 1.0) / apv[s]));
        b.add(S_APV, q, ban * (-(qn * 1.0) / apv[q]));
    }
    if (parts & MC_SU) {
        const double bsu = b.take(co_slot(EQ_PP, CK_SU), q);
        const bool pinned = (C.ibc_xm == 2 && i == 1) || (C.ibc_xp == 2 && i == nx - 2) || (C.ibc_ym == 2 && j == 1) ||
                            (C.ibc_yp == 2 && j == ny - 2);
        if (bsu == 0.0 || pinned) return;
        // su = -(Ax u_P - Ax u_W + Ay v_P - Ay v_S)
        const double axq = AX[q], ayq = AY[q];
        b.add(S_U, q, -(bsu * axq));
        b.add(S_U, q - 1, bsu * axq);
        b.add(S_V, q, -(bsu * ayq));
        b.add(S_V, s, bsu * ayq);
    }
}

// P_UPDATE at interior cell q: u += Ax (p'_P - p'_E) / apu (parts & 1), v likewise with
// p'_N and apv (2), p += relxp p'_P (4).  Each field's own adjoint passes through
// unchanged (d new / d old = 1).
__device__ void update_adj(const CaseDev &C, const LevelDev &L, const Bars &b, int q, int parts)
{
    const double *pp = L.f[S_PP];
    if (parts & 1) {
        const double y = b.B.t[S_U][q];
        if (y != 0.0) {
            const double a = L.f[S_AREAX][q], apu = L.f[S_APU][q];
            const double r = a * (pp[q] - pp[q + 1]) / apu;
            b.add(S_PP, q, y * (a / apu));
            b.add(S_PP, q + 1, -(y * (a / apu)));
            b.add(S_APU, q, y * (-(r * 1.0) / apu));
        }
    }
    if (parts & 2) {
        const double y = b.B.t[S_V][q];
        if (y != 0.0) {
            const int n = q + L.npx;
            const double a = L.f[S_AREAY][q], apv = L.f[S_APV][q];
            const double r = a * (pp[q] - pp[n]) / apv;
            b.add(S_PP, q, y * (a / apv));
            b.add(S_PP, n, -(y * (a / apv)));
            b.add(S_APV, q, y * (-(r * 1.0) / apv));
        }
    }
    if (parts & 4) {
        const double y = b.B.t[S_P][q];
        if (y != 0.0) b.add(S_PP, q, y * C.relxp);
    }
}

// The transfers (linear maps of the fine and coarse states).
// P_RESTV at coarse cell (ic, jc): coarse x and R(x_f) of part `parts` (1 u, 2 v, 4 p, 8 sc).
__device__ void restv_adj(const LevelDev &F, const LevelDev &K, const Bars &bf, const Bars &bk, int ic, int jc,
                          int parts)
{
    const int nxf = F.npx, qc = jc * K.npx + ic, q = 2 * jc * nxf + 2 * ic, qw = q - 1, qs = q - nxf;
    if (parts & 1) {
        const double y = bk.take(S_U, qc) + bk.take(S_RU, qc);
        const double den = K.f[S_AREAX][qc] + 1.0e-30;
        bf.add(S_U, q, y * (F.f[S_AREAX][q] / den));
        bf.add(S_U, qs, y * (F.f[S_AREAX][qs] / den));
    }
    if (parts & 2) {
        const double y = bk.take(S_V, qc) + bk.take(S_RV, qc);
        const double den = K.f[S_AREAY][qc] + 1.0e-30;
        bf.add(S_V, q, y * (F.f[S_AREAY][q] / den));
        bf.add(S_V, qw, y * (F.f[S_AREAY][qw] / den));
    }
    for (int k = 2; k < 4; ++k) {
        if (!(parts & (1 << k))) continue;
        const int x = k == 2 ? S_P : S_SC, rx = k == 2 ? S_RP : S_RSC;
        const double y = 0.25 * (bk.take(x, qc) + bk.take(rx, qc));
        bf.add(x, q, y); bf.add(x, qw, y); bf.add(x, qs, y); bf.add(x, qs - 1, y);
    }
}

// P_PROL_CORR at coarse interior cell (ic, jc): c = x_c - R(x_f) (p's zeroed under solids).
__device__ void prol_corr_adj(const LevelDev &F, const LevelDev &K, const Bars &bf, const Bars &bk, int ic, int jc,
                              int parts)
{
    const int nxf = F.npx, nxc = K.npx, nyc = K.npy, qc = jc * nxc + ic, q = 2 * jc * nxf + 2 * ic, qs = q - nxf;
    if ((parts & 1) && ic <= nxc - 3) {
        const double y = bk.take(S_CU, qc);
        const double den = K.f[S_AREAX][qc] + 1.0E-30;
        bk.add(S_U, qc, y);
        bf.add(S_U, q, -(y * (F.f[S_AREAX][q] / den)));
        bf.add(S_U, qs, -(y * (F.f[S_AREAX][qs] / den)));
    }
    if ((parts & 2) && jc <= nyc - 3) {
        const double y = bk.take(S_CV, qc);
        const double den = K.f[S_AREAY][qc] + 1.0E-30;
        bk.add(S_V, qc, y);
        bf.add(S_V, q, -(y * (F.f[S_AREAY][q] / den)));
        bf.add(S_V, q - 1, -(y * (F.f[S_AREAY][q - 1] / den)));
    }
    for (int k = 2; k < 4; ++k) {
        if (!(parts & (1 << k))) continue;
        const int x = k == 2 ? S_P : S_SC;
        const double y = bk.take(k == 2 ? S_CP : S_C, qc);
        if (k == 2 && F.f[S_SPU][q] > 1.0e10) continue;
        bk.add(x, qc, y);
        const double r = -(0.25 * y);
        bf.add(x, q, r); bf.add(x, q - 1, r); bf.add(x, qs, r); bf.add(x, qs - 1, r);
    }
}

// P_PROL_APPLY at fine interior cell (i, j): the gather of cell_prol_apply_io (the
// corrections read from the arrays); the fine field's own adjoint passes through.
__device__ void prol_apply_adj(const LevelDev &F, const LevelDev &K, const Bars &bf, const Bars &bk, int i, int j,
                               int parts)
{
    const int nxf = F.npx, nyf = F.npy, nxc = K.npx, nyc = K.npy, q = j * nxf + i;
    const double f1 = 3. / 4., f2 = 1. / 4.;
    const double *spu = F.f[S_SPU], *spv = F.f[S_SPV];
    auto corr = [&](int slot, int ia, int ja, int ib, int jb, double w) {
        bk.add(slot, ja * nxc + ia, w * f1);
        bk.add(slot, jb * nxc + ib, w * f2);
    };
    if ((parts & 1) && i <= nxf - 3) {
        const double y = bf.B.t[S_U][q];
        if (y != 0.0) {
            const bool up = (j & 1) == 0;
            const int jc = up ? j / 2 : (j + 1) / 2, jn = up ? jc + 1 : jc - 1;
            if ((i & 1) == 0) {
                const int ic = i / 2;
                if (!(spu[2 * jc * nxf + 2 * ic] > 1.0e10)) corr(S_CU, ic, jc, ic, jn, y);
            } else {
                const int ia = (i - 1) / 2, ib = (i + 1) / 2;
                if (ia >= 1 && !(spu[2 * jc * nxf + 2 * ia] > 1.0e10)) corr(S_CU, ia, jc, ia, jn, 0.5 * y);
                if (ib <= nxc - 3 && !(spu[2 * jc * nxf + 2 * ib] > 1.0e10)) corr(S_CU, ib, jc, ib, jn, 0.5 * y);
            }
        }
    }
    if ((parts & 2) && j <= nyf - 3) {
        const double y = bf.B.t[S_V][q];
        if (y != 0.0) {
            const bool right = (i & 1) == 0;
            const int ic = right ? i / 2 : (i + 1) / 2, in = right ? ic + 1 : ic - 1;
            if ((j & 1) == 0) {
                const int jc = j / 2;
                if (!(spv[2 * jc * nxf + 2 * ic] > 1.0e10)) corr(S_CV, ic, jc, in, jc, y);
            } else {
                const int ja = (j - 1) / 2, jb = (j + 1) / 2;
                if (ja >= 1 && !(spv[2 * ja * nxf + 2 * ic] > 1.0e10)) corr(S_CV, ic, ja, in, ja, 0.5 * y);
                if (jb <= nyc - 3 && !(spv[2 * jb * nxf + 2 * ic] > 1.0e10)) corr(S_CV, ic, jb, in, jb, 0.5 * y);
            }
        }
    }
    const double g1 = 9. / 16., g2 = 3. / 16., g3 = 3. / 16., g4 = 1. / 16.;
    const int ic = (i + 1) / 2, jc = (j + 1) / 2;
    const int in = (i & 1) == 0 ? ic + 1 : ic - 1, jn = (j & 1) == 0 ? jc + 1 : jc - 1;
    for (int k = 2; k < 4; ++k) {
        if (!(parts & (1 << k))) continue;
        const double y = bf.B.t[k == 2 ? S_P : S_SC][q];
        if (y == 0.0) continue;
        const int c = k == 2 ? S_CP : S_C;
        bk.add(c, jc * nxc + ic, y * g1);
        bk.add(c, jc * nxc + in, y * g2);
        bk.add(c, jn * nxc + ic, y * g3);
        bk.add(c, jn * nxc + in, y * g4);
    }
}

// The closed-form transpose of one cell of phase P, for the kinds that have one;
// false: transpose it by probes.
__device__ __forceinline__ bool adj_closed(const CaseDev &C, const CaseTan &B, const Phase &P, int i, int j,
                                           ParAcc &pa)
{
    const LevelDev &F = C.lv[P.ig];
    const Bars bf{B.lv[P.ig]};
    switch (P.kind) {
    case P_ASM_U: asm_u_adj(C, F, bf, i, j, pa); return true;
    case P_ASM_V: asm_v_adj(C, F, bf, i, j, pa); return true;
    case P_ASM_SC: asm_sc_adj(F, bf, i, j, pa); return true;
    case P_FINE_RES: fine_res_adj(F, bf, i, j, P.a, pa); return true;
    case P_RESTRICT: restrict_adj(F, C.lv[P.ig + 1], bf, Bars{B.lv[P.ig + 1]}, i, j, P.a, pa); return true;
    case P_MASS_COEFP: mass_coefp_adj(C, F, bf, i, j, P.a); return true;
    case P_RESTV: restv_adj(F, C.lv[P.ig + 1], bf, Bars{B.lv[P.ig + 1]}, i, j, P.a); return true;
    case P_PROL_CORR: prol_corr_adj(F, C.lv[P.ig + 1], bf, Bars{B.lv[P.ig + 1]}, i, j, P.a); return true;
    case P_PROL_APPLY: prol_apply_adj(F, C.lv[P.ig + 1], bf, Bars{B.lv[P.ig + 1]}, i, j, P.a); return true;
    case P_UPDATE: update_adj(C, F, bf, j * F.npx + i, P.a); return true;
    default: return false;
    }
}

// ----------------------------------------------------------------- kernel
// Add a phase's amu/amusc adjoints of every thread to the case's per-level sums: a
// warp sum, then one atomic per warp and value.
__device__ __forceinline__ void flush_par(ParAcc &pa, const Phase &P, double *pacc)
{
    double v[4] = {pa.amu_f, pa.amusc_f, pa.amu_k, pa.amusc_k};
#pragma unroll
    for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0) {
        if (v[0] != 0.0) atomicAdd(pacc + 2 * P.ig, v[0]);
        if (v[1] != 0.0) atomicAdd(pacc + 2 * P.ig + 1, v[1]);
        if (v[2] != 0.0) atomicAdd(pacc + 2 * (P.ig + 1), v[2]);
        if (v[3] != 0.0) atomicAdd(pacc + 2 * (P.ig + 1) + 1, v[3]);
    }
    pa = ParAcc{0.0, 0.0, 0.0, 0.0};
}

// One V-cycle of case blockIdx.y, taped, then its transpose, on a cluster of
// gridDim.x CTAs (the cluster is the case: every phase is spread over its threads and
// separated from the next by a cluster barrier).  No thread leaves before the last
// barrier: every CTA of the cluster takes the same phases.
__global__ void __launch_bounds__(ADJ_BLOCK, 1) k_adj_cycle(const CaseDev *__restrict__ cs, CaseState *st,
                                                            const CaseTan *__restrict__ ts, const CaseAdj *__restrict__ as)
{
    __shared__ int bad_s;
    const CaseDev &C = cs[blockIdx.y];
    const CaseAdj &A = as[blockIdx.y];
    const CaseTan &B = ts[blockIdx.y];
    if (A.nphase <= 0) return;   // the same for every CTA of the cluster
    if (threadIdx.x == 0) bad_s = 0;
    __syncthreads();
    int bad = 0;
    // forward, taped (a half-sweep tapes and updates each cell in one pass)
    for (int p = 0; p < A.nphase; ++p) {
        const Phase P = A.prog[p];
        if (P.kind == P_GS && !A.generic) {
            double *tape = A.tape + P.off;
            gs_cells(C.lv[P.ig], P, [&](int i, int j, int t) { fwd_gs_cell(C.lv[P.ig], P.a, i, j, tape, t); });
            case_barrier();
            continue;
        }
        tape_copy(C, A, P, true);
        case_barrier();
        const RecCase X{C, write_level(P), write_mask(P), &bad};
        phase_cells(C, P, [&](int i, int j) { phase_cell(X, P, i, j); });
        case_barrier();
    }
    // reverse
    ParAcc pa{0.0, 0.0, 0.0, 0.0};
    for (int p = A.nphase - 1; p >= 0; --p) {
        const Phase P = A.prog[p];
        if (P.kind == P_GS && !A.generic) {
            const double *tape = A.tape + P.off;
            gs_cells(C.lv[P.ig], P,
                     [&](int i, int j, int t) { adj_gs_cell(C.lv[P.ig], B.lv[P.ig], P.a, i, j, tape, t); });
            case_barrier();
            continue;
        }
        tape_copy(C, A, P, false);
        case_barrier();
        {
            const bool closed = !A.generic && (P.kind == P_ASM_U || P.kind == P_ASM_V || P.kind == P_ASM_SC ||
                                               P.kind == P_FINE_RES || P.kind == P_RESTRICT ||
                                               P.kind == P_MASS_COEFP || P.kind == P_UPDATE || P.kind == P_RESTV ||
                                               P.kind == P_PROL_CORR || P.kind == P_PROL_APPLY);
            if (closed)
                phase_cells(C, P, [&](int i, int j) { adj_closed(C, B, P, i, j, pa); });
            else
                phase_cells(C, P, [&](int i, int j) { adj_cell(C, B, P, i, j, pa, &bad); });
            flush_par(pa, P, A.pacc);
        }
        case_barrier();
    }
    if (bad) atomicOr(&bad_s, 1);
    __syncthreads();
    if (threadIdx.x == 0 && bad_s) atomicOr(&st[blockIdx.y].status, (int)CASE_TAPE_ESCAPE);
}

__global__ void k_live_copy(const CaseDev *__restrict__ cs, const long long *__restrict__ off, double *buf, int dir)
{
    const CaseDev &C = cs[blockIdx.y];
    const int ig = blockIdx.z;
    if (ig >= C.ngrid) return;
    const LevelDev &L = C.lv[ig];
    long long base = off[blockIdx.y];
    for (int l = 0; l < ig; ++l) base += 4LL * C.lv[l].npx * C.lv[l].npy;
    const int n = L.npx * L.npy;
    const int slots[4] = {S_U, S_V, S_P, S_SC};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 4 * n; k += gridDim.x * blockDim.x) {
        double *a = L.f[slots[k / n]] + (k % n);
        double *b = buf + base + k;
        if (dir == 0) *b = *a;
        else *a = *b;
    }
}

}  // namespace

// ------------------------------------------------------------------ host
bool build_adj_program(const CaseDev &hc, const Sched &S, std::vector<Phase> &prog, long long &tape)
{
    prog.clear();
    tape = 0;
    if (hc.ibc_xm == 3 || hc.ibc_xp == 3 || hc.ibc_ym == 3 || hc.ibc_yp == 3) return false;
    const int ng = hc.ngrid;
    auto add = [&](int kind, int ig, int a = 0, int b = 0) {
        Phase P{kind, ig, a, b, tape};
        const LevelDev &L = hc.lv[write_level(P)];
        const unsigned long long m = write_mask(P);
        long long n = 0;
        if (kind == P_GS) {
            const Box d = box_eq(L.npx, L.npy, a);
            n = (long long)std::max(0, (d.wi + 1) >> 1) * std::max(0, d.wj);
        } else {
            for (int s = 0; s < NSLOTS; ++s)
                if ((m >> s) & 1ULL) n += (long long)L.npx * L.npy;
            if ((m >> PB_BIT) & 1ULL) n += L.ncopy;
        }
        tape += n;
        prog.push_back(P);
    };
    auto smooth = [&](int ig, const int *eqs, int ne, int nsw) {
        if (nsw <= 0) return;
        if (S.isolve == MGFVM_JACOBI) {
            for (int k = 0; k < ne; ++k) add(P_JAC_RING, ig, eqs[k]);
            for (int it = 0; it < nsw; ++it)
                for (int k = 0; k < ne; ++k) add(P_JAC_SWEEP, ig, eqs[k], it & 1);
            if (nsw & 1)
                for (int k = 0; k < ne; ++k) add(P_JAC_COPY, ig, eqs[k]);
        } else if (S.isolve == MGFVM_GAUSS_SEIDEL) {
            for (int h = 0; h < 2 * nsw; ++h)
                for (int k = 0; k < ne; ++k) add(P_GS, ig, eqs[k], h & 1);
        }
    };
    // one SIMPLE step on level ig (down leg :201-207, up leg :235-244)
    auto step = [&](int ig, bool down) {
        const int uvsc[3] = {EQ_U, EQ_V, EQ_SC}, pp[1] = {EQ_PP};
        add(P_ASM_U, ig);
        add(P_ASM_V, ig);
        add(P_ASM_SC, ig);
        if (down && hc.ibc_xp == 4) add(P_SC_OUTFLOW, ig);
        smooth(ig, uvsc, 3, S.nswpm);
        // multi-output routines run one output group per phase: a transposed phase then
        // probes only the reads of that group
        add(P_MASS_COEFP, ig, MC_COEF);
        add(P_MASS_COEFP, ig, MC_SU);
        smooth(ig, pp, 1, S.nswpp);
        for (int part = 1; part <= 4; part <<= 1) add(P_UPDATE, ig, part);
        if (hc.lv[ig].ncopy > 0) {
            if (hc.lv[ig].hazard) {
                add(P_PFIX_GATHER, ig);
                add(P_PFIX_SCATTER, ig);
            } else {
                add(P_PFIX, ig);
            }
        }
        if (hc.ibc_xp == 4) add(P_OUTFLOW, ig, 0, down ? 0 : 1);
    };
    for (int ig = 0; ig < ng; ++ig) {
        step(ig, true);
        if (ig != ng - 1) {
            for (int part = 1; part <= 8; part <<= 1) add(P_RESTV, ig, part);
            for (int w = 0; w < 3; ++w) add(P_FINE_RES, ig, w);
            for (int w = 0; w < 3; ++w) add(P_RESTRICT, ig, w);
        }
    }
    for (int ig = ng - 1; ig > 0; --ig) {
        for (int part = 1; part <= 8; part <<= 1) add(P_PROL_CORR, ig - 1, part);
        for (int part = 1; part <= 8; part <<= 1) add(P_PROL_APPLY, ig - 1, part);
        if (ig != 1) step(ig - 1, false);
    }
    return true;
}

cudaError_t launch_adj_cycle(const CaseDev *dc, CaseState *ds, const CaseTan *dt, const CaseAdj *da, int ncases,
                             int cluster, cudaStream_t st)
{
    if (cluster < 1 || cluster > 8) return cudaErrorInvalidValue;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3((unsigned)cluster, (unsigned)ncases, 1);
    c.blockDim = dim3(ADJ_BLOCK, 1, 1);
    c.stream = st;
    c.attrs = at;
    c.numAttrs = 1;
    return cudaLaunchKernelEx(&c, k_adj_cycle, dc, ds, dt, da);
}

int adj_cluster_size(int ncases, int sms)
{
    int g = 1;
    while (g < 8 && (long long)ncases * (g * 2) <= sms) g *= 2;
    return g;
}

cudaError_t launch_live_copy(const CaseDev *dc, const long long *off, double *buf, int ncases, int maxcells,
                             int maxng, int dir, cudaStream_t st)
{
    const int blocks = (4 * maxcells + BLOCK - 1) / BLOCK;
    k_live_copy<<<dim3(std::max(1, std::min(blocks, 1024)), ncases, maxng), BLOCK, 0, st>>>(dc, off, buf, dir);
    return cudaGetLastError();
}

}  // namespace mg
