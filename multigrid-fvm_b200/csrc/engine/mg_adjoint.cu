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

// The transpose of one red-black half-sweep cell, phi_c = (sum a_nb phi_nb + su) / ap
// (gs_value), written out: d/da_nb = phi_nb / ap, d/dphi_nb = a_nb / ap, d/dsu = 1 / ap,
// d/dap = -phi_c / ap, the partial derivatives the dual arithmetic of adj_cell forms,
// here with the adjoint divided by ap once (the same numbers to rounding) at one
// evaluation instead of eleven.  The cell's coefficients are read by no other cell of
// the half-sweep, so their adjoints take plain additions; the neighbours' take atomics.
__device__ __forceinline__ void adj_gs_cell(const LevelDev &L, const LevelTan &B, int e, int i, int j)
{
    const int nx = L.npx, q = j * nx + i, phi = field_of(e);
    double *yp = B.t[phi] + q;
    const double yb = *yp;
    *yp = 0.0;
    if (yb == 0.0) return;
    const double aw = L.f[co_slot(e, CK_AW)][q], ae = L.f[co_slot(e, CK_AE)][q], as = L.f[co_slot(e, CK_AS)][q],
                 an = L.f[co_slot(e, CK_AN)][q], ap = L.f[co_slot(e, CK_AP)][q], su = L.f[co_slot(e, CK_SU)][q];
    const double *f = L.f[phi];
    const double pw = f[q - 1], pe = f[q + 1], ps = f[q - nx], pn = f[q + nx];
    const double val = gs_value(aw, ae, as, an, ap, su, pw, pe, ps, pn);
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
    // forward, taped
    for (int p = 0; p < A.nphase; ++p) {
        const Phase P = A.prog[p];
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
        tape_copy(C, A, P, false);
        case_barrier();
        if (P.kind == P_GS && !A.generic) {
            phase_cells(C, P, [&](int i, int j) { adj_gs_cell(C.lv[P.ig], B.lv[P.ig], P.a, i, j); });
        } else {
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
