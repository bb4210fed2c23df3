// mg_kernels.cu — the engine's kernels.
//
// Two execution shapes share the per-cell arithmetic of mg_cells.cuh:
//   * grid-wide kernels: one thread per cell, blockIdx.y selects the case, so one
//     launch advances one routine on one level of every case in the batch;
//   * k_tail: one CTA per case runs every coarse level of the V-cycle (down leg,
//     restrictions, prolongations, up leg) with __syncthreads() between routines,
//     because coarse grids are too small to fill the GPU and would otherwise be
//     pure launch overhead.
// All reductions are two-level and fixed-order (block tree, then the last block
// over the per-block partials), so results are reproducible run to run.
#include "mg_cells.cuh"
#include "mg_kernels.cuh"

namespace mg {

struct Dom { int i0, j0, wi, wj; };

__device__ __forceinline__ Dom dom_interior(const LevelDev &L) { return {1, 1, L.npx - 2, L.npy - 2}; }
__device__ __forceinline__ Dom dom_u(const LevelDev &L) { return {1, 1, L.npx - 3, L.npy - 2}; }
__device__ __forceinline__ Dom dom_v(const LevelDev &L) { return {1, 1, L.npx - 2, L.npy - 3}; }
__device__ __forceinline__ Dom dom_flux(const LevelDev &L) { return {0, 0, L.npx - 1, L.npy - 1}; }
// sweep extent of each equation (solve_u/v/pprime/sc :701, :710, :725, :735)
__device__ __forceinline__ Dom dom_eq(const LevelDev &L, int e)
{
    return e == 0 ? dom_u(L) : e == 1 ? dom_v(L) : dom_interior(L);
}
__device__ __forceinline__ int eq_slot(int e) { return e == 0 ? S_U : e == 1 ? S_V : e == 2 ? S_PP : S_SC; }

__device__ __forceinline__ bool cell_at(const Dom &d, int t, int &i, int &j)
{
    if (d.wi <= 0 || d.wj <= 0 || t >= d.wi * d.wj) return false;
    j = d.j0 + t / d.wi;
    i = d.i0 + t % d.wi;
    return true;
}

// ------------------------------------------------------------ reductions
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV])
{
    __shared__ double red[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            v[k] = lane < nw ? red[lane][k] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
    }
    __syncthreads();
}

// Write this block's NV partial sums; returns true (in every thread) for the last
// block to arrive, which then sees every block's partials.
template <int NV>
__device__ __forceinline__ bool publish_partials(double *partials, unsigned *counter, const double (&v)[NV],
                                                 int nblocks)
{
    __shared__ int is_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[blockIdx.x * RED_STRIDE + k] = v[k];
        __threadfence();
        unsigned prev = atomicAdd(counter, 1u);
        is_last = (prev == (unsigned)nblocks - 1u);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last != 0;
}

template <int NV>
__device__ __forceinline__ void gather_partials(const double *partials, int nblocks, double (&v)[NV])
{
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += __ldcg(&partials[b * RED_STRIDE + k]);
    block_sum<NV>(v);
}

// ------------------------------------------------------ grid-wide kernels
#define CASE_PROLOGUE(mode)                          \
    CaseDev &C = cs[blockIdx.y];                     \
    if (!case_active(C, ig, (mode))) return;         \
    const LevelDev &L = C.lv[ig];                    \
    const int t = blockIdx.x * blockDim.x + threadIdx.x;

__global__ void __launch_bounds__(BLOCK) k_fluxes(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_flux(L), t, i, j)) cell_fluxes(L, j * L.npx + i);
}

__global__ void __launch_bounds__(BLOCK) k_mom_u(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_u(L), t, i, j)) cell_mom_u(L, C, i, j);
}

__global__ void __launch_bounds__(BLOCK) k_mom_v(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_v(L), t, i, j)) cell_mom_v(L, C, i, j);
}

__global__ void __launch_bounds__(BLOCK) k_sc(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_interior(L), t, i, j)) cell_sc(L, C, i, j);
}

__global__ void __launch_bounds__(BLOCK) k_update(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_interior(L), t, i, j)) cell_update(L, C, j * L.npx + i);
}

// masserror + coefp; with `reduce`, sum|div| of this level lands in C.last_err.
__global__ void __launch_bounds__(BLOCK) k_mass_coefp(CaseDev *cs, int ig, int mode, int reduce)
{
    CASE_PROLOGUE(mode);
    const Dom d = dom_interior(L);
    const int n = d.wi * d.wj, nb = (n + blockDim.x - 1) / blockDim.x;
    if ((int)blockIdx.x >= nb) return;
    double a[1] = {0.0};
    int i, j;
    if (cell_at(d, t, i, j)) a[0] = cell_mass_coefp(L, C, i, j);
    if (!reduce) return;
    block_sum<1>(a);
    if (publish_partials<1>(C.partials, &C.counters[0], a, nb)) {
        double s[1];
        gather_partials<1>(C.partials, nb, s);
        if (threadIdx.x == 0) {
            C.last_err = s[0];
            C.counters[0] = 0;
        }
    }
}

// update's obstacle pressure copy as a gather (obstacles.c): phase 0 reads every
// source into pbuf, phase 1 writes them; phase 2 does both in one pass when no
// source is also a destination.
__global__ void __launch_bounds__(BLOCK) k_pfix(CaseDev *cs, int ig, int mode, int phase)
{
    CASE_PROLOGUE(mode);
    if (t >= L.ncopy) return;
    double *p = MGF(L, S_P);
    if (phase == 0) L.pbuf[t] = p[L.psrc[t]];
    else if (phase == 1) p[L.pdst[t]] = L.pbuf[t];
    else p[L.pdst[t]] = p[L.psrc[t]];
}

// pbound :1179-1210 — one block per case
__global__ void __launch_bounds__(BLOCK) k_periodic(CaseDev *cs, int ig, int mode)
{
    CaseDev &C = cs[blockIdx.y];
    if (!case_active(C, ig, mode)) return;
    const LevelDev &L = C.lv[ig];
    if (C.ibc_xm == 3)
        for (int j = 1 + threadIdx.x; j < L.npy - 1; j += blockDim.x) row_periodic_x(L, j);
    __syncthreads();
    if (C.ibc_ym == 3 && threadIdx.x == 0) line_periodic_y(L);
}

// outflow :1211-1228
__global__ void __launch_bounds__(BLOCK) k_outflow(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    if (C.ibc_xp != 4) return;
    if (t < L.npy) row_outflow(L, t);
}

// One Jacobi sweep of equation e: sweep index `it` reads phi (even) or the
// ping-pong buffer (odd); the first sweep also copies phi's ring into the buffer,
// since later sweeps read it there (solver :1254-1292).
__global__ void __launch_bounds__(BLOCK) k_jacobi(CaseDev *cs, int ig, int mode, int e, int it)
{
    CASE_PROLOGUE(mode);
    const Dom d = dom_eq(L, e);
    double *phi = MGF(L, eq_slot(e)), *tmp = MGF(L, S_TMP);
    const double *cur = (it & 1) ? tmp : phi;
    double *nxt = (it & 1) ? phi : tmp;
    if (it == 0) {
        const Dom x = {d.i0 - 1, d.j0 - 1, d.wi + 2, d.wj + 2};
        int i, j;
        if (!cell_at(x, t, i, j)) return;
        const int q = j * L.npx + i;
        if (i == x.i0 || i == x.i0 + x.wi - 1 || j == x.j0 || j == x.j0 + x.wj - 1) tmp[q] = phi[q];
        else cell_jacobi(L, cur, nxt, q);
    } else {
        int i, j;
        if (cell_at(d, t, i, j)) cell_jacobi(L, cur, nxt, j * L.npx + i);
    }
}

// After an odd number of sweeps the result sits in the buffer: copy it back.
__global__ void __launch_bounds__(BLOCK) k_jacobi_copyback(CaseDev *cs, int ig, int mode, int e)
{
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_eq(L, e), t, i, j)) {
        const int q = j * L.npx + i;
        MGF(L, eq_slot(e))[q] = MGF(L, S_TMP)[q];
    }
}

// One colour of a red-black Gauss-Seidel sweep (solvergs :1306-1350):
// colour 0 = (i+j) even, 1 = odd; threads map to cells of that colour only.
__global__ void __launch_bounds__(BLOCK) k_gs(CaseDev *cs, int ig, int mode, int e, int colour)
{
    CASE_PROLOGUE(mode);
    const Dom d = dom_eq(L, e);
    const int wr = (d.wi + 1) >> 1;
    if (t >= wr * d.wj) return;
    const int j = d.j0 + t / wr, k = t % wr;
    const int i = d.i0 + (((d.i0 + j) & 1) != colour ? 1 : 0) + 2 * k;
    if (i > d.i0 + d.wi - 1) return;
    cell_gs(L, MGF(L, eq_slot(e)), j * L.npx + i);
}

// restv on coarse level ig+1 from fine level ig
__global__ void __launch_bounds__(BLOCK) k_restv(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (cell_at(dom_interior(K), t, i, j)) cell_restv(L, K, i, j);
}

__global__ void __launch_bounds__(BLOCK) k_restrict(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (cell_at(dom_interior(K), t, i, j)) cell_restrict(L, K, C, i, j);
}

__global__ void __launch_bounds__(BLOCK) k_prol_corr(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (cell_at(dom_interior(K), t, i, j)) cell_prol_corr(L, K, i, j);
}

__global__ void __launch_bounds__(BLOCK) k_prol_apply(CaseDev *cs, int ig, int mode)
{
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (cell_at(dom_interior(L), t, i, j)) cell_prol_apply(L, K, i, j);
}

// End of a V-cycle on the level-0 interior: relative change of u, v, sc and of p
// with its mean removed against the previous cycle, the history entry, the stop
// rule, and prev <- current.  p sums are shifted by the previous cycle's means so a
// uniform pressure drift does not cancel catastrophically.
__global__ void __launch_bounds__(BLOCK) k_endcycle(CaseDev *cs)
{
    CaseDev &C = cs[blockIdx.y];
    if (C.done) return;
    const LevelDev &L = C.lv[0];
    const Dom d = dom_interior(L);
    const int n = d.wi * d.wj, nb = (n + blockDim.x - 1) / blockDim.x;
    if ((int)blockIdx.x >= nb) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double kd = C.shift_d, kp = C.shift_p;
    double a[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) a[k] = 0.0;
    int i, j;
    if (cell_at(d, t, i, j)) {
        const int q = j * L.npx + i;
        const int cur[4] = {S_U, S_V, S_SC, S_P}, prv[4] = {S_PREV_U, S_PREV_V, S_PREV_SC, S_PREV_P};
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            double x = MGF(L, cur[f])[q], y = MGF(L, prv[f])[q], dd = x - y;
            a[2 * f] = dd * dd;
            a[2 * f + 1] = x * x;
            MGF(L, prv[f])[q] = x;
        }
        double x = MGF(L, S_P)[q], y = MGF(L, S_PREV_P)[q];
        double dd = (x - y) - kd, e = x - kp;
        a[6] = dd; a[7] = dd * dd; a[8] = e; a[9] = e * e;
        MGF(L, S_PREV_P)[q] = x;
    }
    block_sum<10>(a);
    if (!publish_partials<10>(C.partials, &C.counters[1], a, nb)) return;
    double s[10];
    gather_partials<10>(C.partials, nb, s);
    if (threadIdx.x != 0) return;
    C.counters[1] = 0;
    const double N = (double)n;
    double worst = 0.0;
    for (int f = 0; f < 4; ++f) {
        double num, den;
        if (f < 3) { num = s[2 * f]; den = s[2 * f + 1]; }
        else {
            num = s[7] - s[6] * s[6] / N;
            den = s[9] - s[8] * s[8] / N;
            if (num < 0.0) num = 0.0;
        }
        double r = num == 0.0 ? 0.0 : (den <= 0.0 ? (double)INFINITY : sqrt(num / den));
        if (r > worst || r != r) worst = r;
    }
    const double err = C.last_err;
    const int k = C.ncyc;
    const double delta = C.have_prev ? worst : 0.0;
    if (k < C.hist_cap) {
        C.hist_err[k] = err;
        C.hist_delta[k] = delta;
    }
    C.ncyc = k + 1;
    C.shift_d = kd + s[6] / N;
    C.shift_p = kp + s[8] / N;
    const bool finite = isfinite(err) && isfinite(delta);
    if (!finite) C.status |= CASE_NONFINITE;
    if (C.stop_enabled) {
        if (!finite) C.done = 1;
        else if (err < C.convergence) { C.done = 1; C.status |= CASE_CONVERGED_REF; }
        else if (C.fp_tol > 0.0 && C.have_prev && delta < C.fp_tol) { C.done = 1; C.status |= CASE_CONVERGED_FP; }
    }
    C.have_prev = 1;
}

// ------------------------------------------------- one-CTA coarse kernel
template <class F>
__device__ __forceinline__ void for_cells(const Dom &d, F f)
{
    const int n = d.wi * d.wj;
    for (int t = threadIdx.x; t < n; t += blockDim.x) f(d.i0 + t % d.wi, d.j0 + t / d.wi);
}

__device__ void tail_smooth(const LevelDev &L, int e, const Sched &S)
{
    const Dom d = dom_eq(L, e);
    double *phi = MGF(L, eq_slot(e)), *tmp = MGF(L, S_TMP);
    const int nsw = e == 2 ? S.nswpp : S.nswpm;
    if (S.isolve == MGFVM_JACOBI) {
        {
            const Dom x = {d.i0 - 1, d.j0 - 1, d.wi + 2, d.wj + 2};
            for_cells(x, [&](int i, int j) {
                if (i == x.i0 || i == x.i0 + x.wi - 1 || j == x.j0 || j == x.j0 + x.wj - 1)
                    tmp[j * L.npx + i] = phi[j * L.npx + i];
            });
        }
        for (int it = 0; it < nsw; ++it) {
            const double *cur = (it & 1) ? tmp : phi;
            double *nxt = (it & 1) ? phi : tmp;
            for_cells(d, [&](int i, int j) { cell_jacobi(L, cur, nxt, j * L.npx + i); });
            __syncthreads();
        }
        if (nsw & 1) {
            for_cells(d, [&](int i, int j) { phi[j * L.npx + i] = tmp[j * L.npx + i]; });
            __syncthreads();
        }
    } else if (S.isolve == MGFVM_GAUSS_SEIDEL) {
        for (int it = 0; it < nsw; ++it)
            for (int colour = 0; colour < 2; ++colour) {
                const int wr = (d.wi + 1) >> 1, n = wr * d.wj;
                for (int t = threadIdx.x; t < n; t += blockDim.x) {
                    const int j = d.j0 + t / wr, k = t % wr;
                    const int i = d.i0 + (((d.i0 + j) & 1) != colour ? 1 : 0) + 2 * k;
                    if (i <= d.i0 + d.wi - 1) cell_gs(L, phi, j * L.npx + i);
                }
                __syncthreads();
            }
    }
}

// One SIMPLE step on level ig (down leg :201-207, up leg :235-244).
__device__ void tail_step(CaseDev &C, int ig, bool down, const Sched &S)
{
    const LevelDev &L = C.lv[ig];
    for_cells(dom_flux(L), [&](int i, int j) { cell_fluxes(L, j * L.npx + i); });
    __syncthreads();
    for_cells(dom_u(L), [&](int i, int j) { cell_mom_u(L, C, i, j); });
    __syncthreads();
    tail_smooth(L, 0, S);
    for_cells(dom_v(L), [&](int i, int j) { cell_mom_v(L, C, i, j); });
    __syncthreads();
    tail_smooth(L, 1, S);
    double acc[1] = {0.0};
    for_cells(dom_interior(L), [&](int i, int j) { acc[0] += cell_mass_coefp(L, C, i, j); });
    if (ig == 0 && down) {
        block_sum<1>(acc);
        if (threadIdx.x == 0) C.last_err = acc[0];
    }
    __syncthreads();
    tail_smooth(L, 2, S);
    for_cells(dom_interior(L), [&](int i, int j) { cell_update(L, C, j * L.npx + i); });
    __syncthreads();
    if (L.ncopy > 0) {
        double *p = MGF(L, S_P);
        if (L.hazard) {
            for (int t = threadIdx.x; t < L.ncopy; t += blockDim.x) L.pbuf[t] = p[L.psrc[t]];
            __syncthreads();
            for (int t = threadIdx.x; t < L.ncopy; t += blockDim.x) p[L.pdst[t]] = L.pbuf[t];
        } else {
            for (int t = threadIdx.x; t < L.ncopy; t += blockDim.x) p[L.pdst[t]] = p[L.psrc[t]];
        }
        __syncthreads();
    }
    if (C.ibc_xm == 3) {
        for (int j = 1 + threadIdx.x; j < L.npy - 1; j += blockDim.x) row_periodic_x(L, j);
        __syncthreads();
    }
    if (C.ibc_ym == 3) {
        if (threadIdx.x == 0) line_periodic_y(L);
        __syncthreads();
    }
    const bool outflow = C.ibc_xp == 4;
    if (down && outflow) {
        for (int j = threadIdx.x; j < L.npy; j += blockDim.x) row_outflow(L, j);
        __syncthreads();
    }
    for_cells(dom_interior(L), [&](int i, int j) { cell_sc(L, C, i, j); });
    __syncthreads();
    tail_smooth(L, 3, S);
    if (!down && outflow) {
        for (int j = threadIdx.x; j < L.npy; j += blockDim.x) row_outflow(L, j);
        __syncthreads();
    }
}

__device__ void tail_restrict(CaseDev &C, int ig)
{
    const LevelDev &F = C.lv[ig], &K = C.lv[ig + 1];
    for_cells(dom_interior(K), [&](int i, int j) { cell_restv(F, K, i, j); });
    __syncthreads();
    for_cells(dom_flux(K), [&](int i, int j) { cell_fluxes(K, j * K.npx + i); });
    for_cells(dom_flux(F), [&](int i, int j) { cell_fluxes(F, j * F.npx + i); });
    __syncthreads();
    for_cells(dom_interior(K), [&](int i, int j) { cell_restrict(F, K, C, i, j); });
    __syncthreads();
}

__device__ void tail_prolong(CaseDev &C, int ig)
{
    const LevelDev &F = C.lv[ig], &K = C.lv[ig + 1];
    for_cells(dom_interior(K), [&](int i, int j) { cell_prol_corr(F, K, i, j); });
    __syncthreads();
    for_cells(dom_interior(F), [&](int i, int j) { cell_prol_apply(F, K, i, j); });
    __syncthreads();
}

// Every level at or below C.tail of one case (blockIdx.x): the down leg from
// C.tail, the restrictions between those levels, and the up leg back to C.tail.
__global__ void __launch_bounds__(TAIL_BLOCK, 1) k_tail(CaseDev *cs, Sched S)
{
    CaseDev &C = cs[blockIdx.x];
    if (C.done || C.tail >= C.ngrid) return;
    for (int ig = C.tail; ig < C.ngrid; ++ig) {
        tail_step(C, ig, true, S);
        if (ig != C.ngrid - 1) tail_restrict(C, ig);
    }
    for (int ig = C.ngrid - 1; ig > C.tail; --ig) {
        tail_prolong(C, ig - 1);
        if (ig != 1) tail_step(C, ig - 1, false, S);
    }
}

// ------------------------------------------------------------- launcher
cudaError_t launch_one(const Launch &X, CaseDev *dc, const Sched &S, cudaStream_t st)
{
    const dim3 g = X.grid;
    const int b = X.block;
    switch (X.kernel) {
    case K_FLUXES: k_fluxes<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_MOM_U: k_mom_u<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_MOM_V: k_mom_v<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_MASS_COEFP: k_mass_coefp<<<g, b, 0, st>>>(dc, X.ig, X.mode, X.a0); break;
    case K_UPDATE: k_update<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_PFIX: k_pfix<<<g, b, 0, st>>>(dc, X.ig, X.mode, X.a0); break;
    case K_PERIODIC: k_periodic<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_OUTFLOW: k_outflow<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_SC: k_sc<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_JACOBI: k_jacobi<<<g, b, 0, st>>>(dc, X.ig, X.mode, X.a0, X.a1); break;
    case K_JACOBI_COPYBACK: k_jacobi_copyback<<<g, b, 0, st>>>(dc, X.ig, X.mode, X.a0); break;
    case K_GS: k_gs<<<g, b, 0, st>>>(dc, X.ig, X.mode, X.a0, X.a1); break;
    case K_RESTV: k_restv<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_RESTRICT: k_restrict<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_PROL_CORR: k_prol_corr<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_PROL_APPLY: k_prol_apply<<<g, b, 0, st>>>(dc, X.ig, X.mode); break;
    case K_TAIL: k_tail<<<g, b, 0, st>>>(dc, S); break;
    case K_ENDCYCLE: k_endcycle<<<g, b, 0, st>>>(dc); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ----------------------------------------------- raw-pointer entry points
__global__ void __launch_bounds__(BLOCK) r_jacobi(const double *__restrict__ aw, const double *__restrict__ ae,
                                                  const double *__restrict__ as, const double *__restrict__ an,
                                                  const double *__restrict__ ap, const double *__restrict__ su,
                                                  const double *cur, double *nxt, const double *phi, double *tmp,
                                                  int npx, int nx, int ny, int first)
{
    const int wi = first ? nx + 1 : nx - 1, wj = first ? ny + 1 : ny - 1, o = first ? 0 : 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi <= 0 || wj <= 0 || t >= wi * wj) return;
    const int i = o + t % wi, j = o + t / wi, q = j * npx + i;
    if (first && (i == 0 || i == nx || j == 0 || j == ny)) { tmp[q] = phi[q]; return; }
    const double wj1 = 1.0;
    double nb = aw[q] * cur[q - 1] + ae[q] * cur[q + 1] + as[q] * cur[q - npx] + an[q] * cur[q + npx];
    double g = (nb + su[q]) / (ap[q] + 1.0e-30);
    nxt[q] = (1.0 - wj1) * cur[q] + wj1 * g;
}

__global__ void __launch_bounds__(BLOCK) r_copy(const double *src, double *dst, int npx, int nx, int ny)
{
    const int wi = nx - 1, t = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi <= 0 || t >= wi * (ny - 1)) return;
    const int q = (1 + t / wi) * npx + 1 + t % wi;
    dst[q] = src[q];
}

__global__ void __launch_bounds__(BLOCK) r_gs(const double *__restrict__ aw, const double *__restrict__ ae,
                                              const double *__restrict__ as, const double *__restrict__ an,
                                              const double *__restrict__ ap, const double *__restrict__ su,
                                              double *phi, int npx, int nx, int ny, int colour)
{
    const int wi = nx - 1, wr = (wi + 1) >> 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi <= 0 || t >= wr * (ny - 1)) return;
    const int j = 1 + t / wr, k = t % wr;
    const int i = 1 + (((1 + j) & 1) != colour ? 1 : 0) + 2 * k;
    if (i > nx - 1) return;
    const int q = j * npx + i;
    double nb = aw[q] * phi[q - 1] + ae[q] * phi[q + 1] + as[q] * phi[q - npx] + an[q] * phi[q + npx];
    phi[q] = (nb + su[q]) / ap[q];
}

__global__ void __launch_bounds__(BLOCK) r_masserror(const double *u, const double *v, const double *ax,
                                                     const double *ay, double *su, double *pp, int npx,
                                                     int npy, double *err_out, double *partials)
{
    const int wi = npx - 2, n = wi * (npy - 2), nb = (n + blockDim.x - 1) / blockDim.x;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double a[1] = {0.0};
    if (t < n) {
        const int q = (1 + t / wi) * npx + 1 + t % wi;
        const double axq = ax[q], ayq = ay[q];
        double div = axq * u[q] - axq * u[q - 1] + ayq * v[q] - ayq * v[q - npx];
        su[q] = -div;
        pp[q] = 0.0;
        a[0] = fabs(div);
    }
    block_sum<1>(a);
    unsigned *counter = reinterpret_cast<unsigned *>(partials + (size_t)nb * RED_STRIDE);
    if (publish_partials<1>(partials, counter, a, nb)) {
        double s[1];
        gather_partials<1>(partials, nb, s);
        if (threadIdx.x == 0) { *err_out = s[0]; *counter = 0; }
    }
}

static inline int blocks_for(long long n) { return (int)((n + BLOCK - 1) / BLOCK); }

cudaError_t raw_jacobi(const double *aw, const double *ae, const double *as, const double *an,
                       const double *ap, const double *su, double *phi, double *scratch, int npx,
                       int npy, int nx, int ny, int nsw, cudaStream_t s)
{
    (void)npy;
    if (nsw <= 0 || nx < 2 || ny < 2) return cudaSuccess;
    for (int it = 0; it < nsw; ++it) {
        const double *cur = (it & 1) ? scratch : phi;
        double *nxt = (it & 1) ? phi : scratch;
        const long long n = it == 0 ? (long long)(nx + 1) * (ny + 1) : (long long)(nx - 1) * (ny - 1);
        r_jacobi<<<blocks_for(n), BLOCK, 0, s>>>(aw, ae, as, an, ap, su, cur, nxt, phi, scratch, npx, nx, ny,
                                                 it == 0);
    }
    if (nsw & 1) r_copy<<<blocks_for((long long)(nx - 1) * (ny - 1)), BLOCK, 0, s>>>(scratch, phi, npx, nx, ny);
    return cudaGetLastError();
}

cudaError_t raw_rbgs(const double *aw, const double *ae, const double *as, const double *an,
                     const double *ap, const double *su, double *phi, int npx, int npy, int nx, int ny,
                     int nsw, cudaStream_t s)
{
    (void)npy;
    if (nsw <= 0 || nx < 2 || ny < 2) return cudaSuccess;
    const long long n = (long long)((nx - 1 + 1) / 2) * (ny - 1);
    for (int it = 0; it < nsw; ++it)
        for (int c = 0; c < 2; ++c)
            r_gs<<<blocks_for(n), BLOCK, 0, s>>>(aw, ae, as, an, ap, su, phi, npx, nx, ny, c);
    return cudaGetLastError();
}

size_t raw_masserror_blocks(int npx, int npy)
{
    long long n = (long long)(npx - 2) * (npy - 2);
    return n > 0 ? (size_t)blocks_for(n) : 0;
}

cudaError_t raw_masserror(const double *u, const double *v, const double *ax, const double *ay, double *su,
                          double *pp, int npx, int npy, double *err_out, double *partials, cudaStream_t s)
{
    const int nb = (int)raw_masserror_blocks(npx, npy);
    if (nb == 0) return cudaMemsetAsync(err_out, 0, sizeof(double), s);
    r_masserror<<<nb, BLOCK, 0, s>>>(u, v, ax, ay, su, pp, npx, npy, err_out, partials);
    return cudaGetLastError();
}

}  // namespace mg
