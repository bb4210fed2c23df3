// mg_kernels.cu — the engine's kernels.
//
// Three execution shapes share the per-cell arithmetic of mg_cells.cuh:
//   * grid-wide kernels: one thread per cell, blockIdx.y selects the case, so one
//     launch advances one routine on one level of every case in the batch;
//   * k_smooth: shared-memory tiles that run several smoother sweeps per launch on
//     a tile plus a halo as deep as the sweeps (temporal blocking); it reads one
//     buffer and writes the other, so no CTA ever loads a halo another CTA of the
//     same launch has already updated;
//   * k_tail: one CTA per case runs every coarse level of the V-cycle (down leg,
//     restrictions, prolongations, up leg) with __syncthreads() between routines,
//     because coarse grids are too small to fill the GPU and would otherwise be
//     pure launch overhead.
// Within a level visit the u, v and scalar equations depend only on the fluxes at
// the start of the visit (solve_u/v/sc :696-737 read cx, cy from fluxes :678-694),
// so they are assembled in one pass and smoothed in the same launches; p' follows.
// All reductions are two-level and fixed-order, so results are reproducible.
#include "mg_cells.cuh"
#include "mg_kernels.cuh"
#include "mg_tangent.cuh"

#include <type_traits>

namespace mg {

struct Dom { int i0, j0, wi, wj; };

__device__ __forceinline__ Dom dom_all(const LevelDev &L) { return {0, 0, L.npx, L.npy}; }
__device__ __forceinline__ Dom dom_interior(const LevelDev &L) { return {1, 1, L.npx - 2, L.npy - 2}; }
__device__ __forceinline__ Dom dom_flux(const LevelDev &L) { return {0, 0, L.npx - 1, L.npy - 1}; }
// sweep extent of each equation (solve_u/v/pprime/sc :701, :710, :725, :735)
__device__ __forceinline__ Dom dom_eq(const LevelDev &L, int e)
{
    if (e == EQ_U) return {1, 1, L.npx - 3, L.npy - 2};
    if (e == EQ_V) return {1, 1, L.npx - 2, L.npy - 3};
    return dom_interior(L);
}

__device__ __forceinline__ bool cell_at(const Dom &d, int t, int &i, int &j)
{
    if (d.wi <= 0 || d.wj <= 0 || t >= d.wi * d.wj) return false;
    j = d.j0 + t / d.wi;
    i = d.i0 + t % d.wi;
    return true;
}

__device__ __forceinline__ int nth_eq(int mask, int k)
{
    for (int e = 0; e < 4; ++e)
        if ((mask >> e) & 1) {
            if (k == 0) return e;
            --k;
        }
    return -1;
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

// ---------------------------------------------- programmatic dependent launch
// The V-cycle's kernels are launched with programmatic stream serialization (when the
// schedule's `pdl` switch is on), so a kernel's CTAs may be scheduled while its
// predecessor is still running.  Every kernel therefore starts by waiting until the
// grids it depends on have completed and their memory is visible (a no-op for a
// kernel launched without the attribute), and then lets its own dependent launch
// begin: at most one kernel waits ahead of the running one, and nothing a kernel
// reads or writes is touched before its predecessors are done.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ------------------------------------------------------ grid-wide kernels
#define CASE_PROLOGUE(mode)                          \
    const CaseDev &C = cs[blockIdx.y];               \
    CaseState &ST = st[blockIdx.y];                  \
    if (!case_active(C, ST, ig, (mode))) return;     \
    const LevelDev &L = C.lv[ig];                    \
    const int t = blockIdx.x * blockDim.x + threadIdx.x;

__global__ void __launch_bounds__(BLOCK) k_fluxes(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_flux(L), t, i, j)) cell_fluxes(L, j * L.npx + i);
}

// ------------------------------------------------ mixed precision: FP32 operands
// In a mixed-precision context the levels smoothed in tiles keep their smoother
// operands in FP32.  The assembly forms each equation's coefficients in FP64 with the
// same routines, then the FP64 residual of the current field, r = su + sum a_nb phi_nb
// - ap phi (the outer defect), and stores aw, ae, as, an, 1/ap and r as floats in the
// first halves of the equation's six coefficient arrays.  The smoother iterates the
// correction delta of A (phi + delta) = b in FP32 from zero, keeping delta between
// launches in two FP32 ping-pong buffers (the halves of the equation's buffer array),
// and its last launch adds delta to the FP64 field.  p' starts at zero, so its
// correction is p' itself: masserror + coefp store its operands (r = su) and update
// reads the FP32 p'.  The restriction, prolongation, norms and the coarse levels one
// CTA holds stay FP64.
__device__ __forceinline__ float *op32(const LevelDev &L, int e, int k)
{
    return reinterpret_cast<float *>(L.f[co_slot(e, k)]);
}
__device__ __forceinline__ float *del32(const LevelDev &L, int e, int buf)
{
    return reinterpret_cast<float *>(L.f[eq_tmp(e)]) + (size_t)buf * L.npx * L.npy;
}

// Prim whose stores of equation e's coefficient set (aw .. su) land in `k` instead of
// the arrays; every other store goes to the arrays.
struct Capture {
    using T = double;
    const LevelDev &L;
    int e;
    double *k;
    __device__ __forceinline__ double ld(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ void st(int s, int q, double v) const
    {
        const int c = s - co_slot(e, 0);
        if (c >= 0 && c < NCOEF) k[c] = v;
        else L.f[s][q] = v;
    }
    __device__ __forceinline__ double g(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ double amu() const { return L.amu; }
    __device__ __forceinline__ double amusc() const { return L.amusc; }
    __device__ __forceinline__ double pb(int i) const { return L.pbuf[i]; }
    __device__ __forceinline__ void set_pb(int i, double v) const { L.pbuf[i] = v; }
};

// The FP32 operands of equation e at cell q from its FP64 coefficients k (aw .. su)
// and field values phi (centre), pe (east; the caller knows when outflow moves it).
__device__ __forceinline__ void store_ops32(const LevelDev &L, int e, int q, const double *k, bool jac, double pe)
{
    const double *phi = L.f[eq_field(e)];
    const int nx = L.npx;
    const double ap = jac ? k[CK_AP] + 1.0e-30 : k[CK_AP];
    const double nb = k[CK_AW] * phi[q - 1] + k[CK_AE] * pe + k[CK_AS] * phi[q - nx] + k[CK_AN] * phi[q + nx];
    const double r = (nb + k[CK_SU]) - ap * phi[q];
    op32(L, e, CK_AW)[q] = (float)k[CK_AW];
    op32(L, e, CK_AE)[q] = (float)k[CK_AE];
    op32(L, e, CK_AS)[q] = (float)k[CK_AS];
    op32(L, e, CK_AN)[q] = (float)k[CK_AN];
    op32(L, e, CK_AP)[q] = (float)(1.0 / ap);
    op32(L, e, CK_SU)[q] = (float)r;
}

// cell_asm with A_F32: the same assemblies, FP32 operands stored instead of the FP64
// coefficient sets (APU, APV, the fluxes and the scalar ghost as before).  `sc_out`:
// the scalar's outflow ghost is (being) set from the cell west of it in this launch,
// so that cell's east value is its own.
__device__ __forceinline__ void cell_asm_f32(const LevelDev &L, const CaseDev &C, int i, int j, unsigned what,
                                             bool sc_out)
{
    const int nx = L.npx, ny = L.npy, q = j * nx + i;
    const FluxLive fl(L);
    const bool jac = (what & A_JAC) != 0;
    if ((what & A_FLUX) && i <= nx - 2 && j <= ny - 2) cell_fluxes(L, q);
    const bool in = i >= 1 && j >= 1 && i <= nx - 2 && j <= ny - 2;
    double k[NCOEF];
    if ((what & A_U) && in && i <= nx - 3) {
        cell_mom_u(Capture{L, EQ_U, k}, C, fl, i, j);
        store_ops32(L, EQ_U, q, k, jac, L.f[S_U][q + 1]);
    }
    if ((what & A_V) && in && j <= ny - 3) {
        cell_mom_v(Capture{L, EQ_V, k}, C, fl, i, j);
        store_ops32(L, EQ_V, q, k, jac, L.f[S_V][q + 1]);
    }
    if ((what & A_SC) && in) {
        cell_sc(Capture{L, EQ_SC, k}, C, fl, i, j);
        store_ops32(L, EQ_SC, q, k, jac, sc_out && i == nx - 2 ? L.f[S_SC][q] : L.f[S_SC][q + 1]);
    }
    if ((what & A_SC_OUTFLOW) && i == nx - 1 && C.ibc_xp == 4) L.f[S_SC][q] = L.f[S_SC][q - 1];
}

// Fused assembly over the padded array: fluxes, coefu+umom, coefv+vmom,
// coefsc+scalar, the scalar outflow ghost (AsmBits).  LIVE recomputes the fluxes
// from u, v (valid at the start of a level visit, before any of them changes).
template <int LIVE>
__global__ void __launch_bounds__(BLOCK) k_asm(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, unsigned what)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    int i, j;
    if (!cell_at(dom_all(L), t, i, j)) return;
    const unsigned w = asm_slice(what, blockIdx.z, gridDim.z);
    if (w & A_F32) cell_asm_f32(L, C, i, j, w, (w & A_SC_OUTFLOW) && C.ibc_xp == 4);
    else if (LIVE) cell_asm(L, C, FluxLive(L), i, j, w);
    else cell_asm(L, C, FluxArrays(L), i, j, w);
}

// update :1127-1152; with `fuse` bit 1 also outflow :1211-1228 of u, v, p (bit 2: and
// sc), with bit 4 also update's obstacle pressure copy (:1153-1177); bit 8: p' is in its
// ping-pong buffer (an odd number of smoother launches), read from there and copied back;
// bit 16: mixed precision, p' is the FP32 correction in buffer (bit 32 ? 1 : 0).  The copy gives
// every destination the post-update pressure of its source; each is written by one
// thread, the one updating the source (or, for a source on the boundary ring, the
// nearest interior cell, which reads it before writing anything), and destinations
// skip their own pressure write, so no thread reads a pressure another has changed.
// Outflow is fused when nothing between update and outflow in the reference (pbound,
// or the copy when it is not fused here) touches the outlet columns: the cell at
// i = npx-3 writes its new u to its face and the outlet face, the cell at i = npx-2 its
// new v and p to the ghost column (its copy's owner the copied p), and two extra
// threads copy the ghosts of the boundary rows.
// One interior cell of update (+ the fusions above): ppq, ppe, ppn = p' at the cell and
// its east and north neighbours.
// the values of its own cell an update reads besides p'
struct UpdIn {
    double u, v, p, ax, ay, apu, apv;
};
__device__ __forceinline__ UpdIn update_in(const LevelDev &L, int q)
{
    return {MGF(L, S_U)[q], MGF(L, S_V)[q], MGF(L, S_P)[q], MGF(L, S_AREAX)[q], MGF(L, S_AREAY)[q],
            MGF(L, S_APU)[q], MGF(L, S_APV)[q]};
}
__device__ __forceinline__ void update_cell(const LevelDev &L, const CaseDev &C, int i, int j, double ppq, double ppe,
                                            double ppn, bool out, int fuse, const UpdIn &in)
{
    const int nx = L.npx, q = j * nx + i;
    double *u = MGF(L, S_U), *v = MGF(L, S_V), *p = MGF(L, S_P);
    const double ppref = 0.0;
    const double un = in.u + in.ax * (ppq - ppe) / in.apu;
    const double vn = in.v + in.ay * (ppq - ppn) / in.apv;
    const double pn = in.p + C.relxp * (ppq - ppref);
    const int code = ((fuse & 4) && L.pcode) ? L.pcode[q] : 0;
    if (code & ~PCODE_DST) {
        for (int k = (code & ~PCODE_DST) - 1;; ++k) {
            const int e = L.pfan[2 * k], src = L.pfan[2 * k + 1], dq = e & ~PFAN_END;
            const double val = src < 0 ? pn : p[src];
            p[dq] = val;
            if (out && dq % nx == nx - 2) p[dq + 1] = val;
            if (e & PFAN_END) break;
        }
    }
    const bool dst = (code & PCODE_DST) != 0;
    if (!out || i != nx - 2) u[q] = un;
    v[q] = vn;
    if (!dst) p[q] = pn;
    if (out && i == nx - 3) u[q + 1] = un;
    if (out && i == nx - 2) {
        v[q + 1] = vn;
        if (!dst) p[q + 1] = pn;
        if (fuse & 2) MGF(L, S_SC)[q + 1] = MGF(L, S_SC)[q];
    }
}
__device__ __forceinline__ void update_cell(const LevelDev &L, const CaseDev &C, int i, int j, double ppq, double ppe,
                                            double ppn, bool out, int fuse)
{
    update_cell(L, C, i, j, ppq, ppe, ppn, out, fuse, update_in(L, j * L.npx + i));
}

// EARLY: the previous launch is a p' smoother, which writes none of the cell's other
// operands (u, v, p, areas, apu, apv), so they are read before waiting for it (a
// finished case, ST.done, set at the end of a cycle, loads nothing).
template <bool EARLY>
__global__ void __launch_bounds__(BLOCK) k_update(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode,
                                                  int fuse)
{
    if (!EARLY) pdl_enter();
    CASE_PROLOGUE(mode);
    const Dom d = dom_interior(L);
    const int n = d.wi * d.wj, nx = L.npx;
    const bool out = (fuse & 1) && C.ibc_xp == 4;
    int i, j;
    if (cell_at(d, t, i, j)) {
        const int q = j * nx + i;
        const UpdIn in = update_in(L, q);
        if (EARLY) pdl_enter();
        if (fuse & 16) {   // mixed precision: p' is FP32, in buffer (fuse & 32 ? 1 : 0) of its correction
            const float *pf = del32(L, EQ_PP, (fuse & 32) ? 1 : 0);
            update_cell(L, C, i, j, (double)pf[q], (double)pf[q + 1], (double)pf[q + nx], out, fuse, in);
            return;
        }
        const double *pp = MGF(L, (fuse & 8) ? S_TMP0 : S_PP);
        const double ppq = pp[q];
        if (fuse & 8) MGF(L, S_PP)[q] = ppq;
        update_cell(L, C, i, j, ppq, pp[q + 1], pp[q + nx], out, fuse, in);
    } else {
        if (EARLY) pdl_enter();
        if (out && t < n + 2) {
            const int jb = t == n ? 0 : L.npy - 1;
            row_outflow(L, jb, (fuse & 2) != 0);
        }
    }
}

// masserror + coefp; with `reduce`, sum|div| of this level lands in C.last_err.
// `flags` bit 1: u, v, sc are in their ping-pong buffers (an odd number of smoother
// launches); read from there and copied back.  Bit 2: mixed precision, p' operands
// stored in FP32 (r = su, as p' starts from zero; p' itself is not written); bit 4:
// with bit 2, the smoother is Jacobi.
// EARLY: the previous launch is a smoother, which writes none of the coefficients'
// operands (areas, apu, apv, tag): the coefficients are formed before waiting for it,
// u and v read after (a finished case, ST.done, set at the end of a cycle, forms nothing).
template <bool EARLY>
__global__ void __launch_bounds__(BLOCK) k_mass_coefp(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int reduce,
                                                      int flags)
{
    if (!EARLY) pdl_enter();
    CASE_PROLOGUE(mode);
    const Dom d = dom_interior(L);
    const int n = d.wi * d.wj, nb = (n + blockDim.x - 1) / blockDim.x;
    if ((int)blockIdx.x >= nb) return;
    double a[1] = {0.0};
    int i, j;
    if (EARLY) {
        const bool cell = cell_at(d, t, i, j);
        Coef k;
        double su = 0.0;
        if (cell) mass_coefp_io(Prim{L}, C, i, j, k, su, S_U, S_V, MC_COEF);
        pdl_enter();
        if (cell) {
            const Prim io{L};
            const int q = j * L.npx + i;
            const int us = (flags & 1) ? S_TMP0 : S_U, vs = (flags & 1) ? S_TMP1 : S_V;
            a[0] = mass_coefp_io(io, C, i, j, k, su, us, vs, MC_SU);
            if (flags & 2) {
                const double ap = (flags & 4) ? k.ap + 1.0e-30 : k.ap;
                op32(L, EQ_PP, CK_AW)[q] = (float)k.aw;
                op32(L, EQ_PP, CK_AE)[q] = (float)k.ae;
                op32(L, EQ_PP, CK_AS)[q] = (float)k.as;
                op32(L, EQ_PP, CK_AN)[q] = (float)k.an;
                op32(L, EQ_PP, CK_AP)[q] = (float)(1.0 / ap);
                op32(L, EQ_PP, CK_SU)[q] = (float)su;
            } else {
                // cell_mass_coefp's stores
                if (flags & 1) {
                    if (i <= L.npx - 3) io.st(S_U, q, io.ld(us, q));
                    if (j <= L.npy - 3) io.st(S_V, q, io.ld(vs, q));
                    io.st(S_SC, q, io.ld(S_TMP2, q));
                }
                io.st(S_PP, q, 0.0);
                store_coef(io, EQ_PP, q, k, su);
            }
        }
    } else if (cell_at(d, t, i, j)) {
        if (flags & 2) {
            Coef k;
            double su;
            a[0] = mass_coefp_values(L, C, i, j, k, su, S_U, S_V);
            const int q = j * L.npx + i;
            const double ap = (flags & 4) ? k.ap + 1.0e-30 : k.ap;
            op32(L, EQ_PP, CK_AW)[q] = (float)k.aw;
            op32(L, EQ_PP, CK_AE)[q] = (float)k.ae;
            op32(L, EQ_PP, CK_AS)[q] = (float)k.as;
            op32(L, EQ_PP, CK_AN)[q] = (float)k.an;
            op32(L, EQ_PP, CK_AP)[q] = (float)(1.0 / ap);
            op32(L, EQ_PP, CK_SU)[q] = (float)su;
        } else {
            a[0] = cell_mass_coefp(L, C, i, j, (flags & 1) != 0);
        }
    }
    if (!reduce) return;
    block_sum<1>(a);
    if (publish_partials<1>(C.partials, &C.counters[0], a, nb)) {
        double s[1];
        gather_partials<1>(C.partials, nb, s);
        if (threadIdx.x == 0) {
            ST.last_err = s[0];
            C.counters[0] = 0;
        }
    }
}

// update's obstacle pressure copy as a gather (obstacles.c): phase 0 reads every
// source into pbuf, phase 1 writes them; phase 2 does both in one pass when no
// source is also a destination.
__global__ void __launch_bounds__(BLOCK) k_pfix(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int phase)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    if (t >= L.ncopy) return;
    double *p = MGF(L, S_P);
    if (phase == 0) L.pbuf[t] = p[L.psrc[t]];
    else if (phase == 1) p[L.pdst[t]] = L.pbuf[t];
    else p[L.pdst[t]] = p[L.psrc[t]];
}

// pbound :1179-1210 then outflow :1211-1228 (bits: 1 periodic, 2 outflow of u, v, p,
// 4 the scalar ghost too) — one block per case.
// update's obstacle pressure copy (:1153-1177) by one CTA
template <class IO>
__device__ __forceinline__ void pfix_block_io(const IO &io)
{
    const LevelDev &L = io.L;
    if (L.ncopy <= 0) return;
    if (L.hazard) {
        for (int t = threadIdx.x; t < L.ncopy; t += blockDim.x) io.set_pb(t, io.ld(S_P, L.psrc[t]));
        __syncthreads();
        for (int t = threadIdx.x; t < L.ncopy; t += blockDim.x) io.st(S_P, L.pdst[t], io.pb(t));
    } else {
        for (int t = threadIdx.x; t < L.ncopy; t += blockDim.x) io.st(S_P, L.pdst[t], io.ld(S_P, L.psrc[t]));
    }
    __syncthreads();
}

template <class IO>
__device__ __forceinline__ void bound_block_io(const CaseDev &C, const IO &io, int bits)
{
    const LevelDev &L = io.L;
    if ((bits & 1) && C.ibc_xm == 3) {
        for (int j = 1 + threadIdx.x; j < L.npy - 1; j += blockDim.x) row_periodic_x_io(io, j);
        __syncthreads();
    }
    if ((bits & 1) && C.ibc_ym == 3) {
        if (threadIdx.x == 0) line_periodic_y_io(io);
        __syncthreads();
    }
    if ((bits & 2) && C.ibc_xp == 4) {
        for (int j = threadIdx.x; j < L.npy; j += blockDim.x) row_outflow_io(io, j, (bits & 4) != 0);
        __syncthreads();
    }
}
__device__ __forceinline__ void bound_block(const CaseDev &C, const LevelDev &L, int bits)
{
    bound_block_io(C, Prim{L}, bits);
}

__global__ void __launch_bounds__(BLOCK) k_bound(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int bits)
{
    pdl_enter();
    const CaseDev &C = cs[blockIdx.y];
    if (!case_active(C, st[blockIdx.y], ig, mode)) return;
    bound_block(C, C.lv[ig], bits);
}

// update's obstacle pressure copy (:1153-1177, as k_pfix) followed by pbound/outflow
// (as k_bound), one CTA per case: the copy may write the outlet columns that outflow
// then reads, so the two run in this order with a block barrier between them.
__global__ void __launch_bounds__(PFIX_BOUND_BLOCK) k_pfix_bound(const CaseDev *__restrict__ cs, CaseState *st, int ig,
                                                                 int mode, int bits)
{
    pdl_enter();
    const CaseDev &C = cs[blockIdx.y];
    if (!case_active(C, st[blockIdx.y], ig, mode)) return;
    const LevelDev &L = C.lv[ig];
    double *p = MGF(L, S_P);
    const int n = L.ncopy;
    if (L.hazard) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) L.pbuf[k] = p[L.psrc[k]];
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += blockDim.x) p[L.pdst[k]] = L.pbuf[k];
    } else {
        for (int k = threadIdx.x; k < n; k += blockDim.x) p[L.pdst[k]] = p[L.psrc[k]];
    }
    __syncthreads();
    bound_block(C, L, bits);
}

// Geometry of one smoother CTA (blockIdx.x picks a tile x tile block of equation e's
// sweep domain): the tile, the region it stages (the tile plus a halo of `nu` cells,
// clipped at the domain's boundary ring), and this thread's vertical pair of cells,
// one of each colour (A red: i+j even, B black).
struct PairTile {
    Dom d;
    int x0, y0, x1, y1, dx1, dy1, rx0, ry0, W, Hh, npairs;
    int i, jA, jB, kA, kB, gA, gB;
    int limA, limB;      // a domain cell is inside unit h's window while h <= lim (-1: never)
    bool okA, okB;       // the cell lies in the staged region
    bool outA, outB;     // written back: the tile, plus the boundary ring where it touches it
};

// 0: this CTA has work, 1: it has none, 2: the launch is too small for its region.
// `bx` picks the tile (blockIdx.x in the tiled smoothers).
__device__ __forceinline__ int pair_tile(const LevelDev &L, int e, int nu, int tile, PairTile &P, int bx)
{
    P.d = dom_eq(L, e);
    const Dom &d = P.d;
    if (d.wi <= 0 || d.wj <= 0) return 1;
    const int tx_n = (d.wi + tile - 1) / tile, ty_n = (d.wj + tile - 1) / tile;
    if (bx >= tx_n * ty_n) return 1;
    const int tx = bx % tx_n, ty = bx / tx_n;
    P.dx1 = d.i0 + d.wi - 1;
    P.dy1 = d.j0 + d.wj - 1;
    P.x0 = d.i0 + tx * tile;
    P.y0 = d.j0 + ty * tile;
    P.x1 = min(P.x0 + tile - 1, P.dx1);
    P.y1 = min(P.y0 + tile - 1, P.dy1);
    const int H = nu;
    P.rx0 = max(P.x0 - H, d.i0 - 1);
    P.ry0 = max(P.y0 - H, d.j0 - 1);
    P.W = min(P.x1 + H, P.dx1 + 1) - P.rx0 + 1;
    P.Hh = min(P.y1 + H, P.dy1 + 1) - P.ry0 + 1;
    P.npairs = P.W * ((P.Hh + 1) >> 1);
    if (P.npairs > (int)blockDim.x) return 2;
    const int W = P.W, t = threadIdx.x;
    const bool own = t < P.npairs;
    const int c = own ? t % W : 0, r = own ? 2 * (t / W) : 0;
    const int i = P.rx0 + c, jr = P.ry0 + r;
    const bool two = own && r + 1 < P.Hh;
    P.i = i;
    P.jA = ((i + jr) & 1) == 0 ? jr : jr + 1;
    P.jB = P.jA == jr ? jr + 1 : jr;
    P.okA = own && (P.jA == jr || two);
    P.okB = own && (P.jB == jr || two);
    P.kA = (P.jA - P.ry0) * W + c;
    P.kB = (P.jB - P.ry0) * W + c;
    P.gA = P.jA * L.npx + i;
    P.gB = P.jB * L.npx + i;
    const bool inx = i >= d.i0 && i <= P.dx1;
    const int dxe = min(i - P.x0, P.x1 - i);
    P.limA = P.okA && inx && P.jA >= d.j0 && P.jA <= P.dy1 ? H + min(dxe, min(P.jA - P.y0, P.y1 - P.jA)) : -1;
    P.limB = P.okB && inx && P.jB >= d.j0 && P.jB <= P.dy1 ? H + min(dxe, min(P.jB - P.y0, P.y1 - P.jB)) : -1;
    const bool outx = i >= (P.x0 == d.i0 ? P.x0 - 1 : P.x0) && i <= (P.x1 == P.dx1 ? P.x1 + 1 : P.x1);
    const int oy0 = P.y0 == d.j0 ? P.y0 - 1 : P.y0, oy1 = P.y1 == P.dy1 ? P.y1 + 1 : P.y1;
    P.outA = P.okA && outx && P.jA >= oy0 && P.jA <= oy1;
    P.outB = P.okB && outx && P.jB >= oy0 && P.jB <= oy1;
    return 0;
}

// Temporal-blocked smoother.  blockIdx.z picks an equation of `mask`, blockIdx.x a
// tile.  The CTA stages its region: every thread owns one vertical pair of cells,
// holds both cells' six coefficients in registers and their field values in shared
// memory, so a half-sweep is one update per thread.  It runs `nu` units — half-sweeps
// of red-black Gauss-Seidel (colour of global unit u0+h-1: even = red) or Jacobi
// sweeps — each on a window one cell narrower on every cut side, then writes the tile
// back: dir 0 from the field to the equation's ping-pong buffer, dir 1 the reverse,
// dir 2 in place (a single tile covering the domain: it reads everything before it
// writes).  Every cell update is the reference's formula on the same neighbour values,
// so the result is bit-identical to sweeping the whole level unit by unit.
// EARLY: the coefficients were written before the previous launch (a later launch of a
// smoothing split in several), so they are read before waiting for it (a finished
// case, ST.done, set at the end of a cycle, loads nothing).
template <int ISOLVE, int NT, bool EARLY>
__global__ void __launch_bounds__(NT, SMOOTH_BLOCK / NT) k_smooth(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int mask, int u0, int nu,
                                                         int dir, int tile)
{
    if (!EARLY) pdl_enter();
    extern __shared__ double sm[];
    const CaseDev &C = cs[blockIdx.y];
    if (!case_active(C, st[blockIdx.y], ig, mode)) return;
    const int e = nth_eq(mask, blockIdx.z);
    const LevelDev &L = C.lv[ig];
    PairTile P;
    const int g = pair_tile(L, e, nu, tile, P, blockIdx.x);
    if (g == 1) return;
    if (g == 2) {     // the schedule sizes blocks to fit; never taken
        if (threadIdx.x == 0) atomicOr(&st[blockIdx.y].status, (int)CASE_BAD_LAUNCH);
        return;
    }
    const int W = P.W, kA = P.kA, kB = P.kB, limA = P.limA, limB = P.limB;
    const int fs = eq_field(e), ts = eq_tmp(e);
    const double *src = L.f[dir == 1 ? ts : fs];
    double *dst = L.f[dir == 0 ? ts : fs];
    double *phi = sm, *phi2 = sm + W * P.Hh;
    const double *__restrict__ gaw = L.f[co_slot(e, CK_AW)];
    const double *__restrict__ gae = L.f[co_slot(e, CK_AE)];
    const double *__restrict__ gas = L.f[co_slot(e, CK_AS)];
    const double *__restrict__ gan = L.f[co_slot(e, CK_AN)];
    const double *__restrict__ gap = L.f[co_slot(e, CK_AP)];
    const double *__restrict__ gsu = L.f[co_slot(e, CK_SU)];
    double A[6] = {0, 0, 0, 0, 0, 0}, B[6] = {0, 0, 0, 0, 0, 0}, pA = 0.0, pB = 0.0;
    if (EARLY) {
        if (P.okA) {
            const int g0 = P.gA;
            A[0] = gaw[g0]; A[1] = gae[g0]; A[2] = gas[g0]; A[3] = gan[g0]; A[4] = gap[g0]; A[5] = gsu[g0];
        }
        if (P.okB) {
            const int g0 = P.gB;
            B[0] = gaw[g0]; B[1] = gae[g0]; B[2] = gas[g0]; B[3] = gan[g0]; B[4] = gap[g0]; B[5] = gsu[g0];
        }
        pdl_enter();
        if (P.okA) pA = src[P.gA];
        if (P.okB) pB = src[P.gB];
    } else {
        if (P.okA) {
            const int g0 = P.gA;
            pA = src[g0];
            A[0] = gaw[g0]; A[1] = gae[g0]; A[2] = gas[g0]; A[3] = gan[g0]; A[4] = gap[g0]; A[5] = gsu[g0];
        }
        if (P.okB) {
            const int g0 = P.gB;
            pB = src[g0];
            B[0] = gaw[g0]; B[1] = gae[g0]; B[2] = gas[g0]; B[3] = gan[g0]; B[4] = gap[g0]; B[5] = gsu[g0];
        }
    }
    const double eps = ISOLVE == MGFVM_JACOBI ? 1.0e-30 : 0.0;   // solver's (ap + 1e-30), solvergs' ap
    const Recip RA = make_recip(ISOLVE == MGFVM_JACOBI ? A[4] + eps : A[4]);
    const Recip RB = make_recip(ISOLVE == MGFVM_JACOBI ? B[4] + eps : B[4]);
    if (P.okA) {
        phi[kA] = pA;
        if (ISOLVE == MGFVM_JACOBI) phi2[kA] = pA;
    }
    if (P.okB) {
        phi[kB] = pB;
        if (ISOLVE == MGFVM_JACOBI) phi2[kB] = pB;
    }
    __syncthreads();
    for (int h = 1; h <= nu; ++h) {
        if (ISOLVE == MGFVM_GAUSS_SEIDEL) {
            if (((u0 + h - 1) & 1) == 0) {
                if (h <= limA)
                    phi[kA] = gs_value_r(A[0], A[1], A[2], A[3], RA, A[5], phi[kA - 1], phi[kA + 1], phi[kA - W],
                                         phi[kA + W]);
            } else {
                if (h <= limB)
                    phi[kB] = gs_value_r(B[0], B[1], B[2], B[3], RB, B[5], phi[kB - 1], phi[kB + 1], phi[kB - W],
                                         phi[kB + W]);
            }
        } else {
            const double *cur = ((h - 1) & 1) ? phi2 : phi;
            double *nxt = ((h - 1) & 1) ? phi : phi2;
            if (h <= limA)
                nxt[kA] = jacobi_value_r(A[0], A[1], A[2], A[3], RA, A[5], cur[kA - 1], cur[kA + 1], cur[kA - W],
                                         cur[kA + W], cur[kA]);
            if (h <= limB)
                nxt[kB] = jacobi_value_r(B[0], B[1], B[2], B[3], RB, B[5], cur[kB - 1], cur[kB + 1], cur[kB - W],
                                         cur[kB + W], cur[kB]);
        }
        __syncthreads();
    }
    const double *res = (ISOLVE == MGFVM_JACOBI && (nu & 1)) ? phi2 : phi;
    if (P.outA) dst[P.gA] = res[kA];
    if (P.outB) dst[P.gB] = res[kB];
}

// ------------------------------------------------ TMA-staged tile smoother
// The same tiles, units and windows as k_smooth, with the region staged in shared
// memory by two tensor-memory-accelerator box loads instead of per-thread loads: the
// six coefficient arrays of the equation as one box (they are consecutive slots of the
// level) and the field (or its ping-pong buffer).  The tensor maps view a level's
// slot arrays as one 3-D tensor (x, y, slot; the slots sit at a constant stride) and
// are built per case and launch shape by the host (SmoothMaps).  A box starts at an
// even x (8-byte elements: the copy's x must be a multiple of 2) and is one column
// wider where the region starts at an odd x; cells the box holds beyond the region are
// loaded and never written.  The field box is the shared-memory field the units
// update, so the results are those of k_smooth bit for bit.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// Wait for the mbarrier's phase 0 with at most `polls` polls; false on timeout.
__device__ __forceinline__ bool mbar_wait0(unsigned bar, int polls)
{
    for (int it = 0; it < polls; ++it) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar)
                     : "memory");
        if (done) return true;
    }
    return false;
}

template <int ISOLVE, int NT>
__global__ void __launch_bounds__(NT, SMOOTH_BLOCK / NT)
    k_smooth_tma(const CaseDev *__restrict__ cs, CaseState *st, const SmoothMap *__restrict__ maps, int ig, int mode,
                 int mask, int u0, int nu, int dir, int tile, int bw, int bh, int polls)
{
    pdl_enter();
    extern __shared__ __align__(128) double smt[];
    __shared__ __align__(8) unsigned long long mbar;
    const CaseDev &C = cs[blockIdx.y];
    if (!case_active(C, st[blockIdx.y], ig, mode)) return;
    const int e = nth_eq(mask, blockIdx.z);
    const LevelDev &L = C.lv[ig];
    PairTile P;
    const int g = pair_tile(L, e, nu, tile, P, blockIdx.x);
    if (g == 1) return;
    const int x0 = P.rx0 & ~1, off = P.rx0 - x0;
    if (g == 2 || P.W + off > bw || P.Hh > bh) {   // the schedule sizes blocks and boxes to fit; never taken
        if (threadIdx.x == 0) atomicOr(&st[blockIdx.y].status, (int)CASE_BAD_LAUNCH);
        return;
    }
    const int box = bw * bh;
    double *coef = smt, *phi = smt + NCOEF * box, *phi2 = phi + box;
    const unsigned bar = smem_u32(&mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const SmoothMap &M = maps[blockIdx.y];
        const unsigned bytes = (unsigned)((NCOEF + 1) * box * sizeof(double));
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                     ::"r"(smem_u32(coef)), "l"(&M.coef), "r"(x0), "r"(P.ry0), "r"(co_slot(e, CK_AW)), "r"(bar)
                     : "memory");
        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                     ::"r"(smem_u32(phi)), "l"(&M.field), "r"(x0), "r"(P.ry0), "r"(dir == 1 ? eq_tmp(e) : eq_field(e)),
                       "r"(bar)
                     : "memory");
    }
    // one decision for the whole block (a thread that gave up at the limit while the
    // others saw the copies land must not split the block at the barriers below)
    if (!__syncthreads_and(mbar_wait0(bar, polls))) {
        // record the stall and give the copies a second wait, at the full bound, so they
        // land before the CTA leaves; should that wait expire too, the CTA leaves with
        // copies in flight into shared memory a later CTA on this SM may take, and the
        // call fails with every case's results undefined until mgfvm_reset
        if (threadIdx.x == 0) atomicOr(&st[blockIdx.y].status, (int)CASE_WAIT_TIMEOUT);
        mbar_wait0(bar, TMA_WAIT_POLLS);
        return;
    }
    const int W = bw, limA = P.limA, limB = P.limB;
    const int kA = (P.jA - P.ry0) * bw + (P.i - x0), kB = (P.jB - P.ry0) * bw + (P.i - x0);
    double *dst = L.f[dir == 0 ? eq_tmp(e) : eq_field(e)];
    double A[6] = {0, 0, 0, 0, 0, 0}, B[6] = {0, 0, 0, 0, 0, 0};
    if (P.okA)
        for (int a = 0; a < 6; ++a) A[a] = coef[a * box + kA];
    if (P.okB)
        for (int a = 0; a < 6; ++a) B[a] = coef[a * box + kB];
    const double eps = ISOLVE == MGFVM_JACOBI ? 1.0e-30 : 0.0;   // solver's (ap + 1e-30), solvergs' ap
    const Recip RA = make_recip(ISOLVE == MGFVM_JACOBI ? A[4] + eps : A[4]);
    const Recip RB = make_recip(ISOLVE == MGFVM_JACOBI ? B[4] + eps : B[4]);
    if (ISOLVE == MGFVM_JACOBI) {
        if (P.okA) phi2[kA] = phi[kA];
        if (P.okB) phi2[kB] = phi[kB];
        __syncthreads();
    }
    for (int h = 1; h <= nu; ++h) {
        if (ISOLVE == MGFVM_GAUSS_SEIDEL) {
            if (((u0 + h - 1) & 1) == 0) {
                if (h <= limA)
                    phi[kA] = gs_value_r(A[0], A[1], A[2], A[3], RA, A[5], phi[kA - 1], phi[kA + 1], phi[kA - W],
                                         phi[kA + W]);
            } else {
                if (h <= limB)
                    phi[kB] = gs_value_r(B[0], B[1], B[2], B[3], RB, B[5], phi[kB - 1], phi[kB + 1], phi[kB - W],
                                         phi[kB + W]);
            }
        } else {
            const double *cur = ((h - 1) & 1) ? phi2 : phi;
            double *nxt = ((h - 1) & 1) ? phi : phi2;
            if (h <= limA)
                nxt[kA] = jacobi_value_r(A[0], A[1], A[2], A[3], RA, A[5], cur[kA - 1], cur[kA + 1], cur[kA - W],
                                         cur[kA + W], cur[kA]);
            if (h <= limB)
                nxt[kB] = jacobi_value_r(B[0], B[1], B[2], B[3], RB, B[5], cur[kB - 1], cur[kB + 1], cur[kB - W],
                                         cur[kB + W], cur[kB]);
        }
        __syncthreads();
    }
    const double *res = (ISOLVE == MGFVM_JACOBI && (nu & 1)) ? phi2 : phi;
    if (P.outA) dst[P.gA] = res[kA];
    if (P.outB) dst[P.gB] = res[kB];
}

// All `mu` units of equation e on a level that one CTA holds, in place (k_smooth with
// one tile covering the domain).  Returns pair_tile's verdict (uniform over the CTA).
template <int ISOLVE>
__device__ __forceinline__ int level_smooth_eq(const LevelDev &L, int e, int mu, double *sm)
{
    PairTile P;
    const int g = pair_tile(L, e, mu, max(L.npx, L.npy), P, 0);
    if (g != 0) return g;
    const int W = P.W, kA = P.kA, kB = P.kB, limA = P.limA, limB = P.limB;
    double *phi = sm, *phi2 = sm + W * P.Hh, *fld = MGF(L, eq_field(e));
    double A[6] = {0, 0, 0, 0, 0, 0}, B[6] = {0, 0, 0, 0, 0, 0};
    if (P.okA) {
        const double pa = fld[P.gA];
        for (int a = 0; a < 6; ++a) A[a] = MGF(L, co_slot(e, a))[P.gA];
        phi[kA] = pa;
        if (ISOLVE == MGFVM_JACOBI) phi2[kA] = pa;
    }
    if (P.okB) {
        const double pb = fld[P.gB];
        for (int a = 0; a < 6; ++a) B[a] = MGF(L, co_slot(e, a))[P.gB];
        phi[kB] = pb;
        if (ISOLVE == MGFVM_JACOBI) phi2[kB] = pb;
    }
    const double eps = ISOLVE == MGFVM_JACOBI ? 1.0e-30 : 0.0;
    const Recip RA = make_recip(ISOLVE == MGFVM_JACOBI ? A[4] + eps : A[4]);
    const Recip RB = make_recip(ISOLVE == MGFVM_JACOBI ? B[4] + eps : B[4]);
    __syncthreads();
    for (int h = 1; h <= mu; ++h) {
        if (ISOLVE == MGFVM_GAUSS_SEIDEL) {
            if (((h - 1) & 1) == 0) {
                if (h <= limA)
                    phi[kA] = gs_value_r(A[0], A[1], A[2], A[3], RA, A[5], phi[kA - 1], phi[kA + 1], phi[kA - W],
                                         phi[kA + W]);
            } else {
                if (h <= limB)
                    phi[kB] = gs_value_r(B[0], B[1], B[2], B[3], RB, B[5], phi[kB - 1], phi[kB + 1], phi[kB - W],
                                         phi[kB + W]);
            }
        } else {
            const double *cur = ((h - 1) & 1) ? phi2 : phi;
            double *nxt = ((h - 1) & 1) ? phi : phi2;
            if (h <= limA)
                nxt[kA] = jacobi_value_r(A[0], A[1], A[2], A[3], RA, A[5], cur[kA - 1], cur[kA + 1], cur[kA - W],
                                         cur[kA + W], cur[kA]);
            if (h <= limB)
                nxt[kB] = jacobi_value_r(B[0], B[1], B[2], B[3], RB, B[5], cur[kB - 1], cur[kB + 1], cur[kB - W],
                                         cur[kB + W], cur[kB]);
        }
        __syncthreads();
    }
    const double *res = (ISOLVE == MGFVM_JACOBI && (mu & 1)) ? phi2 : phi;
    if (limA >= 0) fld[P.gA] = res[kA];
    if (limB >= 0) fld[P.gB] = res[kB];
    return 0;
}

// After the update of a one-CTA level: `fuse` bit 128, the obstacle pressure copy (when
// update does not do it); bits 8-10, pbound / outflow with these k_bound bits — the
// launches after_update would add, run by the same CTA.
__device__ __forceinline__ void pp_level_tail(const CaseDev &C, const LevelDev &L, int fuse)
{
    if (!(fuse & (128 | (7 << 8)))) return;
    __syncthreads();
    if (fuse & 128) pfix_block_io(Prim{L});
    if ((fuse >> 8) & 7) bound_block_io(C, Prim{L}, (fuse >> 8) & 7);
}

// solve_pprime and update on a level that one CTA per case holds (at most SMOOTH_BLOCK
// vertical cell pairs): masserror + coefp for every interior cell (:1096-1125,
// :1018-1092), all `nu` p' units in shared memory (as k_smooth with one tile), then
// update (:1127-1152) with k_update's fusions (`fuse` bits 1, 2, 4) reading p' from
// shared memory, and the final p' written to the field.  The p' coefficients stay in
// registers (nothing else reads them).  With `reduce` the level's sum |div| (a block
// tree) becomes the case's mass error; then pp_level_tail (`fuse` bits 128, 8-10).
// Same bits as the separate kernels.
template <int ISOLVE>
__device__ __forceinline__ void pp_level_body(const CaseDev &C, CaseState &ST, const LevelDev &L, int nu, int reduce,
                                              int fuse, double *sm)
{
    PairTile P;
    const int g = pair_tile(L, EQ_PP, nu, max(L.npx, L.npy), P, 0);
    if (g == 1) {
        pp_level_tail(C, L, fuse);
        return;
    }
    if (g == 2) {
        if (threadIdx.x == 0) atomicOr(&ST.status, (int)CASE_BAD_LAUNCH);
        return;
    }
    const int W = P.W, kA = P.kA, kB = P.kB, limA = P.limA, limB = P.limB;
    double *phi = sm, *phi2 = sm + W * P.Hh;
    double *pp = MGF(L, S_PP);
    double A[6] = {0, 0, 0, 0, 0, 0}, B[6] = {0, 0, 0, 0, 0, 0}, pA = 0.0, pB = 0.0, divs = 0.0;
    {
        Coef k;
        double su;
        if (P.okA) {
            if (limA >= 0) {
                divs += mass_coefp_values(L, C, P.i, P.jA, k, su, S_U, S_V);
                A[0] = k.aw; A[1] = k.ae; A[2] = k.as; A[3] = k.an; A[4] = k.ap; A[5] = su;
            } else {
                pA = pp[P.gA];      // boundary ring: masserror leaves it
            }
        }
        if (P.okB) {
            if (limB >= 0) {
                divs += mass_coefp_values(L, C, P.i, P.jB, k, su, S_U, S_V);
                B[0] = k.aw; B[1] = k.ae; B[2] = k.as; B[3] = k.an; B[4] = k.ap; B[5] = su;
            } else {
                pB = pp[P.gB];
            }
        }
    }
    const double eps = ISOLVE == MGFVM_JACOBI ? 1.0e-30 : 0.0;
    const Recip RA = make_recip(ISOLVE == MGFVM_JACOBI ? A[4] + eps : A[4]);
    const Recip RB = make_recip(ISOLVE == MGFVM_JACOBI ? B[4] + eps : B[4]);
    if (P.okA) {
        phi[kA] = pA;
        if (ISOLVE == MGFVM_JACOBI) phi2[kA] = pA;
    }
    if (P.okB) {
        phi[kB] = pB;
        if (ISOLVE == MGFVM_JACOBI) phi2[kB] = pB;
    }
    __syncthreads();
    for (int h = 1; h <= nu; ++h) {
        if (ISOLVE == MGFVM_GAUSS_SEIDEL) {
            if (((h - 1) & 1) == 0) {
                if (h <= limA)
                    phi[kA] = gs_value_r(A[0], A[1], A[2], A[3], RA, A[5], phi[kA - 1], phi[kA + 1], phi[kA - W],
                                         phi[kA + W]);
            } else {
                if (h <= limB)
                    phi[kB] = gs_value_r(B[0], B[1], B[2], B[3], RB, B[5], phi[kB - 1], phi[kB + 1], phi[kB - W],
                                         phi[kB + W]);
            }
        } else {
            const double *cur = ((h - 1) & 1) ? phi2 : phi;
            double *nxt = ((h - 1) & 1) ? phi : phi2;
            if (h <= limA)
                nxt[kA] = jacobi_value_r(A[0], A[1], A[2], A[3], RA, A[5], cur[kA - 1], cur[kA + 1], cur[kA - W],
                                         cur[kA + W], cur[kA]);
            if (h <= limB)
                nxt[kB] = jacobi_value_r(B[0], B[1], B[2], B[3], RB, B[5], cur[kB - 1], cur[kB + 1], cur[kB - W],
                                         cur[kB + W], cur[kB]);
        }
        __syncthreads();
    }
    const double *res = (ISOLVE == MGFVM_JACOBI && (nu & 1)) ? phi2 : phi;
    const bool out = (fuse & 1) && C.ibc_xp == 4;
    // the region is the padded level (W = npx), so shared and global indices coincide
    if (limA >= 0) {
        pp[P.gA] = res[kA];
        update_cell(L, C, P.i, P.jA, res[kA], res[kA + 1], res[kA + W], out, fuse);
    }
    if (limB >= 0) {
        pp[P.gB] = res[kB];
        update_cell(L, C, P.i, P.jB, res[kB], res[kB + 1], res[kB + W], out, fuse);
    }
    if (out && threadIdx.x < 2) row_outflow(L, threadIdx.x == 0 ? 0 : L.npy - 1, (fuse & 2) != 0);
    if (reduce) {
        double a[1] = {divs};
        block_sum<1>(a);
        if (threadIdx.x == 0) ST.last_err = a[0];
    }
    pp_level_tail(C, L, fuse);
}

template <int ISOLVE>
__global__ void __launch_bounds__(SMOOTH_BLOCK, 1) k_pp_level(const CaseDev *__restrict__ cs, CaseState *st, int ig,
                                                              int mode, int nu, int reduce, int fuse)
{
    pdl_enter();
    extern __shared__ double sm[];
    const CaseDev &C = cs[blockIdx.y];
    CaseState &ST = st[blockIdx.y];
    if (!case_active(C, ST, ig, mode)) return;
    pp_level_body<ISOLVE>(C, ST, C.lv[ig], nu, reduce, fuse, sm);
}

// Every thread of the cluster arrives; memory written before it (global included) is
// visible to every thread of the cluster after it.
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// A whole visit to a level that one CTA per case holds, as one launch of a cluster of
// three CTAs per case (cluster rank r = blockIdx.x: u, v, sc).  CTA r runs its part of
// the level's assembly `what` (the slices of k_asm with three slices: fluxes + u, v,
// sc + outflow ghost) over every cell, then — once the whole cluster has assembled, as
// the smoothers read nothing the other parts write — `mu` units of its equation in
// place; after a second cluster barrier CTA 0 runs solve_pprime and update
// (pp_level_body).  No thread leaves before the barriers: the case's activity is the
// same for the three CTAs and only guards the work.
template <int ISOLVE>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(SMOOTH_BLOCK, 1)
    k_level_visit(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int nu, int reduce, int fuse,
                  int what, int mu)
{
    pdl_enter();
    extern __shared__ double sm[];
    const CaseDev &C = cs[blockIdx.y];
    CaseState &ST = st[blockIdx.y];
    const bool active = case_active(C, ST, ig, mode);
    const LevelDev &L = C.lv[ig];
    const int r = blockIdx.x;
    if (what) {
        if (active) {
            const unsigned w = asm_slice((unsigned)what, r, 3);
            const int n = L.npx * L.npy;
            for (int q = threadIdx.x; q < n; q += blockDim.x) cell_asm(L, C, FluxLive(L), q % L.npx, q / L.npx, w);
        }
        cluster_barrier();
    }
    if (active && mu > 0 && level_smooth_eq<ISOLVE>(L, r == 0 ? EQ_U : r == 1 ? EQ_V : EQ_SC, mu, sm) == 2 &&
        threadIdx.x == 0)
        atomicOr(&ST.status, (int)CASE_BAD_LAUNCH);   // the schedule sizes blocks to fit; never taken
    cluster_barrier();
    if (active && r == 0) pp_level_body<ISOLVE>(C, ST, L, nu, reduce, fuse, sm);
}

// ------------------------------------------------ band visits (a cluster per case)
// A whole visit to a level too large for one CTA but small enough for a cluster of G
// (at most 8) CTAs, in one launch.  CTA r of the cluster owns a band of interior rows
// [j0, j1) (band_rows(npy, G) rows each, an even number; the last band may be shorter),
// one thread per interior column and vertical cell pair of its band.  A smoothing
// stages the band and one row on either side (the neighbouring bands' edge rows, or the
// boundary ring) in shared memory.  In every unit each thread updates its cell of the
// unit's colour (both cells, for Jacobi) and, where that cell is on an edge row of the
// band, stores the new value into the neighbouring band's copy of the row
// (distributed shared memory); a cluster barrier ends the unit, so every cell update
// reads the values a whole-level sweep reads: the same bits as the grid kernels.
// Order: the assembly `what` over the cells of the whole level | cluster barrier |
// u, v, sc smoothing (mu units each, one after the other) | cluster barrier |
// masserror + coefp, the p' units, update with k_update's fusions (`fuse`), the level's
// sum |div| with `reduce`.  Every CTA of a cluster takes the same cluster barriers (the
// case's activity is the same for all of them; a CTA without rows only joins them).
__device__ __forceinline__ unsigned cl_rank_k()
{
    unsigned v;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(v));
    return v;
}
__device__ __forceinline__ unsigned cl_size_k()
{
    unsigned v;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(v));
    return v;
}
// the shared::cluster address `p` (a shared-memory location of this CTA) has in CTA `rank`
__device__ __forceinline__ unsigned cl_map(const void *p, unsigned rank)
{
    unsigned a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}
// store v at the shared-memory location `p` has in CTA `rank` of the cluster
__device__ __forceinline__ void st_cluster(double *p, unsigned rank, double v)
{
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(cl_map(p, rank)), "d"(v) : "memory");
}

// One CTA's band and this thread's pair: cells (i, ja) and (i, ja + 1).
struct Band {
    int r, G;
    int j0, j1, b, nx, base;   // rows [j0, j1), full band height b, shared index = q - base
    int i, ja, jb;
    bool ownA, ownB;           // the cell is in the band
    bool below, above;         // a neighbouring band exists below (r - 1) / above (r + 1)
};
__device__ __forceinline__ Band band_of(const LevelDev &L, int r, int G)
{
    Band B;
    B.r = r;
    B.G = G;
    B.nx = L.npx;
    B.b = band_rows(L.npy, G);
    B.j0 = 1 + r * B.b;
    B.j1 = min(B.j0 + B.b, L.npy - 1);
    B.base = (B.j0 - 1) * L.npx;
    const int wc = L.npx - 2, t = threadIdx.x;
    B.i = 1 + t % wc;
    B.ja = B.j0 + 2 * (t / wc);
    B.jb = B.ja + 1;
    const bool some = B.j1 > B.j0;
    const bool own = some && t < wc * (B.b / 2);
    B.ownA = own && B.ja < B.j1;
    B.ownB = own && B.jb < B.j1;
    B.below = some && r > 0;
    B.above = some && B.j1 < L.npy - 1;   // then the band is full height and r + 1 < G
    return B;
}

__device__ __forceinline__ bool in_dom(const Dom &d, int i, int j)
{
    return i >= d.i0 && i < d.i0 + d.wi && j >= d.j0 && j < d.j0 + d.wj;
}

// The two cells of this thread in one equation's smoothing: coefficients, reciprocals,
// shared indices and whether each is in the equation's domain.
struct BandCells {
    double A[6], Bc[6];
    Recip RA, RB;
    int sA, sB;
    bool inA, inB;
};

// `units` units of a smoothing on the staged band (phi; phi2 = phi + stride for
// Jacobi), the neighbours' edge rows exchanged after every unit, a cluster barrier
// after each (a CTA without rows takes them too).  Returns the buffer holding the result.
template <int ISOLVE>
__device__ __forceinline__ const double *band_units(const Band &B, const Dom &d, int units, double *sm, size_t stride,
                                                    const BandCells &K)
{
    constexpr bool JAC = ISOLVE == MGFVM_JACOBI;
    double *phi = sm, *phi2 = sm + stride;
    const int nx = B.nx;
    const bool redA = ((B.i + B.ja) & 1) == 0;
    // after a unit: the cell (i, j) value v just written goes to the neighbouring bands'
    // copies of the row (`buf`: the buffer's offset; every CTA has the same layout)
    auto send = [&](int j, size_t buf, double v) {
        if (j == B.j0 && B.below) st_cluster(sm + buf + (size_t)(B.b + 1) * nx + B.i, B.r - 1, v);
        if (j == B.j1 - 1 && B.above) st_cluster(sm + buf + B.i, B.r + 1, v);
    };
    for (int h = 1; h <= units; ++h) {
        if (!JAC) {
            const bool useA = (((h - 1) & 1) == 0) == redA;
            if (useA ? K.inA : K.inB) {
                const int s = useA ? K.sA : K.sB;
                const double *c = useA ? K.A : K.Bc;
                const double v = gs_value_r(c[0], c[1], c[2], c[3], useA ? K.RA : K.RB, c[5], phi[s - 1], phi[s + 1],
                                            phi[s - nx], phi[s + nx]);
                phi[s] = v;
                send(useA ? B.ja : B.jb, 0, v);
            }
        } else {
            const double *cur = ((h - 1) & 1) ? phi2 : phi;
            double *nxt = ((h - 1) & 1) ? phi : phi2;
            const size_t nb = ((h - 1) & 1) ? 0 : stride;
            if (K.inA) {
                const double v = jacobi_value_r(K.A[0], K.A[1], K.A[2], K.A[3], K.RA, K.A[5], cur[K.sA - 1],
                                                cur[K.sA + 1], cur[K.sA - nx], cur[K.sA + nx], cur[K.sA]);
                nxt[K.sA] = v;
                send(B.ja, nb, v);
            }
            if (K.inB) {
                const double v = jacobi_value_r(K.Bc[0], K.Bc[1], K.Bc[2], K.Bc[3], K.RB, K.Bc[5], cur[K.sB - 1],
                                                cur[K.sB + 1], cur[K.sB - nx], cur[K.sB + nx], cur[K.sB]);
                nxt[K.sB] = v;
                send(B.jb, nb, v);
            }
        }
        cluster_barrier();
    }
    return (JAC && (units & 1)) ? phi2 : phi;
}

// `units` units of equation e's smoother on the banded level, from and back to its field.
template <int ISOLVE>
__device__ void band_smooth_eq(const LevelDev &L, const Band &B, int e, int units, double *sm)
{
    constexpr bool JAC = ISOLVE == MGFVM_JACOBI;
    const Dom d = dom_eq(L, e);
    const int nx = B.nx;
    const size_t stride = (size_t)(B.b + 2) * nx;
    double *fld = L.f[eq_field(e)];
    __syncthreads();   // the previous smoothing's write-back has read the buffers
    if (B.j1 > B.j0) {
        const int n = (B.j1 - B.j0 + 2) * nx;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const double v = fld[B.base + k];
            sm[k] = v;
            if (JAC) sm[stride + k] = v;
        }
    }
    BandCells K;
    K.inA = B.ownA && in_dom(d, B.i, B.ja);
    K.inB = B.ownB && in_dom(d, B.i, B.jb);
    const int qA = B.ja * nx + B.i, qB = B.jb * nx + B.i;
    K.sA = qA - B.base;
    K.sB = qB - B.base;
    for (int a = 0; a < 6; ++a) {
        K.A[a] = K.inA ? L.f[co_slot(e, a)][qA] : 0.0;
        K.Bc[a] = K.inB ? L.f[co_slot(e, a)][qB] : 0.0;
    }
    K.RA = make_recip(JAC ? K.A[4] + 1.0e-30 : K.A[4]);
    K.RB = make_recip(JAC ? K.Bc[4] + 1.0e-30 : K.Bc[4]);
    cluster_barrier();   // every band staged before any neighbour writes into it
    const double *res = band_units<ISOLVE>(B, d, units, sm, stride, K);
    if (K.inA) fld[qA] = res[K.sA];
    if (K.inB) fld[qB] = res[K.sB];
}

// masserror + coefp, the p' units and update (+ fusions) on the banded level.
template <int ISOLVE>
__device__ void band_pp(const CaseDev &C, CaseState &ST, const LevelDev &L, const Band &B, int nu, int reduce,
                        int fuse, double *sm, double *red)
{
    constexpr bool JAC = ISOLVE == MGFVM_JACOBI;
    const Dom d = dom_interior(L);
    const int nx = B.nx;
    const size_t stride = (size_t)(B.b + 2) * nx;
    double *pp = MGF(L, S_PP);
    BandCells K;
    double divs = 0.0;
    K.inA = B.ownA;
    K.inB = B.ownB;
    {
        Coef k;
        double su = 0.0;
        for (int a = 0; a < 6; ++a) K.A[a] = K.Bc[a] = 0.0;
        if (B.ownA) {
            divs += mass_coefp_values(L, C, B.i, B.ja, k, su, S_U, S_V);
            K.A[0] = k.aw; K.A[1] = k.ae; K.A[2] = k.as; K.A[3] = k.an; K.A[4] = k.ap; K.A[5] = su;
        }
        if (B.ownB) {
            divs += mass_coefp_values(L, C, B.i, B.jb, k, su, S_U, S_V);
            K.Bc[0] = k.aw; K.Bc[1] = k.ae; K.Bc[2] = k.as; K.Bc[3] = k.an; K.Bc[4] = k.ap; K.Bc[5] = su;
        }
    }
    // p' starts at zero in the interior (masserror), the ring keeps its values
    __syncthreads();
    if (B.j1 > B.j0) {
        const int n = (B.j1 - B.j0 + 2) * nx;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int q = B.base + k, i = q % nx, j = q / nx;
            const double v = (i >= 1 && i <= nx - 2 && j >= 1 && j <= L.npy - 2) ? 0.0 : pp[q];
            sm[k] = v;
            if (JAC) sm[stride + k] = v;
        }
    }
    K.RA = make_recip(JAC ? K.A[4] + 1.0e-30 : K.A[4]);
    K.RB = make_recip(JAC ? K.Bc[4] + 1.0e-30 : K.Bc[4]);
    const int qA = B.ja * nx + B.i, qB = B.jb * nx + B.i;
    K.sA = qA - B.base;
    K.sB = qB - B.base;
    cluster_barrier();   // every CTA has read u, v and staged its band
    const double *res = band_units<ISOLVE>(B, d, nu, sm, stride, K);
    const bool out = (fuse & 1) && C.ibc_xp == 4;
    if (B.ownA) {
        pp[qA] = res[K.sA];
        update_cell(L, C, B.i, B.ja, res[K.sA], res[K.sA + 1], res[K.sA + nx], out, fuse);
    }
    if (B.ownB) {
        pp[qB] = res[K.sB];
        update_cell(L, C, B.i, B.jb, res[K.sB], res[K.sB + 1], res[K.sB + nx], out, fuse);
    }
    if (out && B.r == 0 && threadIdx.x < 2) row_outflow(L, threadIdx.x == 0 ? 0 : L.npy - 1, (fuse & 2) != 0);
    if (reduce) {
        // the level's sum |div| in a fixed order: a block sum per CTA, the CTAs' sums
        // added in rank order by CTA 0
        double a[1] = {divs};
        block_sum<1>(a);
        if (threadIdx.x == 0) st_cluster(red + B.r, 0, a[0]);
        cluster_barrier();
        if (B.r == 0 && threadIdx.x == 0) {
            double sum = 0.0;
            for (int k = 0; k < B.G; ++k) sum += red[k];
            ST.last_err = sum;
        }
    }
}

template <int ISOLVE>
__global__ void __launch_bounds__(SMOOTH_BLOCK, 1)
    k_band_visit(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int nu, int reduce, int fuse,
                 int what, int mu)
{
    pdl_enter();
    extern __shared__ double sm[];
    __shared__ double red[BAND_MAX_CTAS];
    const CaseDev &C = cs[blockIdx.y];
    CaseState &ST = st[blockIdx.y];
    if (!case_active(C, ST, ig, mode)) return;   // the same for every CTA of the cluster
    const LevelDev &L = C.lv[ig];
    const int r = (int)cl_rank_k(), G = (int)cl_size_k();
    {
        // the schedule sizes the launch for the largest case; never taken (the check
        // depends on the case and the launch only, so the whole cluster leaves together)
        unsigned dyn;
        asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        const int b = band_rows(L.npy, G);
        const size_t need = (size_t)(ISOLVE == MGFVM_JACOBI ? 2 : 1) * (b + 2) * L.npx * sizeof(double);
        if ((L.npx - 2) * (b / 2) > (int)blockDim.x || need > dyn || G > BAND_MAX_CTAS) {
            if (r == 0 && threadIdx.x == 0) atomicOr(&ST.status, (int)CASE_BAD_LAUNCH);
            return;
        }
    }
    if (what) {
        const int n = L.npx * L.npy;
        for (int q = r * blockDim.x + threadIdx.x; q < n; q += G * blockDim.x)
            cell_asm(L, C, FluxLive(L), q % L.npx, q / L.npx, (unsigned)what);
        cluster_barrier();
    }
    const Band B = band_of(L, r, G);
    if (mu > 0) {
        band_smooth_eq<ISOLVE>(L, B, EQ_U, mu, sm);
        band_smooth_eq<ISOLVE>(L, B, EQ_V, mu, sm);
        band_smooth_eq<ISOLVE>(L, B, EQ_SC, mu, sm);
        cluster_barrier();   // u, v written before masserror reads them across bands
    }
    band_pp<ISOLVE>(C, ST, L, B, nu, reduce, fuse, sm, red);
}

// Mixed precision (MGFVM_PREC_MIXED): the tiles, units and windows of k_smooth on
// the FP32 operands the assembly stored (aw, ae, as, an, 1/ap, r; see op32), iterating
// the correction delta_P = (sum a_nb delta_nb + r) / ap in FP32.  `flags` bit 1: the
// first launch of the call (delta starts at zero), bit 2: the last (the field gets
// phi + delta in FP64; p' keeps delta, which is p' itself), bit 4: delta is read from
// buffer 1 and written to buffer 0 (else the reverse).  Every launch writes the tile's
// delta, and zero on the boundary ring where the tile touches it, to its output buffer.
// EARLY: a later launch of the smoothing (not the first): its operands were written
// before the previous launch and are read before waiting for it; the correction after.
template <int ISOLVE, int NT, bool EARLY>
__global__ void __launch_bounds__(NT, SMOOTH_BLOCK / NT) k_smooth_f32(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int mask,
                                                             int u0, int nu, int flags, int tile)
{
    if (!EARLY) pdl_enter();
    extern __shared__ float smf[];
    const CaseDev &C = cs[blockIdx.y];
    if (!case_active(C, st[blockIdx.y], ig, mode)) return;
    const int e = nth_eq(mask, blockIdx.z);
    const LevelDev &L = C.lv[ig];
    PairTile P;
    const int g = pair_tile(L, e, nu, tile, P, blockIdx.x);
    if (g == 1) return;
    if (g == 2) {
        if (threadIdx.x == 0) atomicOr(&st[blockIdx.y].status, (int)CASE_BAD_LAUNCH);
        return;
    }
    const bool first = (flags & 1) != 0, last = (flags & 2) != 0;
    const int rb = (flags & 4) ? 1 : 0;
    const int W = P.W, R = P.W * P.Hh, kA = P.kA, kB = P.kB, limA = P.limA, limB = P.limB;
    const float *src = del32(L, e, rb);
    float *dst = del32(L, e, rb ^ 1);
    float *del = smf, *del2 = smf + R;
    const float *__restrict__ o0 = op32(L, e, CK_AW);
    const float *__restrict__ o1 = op32(L, e, CK_AE);
    const float *__restrict__ o2 = op32(L, e, CK_AS);
    const float *__restrict__ o3 = op32(L, e, CK_AN);
    const float *__restrict__ o4 = op32(L, e, CK_AP);
    const float *__restrict__ o5 = op32(L, e, CK_SU);
    // operands of the cells this launch updates (the domain cells of its windows)
    float A[6] = {0, 0, 0, 0, 0, 0}, B[6] = {0, 0, 0, 0, 0, 0}, dA = 0.0f, dB = 0.0f;
    if (limA >= 1) {
        const int g0 = P.gA;
        A[0] = o0[g0]; A[1] = o1[g0]; A[2] = o2[g0]; A[3] = o3[g0]; A[4] = o4[g0]; A[5] = o5[g0];
    }
    if (limB >= 1) {
        const int g0 = P.gB;
        B[0] = o0[g0]; B[1] = o1[g0]; B[2] = o2[g0]; B[3] = o3[g0]; B[4] = o4[g0]; B[5] = o5[g0];
    }
    if (EARLY) pdl_enter();
    if (!first) {
        if (P.okA) dA = src[P.gA];
        if (P.okB) dB = src[P.gB];
    }
    if (P.okA) { del[kA] = dA; if (ISOLVE == MGFVM_JACOBI) del2[kA] = dA; }
    if (P.okB) { del[kB] = dB; if (ISOLVE == MGFVM_JACOBI) del2[kB] = dB; }
    __syncthreads();
    for (int h = 1; h <= nu; ++h) {
        if (ISOLVE == MGFVM_GAUSS_SEIDEL) {
            if (((u0 + h - 1) & 1) == 0) {
                if (h <= limA)
                    del[kA] = (A[0] * del[kA - 1] + A[1] * del[kA + 1] + A[2] * del[kA - W] + A[3] * del[kA + W] + A[5]) * A[4];
            } else {
                if (h <= limB)
                    del[kB] = (B[0] * del[kB - 1] + B[1] * del[kB + 1] + B[2] * del[kB - W] + B[3] * del[kB + W] + B[5]) * B[4];
            }
        } else {
            const float *cur = ((h - 1) & 1) ? del2 : del;
            float *nxt = ((h - 1) & 1) ? del : del2;
            if (h <= limA)
                nxt[kA] = (A[0] * cur[kA - 1] + A[1] * cur[kA + 1] + A[2] * cur[kA - W] + A[3] * cur[kA + W] + A[5]) * A[4];
            if (h <= limB)
                nxt[kB] = (B[0] * cur[kB - 1] + B[1] * cur[kB + 1] + B[2] * cur[kB - W] + B[3] * cur[kB + W] + B[5]) * B[4];
        }
        __syncthreads();
    }
    const float *res = (ISOLVE == MGFVM_JACOBI && (nu & 1)) ? del2 : del;
    // the tile's cells (lim >= 1) and the ring cells it touches (delta 0 there)
    const float rA = limA >= 1 ? res[kA] : 0.0f, rB = limB >= 1 ? res[kB] : 0.0f;
    if (P.outA) dst[P.gA] = rA;
    if (P.outB) dst[P.gB] = rB;
    if (last && e != EQ_PP) {
        double *phi = L.f[eq_field(e)];
        if (P.outA && limA >= 1) phi[P.gA] = phi[P.gA] + (double)rA;
        if (P.outB && limB >= 1) phi[P.gB] = phi[P.gB] + (double)rB;
    }
}

// After an odd number of smoothing launches the result sits in the ping-pong buffer.
__global__ void __launch_bounds__(BLOCK) k_copy(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode, int mask)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    const int e = nth_eq(mask, blockIdx.z);
    const int fs = e == EQ_U ? S_U : e == EQ_V ? S_V : e == EQ_PP ? S_PP : S_SC;
    int i, j;
    if (cell_at(dom_eq(L, e), t, i, j)) MGF(L, fs)[j * L.npx + i] = MGF(L, eq_tmp(e))[j * L.npx + i];
}

// restv :1354-1389 on coarse level ig+1, fluxes(fine) :216 and the fine residuals of
// restr{u,v,sc}, one thread per (fine cell, slice `which` of 3)
template <class IO>
__device__ __forceinline__ void cell_restv_fluxes_io(const IO &F, const IO &K, const CaseDev &C, int i, int j,
                                                     int which, int nwhich)
{
    if (which == 0) {
        if (i <= F.L.npx - 2 && j <= F.L.npy - 2) cell_fluxes_io(F, j * F.L.npx + i);
        if (((i | j) & 1) == 0) {
            const int ic = i >> 1, jc = j >> 1;
            if (ic >= 1 && jc >= 1 && ic <= K.L.npx - 2 && jc <= K.L.npy - 2) cell_restv_io(F, K, ic, jc);
        }
    }
    for (int w = which; w < 3; w += nwhich) cell_fine_residuals_io(F, C, i, j, w);
}
__device__ __forceinline__ void cell_restv_fluxes(const LevelDev &F, const LevelDev &K, const CaseDev &C, int i,
                                                  int j, int which, int nwhich)
{
    cell_restv_fluxes_io(Prim{F}, Prim{K}, C, i, j, which, nwhich);
}

// restru/restrv/restrsc :1474-1740 and fluxes(coarse) :215, one thread per
// (coarse cell, slice `which` of 3)
template <class IO>
__device__ __forceinline__ void cell_restrict_fluxes_io(const IO &F, const IO &K, const CaseDev &C, int ic, int jc,
                                                        int which, int nwhich)
{
    if (which == 0 && ic <= K.L.npx - 2 && jc <= K.L.npy - 2) cell_fluxes_io(K, jc * K.L.npx + ic);
    if (ic >= 1 && jc >= 1 && ic <= K.L.npx - 2 && jc <= K.L.npy - 2)
        for (int w = which; w < 3; w += nwhich) cell_restrict_io(F, K, C, ic, jc, w);
}
__device__ __forceinline__ void cell_restrict_fluxes(const LevelDev &F, const LevelDev &K, const CaseDev &C,
                                                     int ic, int jc, int which, int nwhich)
{
    cell_restrict_fluxes_io(Prim{F}, Prim{K}, C, ic, jc, which, nwhich);
}

__global__ void __launch_bounds__(BLOCK) k_restv_fluxes(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    int i, j;
    if (cell_at(dom_all(L), t, i, j)) cell_restv_fluxes(L, C.lv[ig + 1], C, i, j, blockIdx.z, gridDim.z);
}

// restr{u,v,sc} + fluxes(coarse); with `what` != 0 also the coarse level's first
// down-leg routine (the fused assembly): the defects a coarse cell's assembly reads
// (resu, resv, ressc of that cell) come from the same thread, everything else from
// restv, which finished in the previous launch.
__global__ void __launch_bounds__(BLOCK) k_restrict(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode,
                                                    unsigned what)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (!cell_at(dom_all(K), t, i, j)) return;
    const int z = blockIdx.z, nz = gridDim.z;
    cell_restrict_fluxes(L, K, C, i, j, z, nz);
    if (!what || !mode_active(C, ig + 1, M_DOWN)) return;
    // slice z assembles the equation whose defect it just computed
    const unsigned w = asm_slice(what, z, nz) & ~(unsigned)(A_FLUX | A_SC_OUTFLOW);
    if (w & A_F32) cell_asm_f32(K, C, i, j, w, (what & A_SC_OUTFLOW) && C.ibc_xp == 4);
    else cell_asm(K, C, FluxLive(K), i, j, w);
    if (nz > 1 && z != 2) return;
    // the scalar outflow ghost of an interior row is read by this kernel only in the
    // defect of the cell west of it, so that cell (this thread, after its defect)
    // writes it; ghosts of the boundary rows are read by nobody here
    if ((what & A_SC_OUTFLOW) && C.ibc_xp == 4) {
        double *sc = MGF(K, S_SC);
        const int q = j * K.npx + i;
        if (i == K.npx - 2 && j >= 1 && j <= K.npy - 2) sc[q + 1] = sc[q];
        if (i == K.npx - 1 && (j == 0 || j == K.npy - 1)) sc[q] = sc[q - 1];
    }
}

__global__ void __launch_bounds__(BLOCK) k_prol_corr(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (cell_at(dom_interior(K), t, i, j)) cell_prol_corr(L, K, i, j);
}

template <bool FUSED>
__global__ void __launch_bounds__(BLOCK) k_prol_apply(const CaseDev *__restrict__ cs, CaseState *st, int ig, int mode)
{
    pdl_enter();
    CASE_PROLOGUE(mode);
    const LevelDev &K = C.lv[ig + 1];
    int i, j;
    if (cell_at(dom_interior(L), t, i, j)) cell_prol_apply<FUSED>(L, K, i, j);
}

// End of a V-cycle on the level-0 interior: relative change of u, v, sc and of p
// with its mean removed against the previous cycle, the history entry, the stop
// rule, and prev <- current.  p sums are shifted by the previous cycle's means so a
// uniform pressure drift does not cancel catastrophically.
// The end-of-cycle work for level-0 cell index t of this block (see k_endcycle).
// History entry and the reference's stop test (:247-248) when the fixed-point change is
// not tracked: one thread per case.
__device__ __forceinline__ void end_of_cycle_err_only(const CaseDev &C, CaseState &ST)
{
    const double err = ST.last_err;
    const int k = ST.ncyc;
    if (k < C.hist_cap) {
        C.hist_err[k] = err;
        C.hist_delta[k] = 0.0;
    }
    ST.ncyc = k + 1;
    const bool finite = isfinite(err);
    if (!finite) ST.status |= CASE_NONFINITE;
    if (C.stop_enabled) {
        if (!finite) ST.done = 1;
        else if (err < C.convergence) { ST.done = 1; ST.status |= CASE_CONVERGED_REF; }
    }
    ST.have_prev = 0;
}

// The fixed-point change (four norms over level 0 and their block reduction) is
// computed only while a solve with fp_tol > 0 runs; otherwise the cycle only records
// its mass error.
__device__ __forceinline__ void end_of_cycle(const CaseDev &C, CaseState &ST, int t, int nb)
{
    if (!(C.fp_tol > 0.0)) {
        if (t == 0) end_of_cycle_err_only(C, ST);
        return;
    }
    const LevelDev &L = C.lv[0];
    const Dom d = dom_interior(L);
    const int n = d.wi * d.wj;
    const double kd = ST.shift_d, kp = ST.shift_p;
    double a[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) a[k] = 0.0;
    int i, j;
    if (cell_at(d, t, i, j)) {
        const int q = j * L.npx + i;
        const int cur[3] = {S_U, S_V, S_SC}, prv[3] = {S_PREV_U, S_PREV_V, S_PREV_SC};
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
    const double err = ST.last_err;
    const int k = ST.ncyc;
    const double delta = ST.have_prev ? worst : 0.0;
    if (k < C.hist_cap) {
        C.hist_err[k] = err;
        C.hist_delta[k] = delta;
    }
    ST.ncyc = k + 1;
    ST.shift_d = kd + s[6] / N;
    ST.shift_p = kp + s[8] / N;
    const bool finite = isfinite(err) && isfinite(delta);
    if (!finite) ST.status |= CASE_NONFINITE;
    if (C.stop_enabled) {
        if (!finite) ST.done = 1;
        else if (err < C.convergence) { ST.done = 1; ST.status |= CASE_CONVERGED_REF; }
        else if (C.fp_tol > 0.0 && ST.have_prev && delta < C.fp_tol) { ST.done = 1; ST.status |= CASE_CONVERGED_FP; }
    }
    ST.have_prev = 1;
}

__global__ void __launch_bounds__(BLOCK) k_endcycle(const CaseDev *__restrict__ cs, CaseState *st)
{
    pdl_enter();
    const CaseDev &C = cs[blockIdx.y];
    CaseState &ST = st[blockIdx.y];
    if (ST.done) return;
    const Dom d = dom_interior(C.lv[0]);
    const int n = d.wi * d.wj, nb = (n + blockDim.x - 1) / blockDim.x;
    if ((int)blockIdx.x >= nb) return;
    end_of_cycle(C, ST, blockIdx.x * blockDim.x + threadIdx.x, nb);
}

// prolongation into level 0 followed by the end of the cycle: every thread reads
// back only the level-0 cell it just wrote.
template <bool FUSED>
__global__ void __launch_bounds__(BLOCK) k_prol_apply_end(const CaseDev *__restrict__ cs, CaseState *st, int mode)
{
    pdl_enter();
    const int ig = 0;
    CASE_PROLOGUE(mode);
    const Dom d = dom_interior(L);
    const int n = d.wi * d.wj, nb = (n + blockDim.x - 1) / blockDim.x;
    if ((int)blockIdx.x >= nb) return;
    int i, j;
    if (cell_at(d, t, i, j)) cell_prol_apply<FUSED>(L, C.lv[1], i, j);
    end_of_cycle(C, ST, t, nb);
}

// ------------------------------------------------- one-CTA coarse kernel
template <class F>
__device__ __forceinline__ void for_cells(const Dom &d, F f)
{
    const int n = d.wi * d.wj;
    for (int t = threadIdx.x; t < n; t += blockDim.x) f(d.i0 + t % d.wi, d.j0 + t / d.wi);
}

// Smooth the equations of `mask` on one level, in place in global memory, every
// equation's unit h in the same phase.
template <class IO>
__device__ void tail_smooth_global(const IO &io, const int *eqs, int ne, int nsw, int isolve)
{
    const LevelDev &L = io.L;
    if (isolve == MGFVM_JACOBI) {
        for (int k = 0; k < ne; ++k) {
            const int e = eqs[k];
            const Dom d = dom_eq(L, e);
            const Dom x = {d.i0 - 1, d.j0 - 1, d.wi + 2, d.wj + 2};
            const int phi = eq_field(e), tmp = eq_tmp(e);
            for_cells(x, [&](int i, int j) {
                if (i == x.i0 || i == x.i0 + x.wi - 1 || j == x.j0 || j == x.j0 + x.wj - 1)
                    io.st(tmp, j * L.npx + i, io.ld(phi, j * L.npx + i));
            });
        }
        for (int it = 0; it < nsw; ++it) {
            for (int k = 0; k < ne; ++k) {
                const int e = eqs[k];
                const int phi = eq_field(e), tmp = eq_tmp(e);
                const int cur = (it & 1) ? tmp : phi, nxt = (it & 1) ? phi : tmp;
                for_cells(dom_eq(L, e), [&](int i, int j) { cell_jacobi_io(io, e, cur, nxt, j * L.npx + i); });
            }
            __syncthreads();
        }
        if (nsw & 1) {
            for (int k = 0; k < ne; ++k) {
                const int e = eqs[k];
                const int phi = eq_field(e), tmp = eq_tmp(e);
                for_cells(dom_eq(L, e), [&](int i, int j) { io.st(phi, j * L.npx + i, io.ld(tmp, j * L.npx + i)); });
            }
            __syncthreads();
        }
    } else if (isolve == MGFVM_GAUSS_SEIDEL) {
        for (int h = 0; h < 2 * nsw; ++h) {
            const int colour = h & 1;
            for (int k = 0; k < ne; ++k) {
                const int e = eqs[k];
                const Dom d = dom_eq(L, e);
                const int phi = eq_field(e);
                const int wr = (d.wi + 1) >> 1, n = wr * d.wj;
                for (int t = threadIdx.x; t < n; t += blockDim.x) {
                    const int j = d.j0 + t / wr;
                    const int i = d.i0 + (((d.i0 + j) & 1) != colour ? 1 : 0) + 2 * (t % wr);
                    if (i <= d.i0 + d.wi - 1) cell_gs_io(io, e, phi, j * L.npx + i);
                }
            }
            __syncthreads();
        }
    }
}

// The same sweeps with each equation's field and coefficients staged in shared
// memory for the whole level (indices as in global memory), as many equations at a
// time as `sm_doubles` holds; results are the same bits, only the latency changes.
__device__ void tail_smooth(const LevelDev &L, int mask, int nsw, int isolve, double *sm, int sm_doubles)
{
    int eqs[4], ne = 0;
    for (int e = 0; e < 4; ++e)
        if ((mask >> e) & 1) eqs[ne++] = e;
    if (nsw <= 0 || (isolve != MGFVM_JACOBI && isolve != MGFVM_GAUSS_SEIDEL)) return;
    const int n = L.npx * L.npy, npx = L.npx;
    const int per = isolve == MGFVM_JACOBI ? 8 : 7;
    int k = 0;
    while (k < ne) {
        int g = 0;
        while (k + g < ne && (long long)(g + 1) * per * n <= sm_doubles) ++g;
        if (g == 0) {
            tail_smooth_global(Prim{L}, eqs + k, 1, nsw, isolve);
            ++k;
            continue;
        }
        for (int m = 0; m < g; ++m) {
            const int e = eqs[k + m];
            double *b = sm + (size_t)m * per * n;
            const double *phi = MGF(L, eq_field(e));
            const double *cw = MGF(L, co_slot(e, CK_AW)), *ce = MGF(L, co_slot(e, CK_AE)),
                         *cs_ = MGF(L, co_slot(e, CK_AS)), *cn = MGF(L, co_slot(e, CK_AN)),
                         *cp = MGF(L, co_slot(e, CK_AP)), *cu = MGF(L, co_slot(e, CK_SU));
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                // every load before the first store: the stores may not be moved above them
                const double ph = phi[q], w = cw[q], ea = ce[q], so = cs_[q], no = cn[q], pc = cp[q], s0 = cu[q];
                b[q] = ph;
                b[n + q] = w; b[2 * n + q] = ea; b[3 * n + q] = so;
                b[4 * n + q] = no; b[5 * n + q] = pc; b[6 * n + q] = s0;
                if (per == 8) b[7 * n + q] = ph;
            }
        }
        __syncthreads();
        const int units = isolve == MGFVM_GAUSS_SEIDEL ? 2 * nsw : nsw;
        for (int h = 0; h < units; ++h) {
            for (int m = 0; m < g; ++m) {
                const int e = eqs[k + m];
                const Dom d = dom_eq(L, e);
                double *b = sm + (size_t)m * per * n;
                const double *aw = b + n, *ae = b + 2 * n, *as = b + 3 * n, *an = b + 4 * n, *ap = b + 5 * n,
                             *su = b + 6 * n;
                if (isolve == MGFVM_GAUSS_SEIDEL) {
                    const int colour = h & 1, wr = (d.wi + 1) >> 1, cnt = wr * d.wj;
                    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
                        const int j = d.j0 + t / wr;
                        const int i = d.i0 + (((d.i0 + j) & 1) != colour ? 1 : 0) + 2 * (t % wr);
                        if (i > d.i0 + d.wi - 1) continue;
                        const int q = j * npx + i;
                        b[q] = gs_value(aw[q], ae[q], as[q], an[q], ap[q], su[q], b[q - 1], b[q + 1], b[q - npx],
                                        b[q + npx]);
                    }
                } else {
                    const double *cur = (h & 1) ? b + 7 * n : b;
                    double *nxt = (h & 1) ? b : b + 7 * n;
                    for_cells(d, [&](int i, int j) {
                        const int q = j * npx + i;
                        nxt[q] = jacobi_value(aw[q], ae[q], as[q], an[q], ap[q], su[q], cur[q - 1], cur[q + 1],
                                              cur[q - npx], cur[q + npx], cur[q]);
                    });
                }
            }
            __syncthreads();
        }
        for (int m = 0; m < g; ++m) {
            const int e = eqs[k + m];
            const double *res = sm + (size_t)m * per * n + ((isolve == MGFVM_JACOBI && (units & 1)) ? 7 * n : 0);
            double *phi = MGF(L, eq_field(e));
            for_cells(dom_eq(L, e), [&](int i, int j) { phi[j * npx + i] = res[j * npx + i]; });
        }
        __syncthreads();
        k += g;
    }
}

// The levels of one case as seen by the one-CTA kernel (TanCase: mg_tangent.cuh).
struct PrimCase {
    const CaseDev &C;
    __device__ __forceinline__ Prim io(int ig) const { return Prim{C.lv[ig]}; }
};


// One SIMPLE step on level ig (down leg :201-207, up leg :235-244).  The plain run
// stages each level's smoothing in shared memory where it fits (tail_smooth); the
// tangent run smooths in global memory.
template <class X>
__device__ void tail_step(const X &cx, CaseState &ST, int ig, bool down, const Sched &S, double *sm, int smd)
{
    const CaseDev &C = cx.C;
    const auto io = cx.io(ig);
    using IO = decltype(io);
    constexpr bool plain = std::is_same<typename std::remove_cv<IO>::type, Prim>::value;
    const LevelDev &L = io.L;
    const FluxLiveT<typename std::remove_cv<IO>::type> fl{io};
    const unsigned what = A_FLUX | A_U | A_V | A_SC | (down ? A_SC_OUTFLOW : 0u);
    for_cells(dom_all(L), [&](int i, int j) { cell_asm_io(io, C, fl, i, j, what); });
    __syncthreads();
    const int uvsc[3] = {EQ_U, EQ_V, EQ_SC}, pp[1] = {EQ_PP};
    if constexpr (plain) tail_smooth(L, (1 << EQ_U) | (1 << EQ_V) | (1 << EQ_SC), S.nswpm, S.isolve, sm, smd);
    else tail_smooth_global(io, uvsc, 3, S.nswpm, S.isolve);
    double acc[1] = {0.0};
    for_cells(dom_interior(L), [&](int i, int j) { acc[0] += val(cell_mass_coefp_io(io, C, i, j)); });
    if (ig == 0 && down) {
        block_sum<1>(acc);
        if (threadIdx.x == 0) ST.last_err = acc[0];
    }
    __syncthreads();
    if constexpr (plain) tail_smooth(L, 1 << EQ_PP, S.nswpp, S.isolve, sm, smd);
    else tail_smooth_global(io, pp, 1, S.nswpp, S.isolve);
    for_cells(dom_interior(L), [&](int i, int j) { cell_update_io(io, C, j * L.npx + i); });
    __syncthreads();
    pfix_block_io(io);
    bound_block_io(C, io, down ? 3 : 7);
}

template <class X>
__device__ void tail_restrict(const X &cx, int ig)
{
    const auto F = cx.io(ig), K = cx.io(ig + 1);
    for_cells(dom_all(F.L), [&](int i, int j) { cell_restv_fluxes_io(F, K, cx.C, i, j, 0, 1); });
    __syncthreads();
    for_cells(dom_all(K.L), [&](int i, int j) { cell_restrict_fluxes_io(F, K, cx.C, i, j, 0, 1); });
    __syncthreads();
}

template <class X>
__device__ void tail_prolong(const X &cx, int ig)
{
    const auto F = cx.io(ig), K = cx.io(ig + 1);
    for_cells(dom_interior(K.L), [&](int i, int j) { cell_prol_corr_io(F, K, i, j); });
    __syncthreads();
    for_cells(dom_interior(F.L), [&](int i, int j) { cell_prol_apply_io(F, K, i, j); });
    __syncthreads();
}

template <class X>
__device__ void tail_cycle(const X &cx, CaseState &ST, const Sched &S, double *sm, int smd)
{
    const CaseDev &C = cx.C;
    for (int ig = C.tail; ig < C.ngrid; ++ig) {
        tail_step(cx, ST, ig, true, S, sm, smd);
        if (ig != C.ngrid - 1) tail_restrict(cx, ig);
    }
    for (int ig = C.ngrid - 1; ig > C.tail; --ig) {
        tail_prolong(cx, ig - 1);
        if (ig != 1) tail_step(cx, ST, ig - 1, false, S, sm, smd);
    }
}

// Every level at or below C.tail of one case (blockIdx.x): the down leg from
// C.tail, the restrictions between those levels, and the up leg back to C.tail.
__global__ void __launch_bounds__(TAIL_BLOCK, 1) k_tail(const CaseDev *__restrict__ cs, CaseState *st, Sched S,
                                                        int smem_doubles)
{
    pdl_enter();
    extern __shared__ double tsm[];
    const CaseDev &C = cs[blockIdx.x];
    CaseState &ST = st[blockIdx.x];
    if (ST.done || C.tail >= C.ngrid) return;
    tail_cycle(PrimCase{C}, ST, S, tsm, smem_doubles);
}

// ------------------------------------------------ the coarse levels in one cluster launch
// Everything a V-cycle does from the restriction into level c0 (the first level one
// CTA holds) to the prolongation out of it, as one launch of a cluster of three CTAs
// per case (rank r): restv + fine fluxes and the FAS restriction (:211-220; slice r of
// three, one cluster barrier after each), each down-leg visit (:201-207), the
// prolongations back up (:230-233, the gather forming its corrections from the saved
// R(x_f)) and the up-leg visits (:235-244).  A visit: the assembly (slice r) | barrier |
// u, v, sc smoothing (equation r, in place) | barrier | CTA 0: masserror + coefp, the p'
// units and update (pp_level_body), then the obstacle pressure copy and pbound /
// outflow of the level | barrier.  The kernels it replaces in the same order, so the
// same bits.  Which levels and transfers a case takes follows its mode flags
// (mode_active); every CTA of a cluster sees the same flags and takes the same barriers.
template <int ISOLVE>
__device__ void cl_visit(const CaseDev &C, CaseState &ST, int ig, bool down, int nu, int mu, int r, double *sm)
{
    const LevelDev &L = C.lv[ig];
    const unsigned what = A_FLUX | A_U | A_V | A_SC | (down ? A_SC_OUTFLOW : 0u);
    const unsigned w = asm_slice(what, r, 3);
    const int n = L.npx * L.npy;
    for (int q = threadIdx.x; q < n; q += blockDim.x) cell_asm(L, C, FluxLive(L), q % L.npx, q / L.npx, w);
    cluster_barrier();
    if (mu > 0 && level_smooth_eq<ISOLVE>(L, r == 0 ? EQ_U : r == 1 ? EQ_V : EQ_SC, mu, sm) == 2 &&
        threadIdx.x == 0)
        atomicOr(&ST.status, (int)CASE_BAD_LAUNCH);   // the schedule sizes blocks to fit; never taken
    cluster_barrier();
    if (r == 0) {
        pp_level_body<ISOLVE>(C, ST, L, nu, ig == 0 && down, 0, sm);
        __syncthreads();
        pfix_block_io(Prim{L});
        bound_block_io(C, Prim{L}, down ? 3 : 7);
    }
    cluster_barrier();
}

// restriction ig -> ig + 1 by a cluster: slice r of three over every cell
__device__ void cl_restrict(const CaseDev &C, int ig, int r)
{
    const LevelDev &F = C.lv[ig], &K = C.lv[ig + 1];
    for (int q = threadIdx.x; q < F.npx * F.npy; q += blockDim.x)
        cell_restv_fluxes(F, K, C, q % F.npx, q / F.npx, r, 3);
    cluster_barrier();
    for (int q = threadIdx.x; q < K.npx * K.npy; q += blockDim.x)
        cell_restrict_fluxes(F, K, C, q % K.npx, q / K.npx, r, 3);
    cluster_barrier();
}

// prolongation ig + 1 -> ig by a cluster: the interior cells of level ig split over it
__device__ void cl_prolong(const CaseDev &C, int ig, int r)
{
    const LevelDev &F = C.lv[ig], &K = C.lv[ig + 1];
    const Dom d = dom_interior(F);
    for (int t = r * blockDim.x + threadIdx.x; t < d.wi * d.wj; t += 3 * blockDim.x)
        cell_prol_apply<true>(F, K, d.i0 + t % d.wi, d.j0 + t / d.wi);
    cluster_barrier();
}

template <int ISOLVE>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(SMOOTH_BLOCK, 1)
    k_coarse_cycle(const CaseDev *__restrict__ cs, CaseState *st, int c0, int nu, int mu)
{
    pdl_enter();
    extern __shared__ double sm[];
    const CaseDev &C = cs[blockIdx.y];
    CaseState &ST = st[blockIdx.y];
    if (ST.done) return;   // the same for the three CTAs
    const int r = blockIdx.x;
    if (c0 >= 1 && mode_active(C, c0 - 1, M_RESTRICT)) cl_restrict(C, c0 - 1, r);
    for (int ig = c0; ig < C.ngrid; ++ig) {
        if (mode_active(C, ig, M_DOWN)) cl_visit<ISOLVE>(C, ST, ig, true, nu, mu, r, sm);
        if (mode_active(C, ig, M_RESTRICT)) cl_restrict(C, ig, r);
    }
    for (int ig = C.ngrid - 1; ig >= c0 && ig >= 1; --ig) {
        if (!mode_active(C, ig - 1, M_PROLONG)) continue;
        cl_prolong(C, ig - 1, r);
        if (ig - 1 >= c0 && ig != 1) cl_visit<ISOLVE>(C, ST, ig - 1, false, nu, mu, r, sm);
    }
}

// The same levels with every value paired with its derivative along the case's
// parameter direction (forward mode, mg_tangent.cuh): the value bits are those of
// k_tail, the derivatives those of the same V-cycle.  Two CTAs per SM (64 registers,
// some spilled): a gradient's 258 directions of a 256^2 case then run as one wave on
// 148 SMs instead of 1.7 (27.8 vs 29.5 ms per V-cycle).
__global__ void __launch_bounds__(TAIL_BLOCK, 2) k_tail_tan(const CaseDev *__restrict__ cs, CaseState *st,
                                                            const CaseTan *__restrict__ ts, Sched S)
{
    pdl_enter();
    const CaseDev &C = cs[blockIdx.x];
    CaseState &ST = st[blockIdx.x];
    if (ST.done || C.tail >= C.ngrid) return;
    tail_cycle(TanCase{C, ts[blockIdx.x]}, ST, S, nullptr, 0);
}

// ------------------------------------------------------------- launcher
int smooth_pairs_side(int units, int threads)
{
    int s = 1;
    while ((s + 1) * ((s + 2) / 2) <= threads) ++s;   // largest square region of <= `threads` pairs
    return s - 2 * units;
}

cudaError_t configure_kernels()
{
    cudaError_t e = cudaFuncSetAttribute(k_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, TAIL_SMEM_MAX);
    const void *tma[] = {(const void *)k_smooth_tma<MGFVM_JACOBI, SMOOTH_BLOCK>,
                         (const void *)k_smooth_tma<MGFVM_JACOBI, SMOOTH_BLOCK / 2>,
                         (const void *)k_smooth_tma<MGFVM_JACOBI, SMOOTH_BLOCK / 4>,
                         (const void *)k_smooth_tma<MGFVM_GAUSS_SEIDEL, SMOOTH_BLOCK>,
                         (const void *)k_smooth_tma<MGFVM_GAUSS_SEIDEL, SMOOTH_BLOCK / 2>,
                         (const void *)k_smooth_tma<MGFVM_GAUSS_SEIDEL, SMOOTH_BLOCK / 4>};
    for (const void *f : tma)
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, SMOOTH_TMA_SMEM_MAX);
    const void *band[] = {(const void *)k_band_visit<MGFVM_JACOBI>, (const void *)k_band_visit<MGFVM_GAUSS_SEIDEL>};
    for (const void *f : band)
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, BAND_SMEM_MAX);
    return e;
}

// Launch `k` on `st`, with programmatic stream serialization when `pdl` (the kernel
// may then be scheduled while its predecessor runs; it waits in pdl_enter()).
template <typename... KP, typename... A>
static cudaError_t launch_k(bool pdl, void (*k)(KP...), dim3 g, int b, int smem, cudaStream_t st, A... args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = g;
    c.blockDim = dim3((unsigned)b, 1, 1);
    c.dynamicSmemBytes = (size_t)smem;
    c.stream = st;
    c.attrs = at;
    c.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&c, k, static_cast<KP>(args)...);
}

// launch_k for a kernel whose CTAs form clusters of `cx` along x
template <typename... KP, typename... A>
static cudaError_t launch_cluster(bool pdl, void (*k)(KP...), dim3 g, int b, int smem, cudaStream_t st, int cx,
                                  A... args)
{
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cx;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = g;
    c.blockDim = dim3((unsigned)b, 1, 1);
    c.dynamicSmemBytes = (size_t)smem;
    c.stream = st;
    c.attrs = at;
    c.numAttrs = pdl ? 2 : 1;
    return cudaLaunchKernelEx(&c, k, static_cast<KP>(args)...);
}

template <int ISOLVE>
static cudaError_t launch_smooth_tma(bool pdl, const Launch &X, dim3 g, int b, const CaseDev *dc, CaseState *ds,
                                     int polls, cudaStream_t st)
{
    cudaError_t le;
    const SmoothMap *m = (const SmoothMap *)X.ptr;
    if (b <= SMOOTH_BLOCK / 4)
        le = launch_k(pdl, k_smooth_tma<ISOLVE, SMOOTH_BLOCK / 4>, g, b, X.smem, st, dc, ds, m, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4, X.bw, X.bh, polls);
    else if (b <= SMOOTH_BLOCK / 2)
        le = launch_k(pdl, k_smooth_tma<ISOLVE, SMOOTH_BLOCK / 2>, g, b, X.smem, st, dc, ds, m, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4, X.bw, X.bh, polls);
    else
        le = launch_k(pdl, k_smooth_tma<ISOLVE, SMOOTH_BLOCK>, g, b, X.smem, st, dc, ds, m, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4, X.bw, X.bh, polls);
    return le;
}

// a3 = flags (bit 8: operands before the wait, EARLY)
template <int ISOLVE, bool EARLY>
static cudaError_t launch_smooth_f32(bool pdl, const Launch &X, dim3 g, int b, const CaseDev *dc, CaseState *ds,
                                     cudaStream_t st)
{
    const int f = X.a3 & 7;
    if (b <= SMOOTH_BLOCK / 4)
        return launch_k(pdl, k_smooth_f32<ISOLVE, SMOOTH_BLOCK / 4, EARLY>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, f, X.a4);
    if (b <= SMOOTH_BLOCK / 2)
        return launch_k(pdl, k_smooth_f32<ISOLVE, SMOOTH_BLOCK / 2, EARLY>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, f, X.a4);
    return launch_k(pdl, k_smooth_f32<ISOLVE, SMOOTH_BLOCK, EARLY>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, f, X.a4);
}

template <int ISOLVE, bool EARLY>
static cudaError_t launch_smooth_e(bool pdl, const Launch &X, dim3 g, int b, const CaseDev *dc, CaseState *ds,
                                   int dir, cudaStream_t st)
{
    cudaError_t le;
    if (b <= SMOOTH_BLOCK / 4)
        le = launch_k(pdl, k_smooth<ISOLVE, SMOOTH_BLOCK / 4, EARLY>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, dir, X.a4);
    else if (b <= SMOOTH_BLOCK / 2)
        le = launch_k(pdl, k_smooth<ISOLVE, SMOOTH_BLOCK / 2, EARLY>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, dir, X.a4);
    else
        le = launch_k(pdl, k_smooth<ISOLVE, SMOOTH_BLOCK, EARLY>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, dir, X.a4);
    return le;
}
// a3 bit 4: the coefficients may be read before the wait for the previous launch
template <int ISOLVE>
static cudaError_t launch_smooth(bool pdl, const Launch &X, dim3 g, int b, const CaseDev *dc, CaseState *ds,
                                 cudaStream_t st)
{
    if (X.a3 & 4) return launch_smooth_e<ISOLVE, true>(pdl, X, g, b, dc, ds, X.a3 & 3, st);
    return launch_smooth_e<ISOLVE, false>(pdl, X, g, b, dc, ds, X.a3, st);
}

cudaError_t launch_one(const Launch &X, const CaseDev *dc, CaseState *ds, const CaseTan *dt, const Sched &S,
                       cudaStream_t st)
{
    const dim3 g = X.grid;
    const int b = X.block;
    const bool pdl = S.pdl;
    cudaError_t le = cudaSuccess;
    switch (X.kernel) {
    case K_FLUXES: le = launch_k(pdl, k_fluxes, g, b, 0, st, dc, ds, X.ig, X.mode); break;
    case K_ASM:
        if (X.a1) le = launch_k(pdl, k_asm<1>, g, b, 0, st, dc, ds, X.ig, X.mode, (unsigned)X.a0);
        else le = launch_k(pdl, k_asm<0>, g, b, 0, st, dc, ds, X.ig, X.mode, (unsigned)X.a0);
        break;
    case K_MASS_COEFP:
        if (X.a1 & 8) le = launch_k(pdl, k_mass_coefp<true>, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0, X.a1 & ~8);
        else le = launch_k(pdl, k_mass_coefp<false>, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0, X.a1);
        break;
    case K_UPDATE:
        if (X.a0 & 64) le = launch_k(pdl, k_update<true>, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0 & ~64);
        else le = launch_k(pdl, k_update<false>, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0);
        break;
    case K_PFIX: le = launch_k(pdl, k_pfix, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0); break;
    case K_BOUND: le = launch_k(pdl, k_bound, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0); break;
    case K_SMOOTH:
        if (b > SMOOTH_BLOCK) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI)
            le = launch_smooth<MGFVM_JACOBI>(pdl, X, g, b, dc, ds, st);
        else
            le = launch_smooth<MGFVM_GAUSS_SEIDEL>(pdl, X, g, b, dc, ds, st);
        break;
    case K_SMOOTH_F32:
        if (b > SMOOTH_BLOCK) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI) {
            if (X.a3 & 8) le = launch_smooth_f32<MGFVM_JACOBI, true>(pdl, X, g, b, dc, ds, st);
            else le = launch_smooth_f32<MGFVM_JACOBI, false>(pdl, X, g, b, dc, ds, st);
        } else {
            if (X.a3 & 8) le = launch_smooth_f32<MGFVM_GAUSS_SEIDEL, true>(pdl, X, g, b, dc, ds, st);
            else le = launch_smooth_f32<MGFVM_GAUSS_SEIDEL, false>(pdl, X, g, b, dc, ds, st);
        }
        break;
    case K_COPY: le = launch_k(pdl, k_copy, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0); break;
    case K_SMOOTH_TMA:
        if (b > SMOOTH_BLOCK || !X.ptr || X.smem > SMOOTH_TMA_SMEM_MAX || (X.bw & 1)) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI) le = launch_smooth_tma<MGFVM_JACOBI>(pdl, X, g, b, dc, ds, S.tma_wait_polls, st);
        else le = launch_smooth_tma<MGFVM_GAUSS_SEIDEL>(pdl, X, g, b, dc, ds, S.tma_wait_polls, st);
        break;
    case K_PP_LEVEL:
        if (b > SMOOTH_BLOCK) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI)
            le = launch_k(pdl, k_pp_level<MGFVM_JACOBI>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2);
        else
            le = launch_k(pdl, k_pp_level<MGFVM_GAUSS_SEIDEL>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2);
        break;
    case K_LEVEL_VISIT:
        if (b > SMOOTH_BLOCK || g.x != 3) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI)
            le = launch_k(pdl, k_level_visit<MGFVM_JACOBI>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4);
        else
            le = launch_k(pdl, k_level_visit<MGFVM_GAUSS_SEIDEL>, g, b, X.smem, st, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4);
        break;
    case K_COARSE_CYCLE:
        if (b > SMOOTH_BLOCK || g.x != 3) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI)
            le = launch_k(pdl, k_coarse_cycle<MGFVM_JACOBI>, g, b, X.smem, st, dc, ds, X.a0, X.a1, X.a2);
        else
            le = launch_k(pdl, k_coarse_cycle<MGFVM_GAUSS_SEIDEL>, g, b, X.smem, st, dc, ds, X.a0, X.a1, X.a2);
        break;
    case K_BAND_VISIT:
        if (b > SMOOTH_BLOCK || g.x < 1 || g.x > BAND_MAX_CTAS || X.smem > BAND_SMEM_MAX) return cudaErrorInvalidValue;
        if (S.isolve == MGFVM_JACOBI)
            le = launch_cluster(pdl, k_band_visit<MGFVM_JACOBI>, g, b, X.smem, st, (int)g.x, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4);
        else
            le = launch_cluster(pdl, k_band_visit<MGFVM_GAUSS_SEIDEL>, g, b, X.smem, st, (int)g.x, dc, ds, X.ig, X.mode, X.a0, X.a1, X.a2, X.a3, X.a4);
        break;
    case K_PFIX_BOUND: le = launch_k(pdl, k_pfix_bound, g, b, 0, st, dc, ds, X.ig, X.mode, X.a0); break;
    case K_RESTV_FLUXES: le = launch_k(pdl, k_restv_fluxes, g, b, 0, st, dc, ds, X.ig, X.mode); break;
    case K_RESTRICT: le = launch_k(pdl, k_restrict, g, b, 0, st, dc, ds, X.ig, X.mode, (unsigned)X.a0); break;
    case K_PROL_CORR: le = launch_k(pdl, k_prol_corr, g, b, 0, st, dc, ds, X.ig, X.mode); break;
    case K_PROL_APPLY:
        if (X.a0) le = launch_k(pdl, k_prol_apply<true>, g, b, 0, st, dc, ds, X.ig, X.mode);
        else le = launch_k(pdl, k_prol_apply<false>, g, b, 0, st, dc, ds, X.ig, X.mode);
        break;
    case K_TAIL: le = launch_k(pdl, k_tail, g, b, X.smem, st, dc, ds, S, X.smem / (int)sizeof(double)); break;
    case K_TAIL_TAN:
        if (!dt) return cudaErrorInvalidValue;
        le = launch_k(pdl, k_tail_tan, g, b, 0, st, dc, ds, dt, S);
        break;
    case K_ENDCYCLE: le = launch_k(pdl, k_endcycle, g, b, 0, st, dc, ds); break;
    case K_PROL_APPLY_END:
        if (X.a0) le = launch_k(pdl, k_prol_apply_end<true>, g, b, 0, st, dc, ds, X.mode);
        else le = launch_k(pdl, k_prol_apply_end<false>, g, b, 0, st, dc, ds, X.mode);
        break;
    default: return cudaErrorInvalidValue;
    }
    return le != cudaSuccess ? le : cudaGetLastError();
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
    nxt[q] = jacobi_value(aw[q], ae[q], as[q], an[q], ap[q], su[q], cur[q - 1], cur[q + 1], cur[q - npx],
                          cur[q + npx], cur[q]);
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
    phi[q] = gs_value(aw[q], ae[q], as[q], an[q], ap[q], su[q], phi[q - 1], phi[q + 1], phi[q - npx], phi[q + npx]);
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

// ----------------------------------------------- division self-test
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Operand k: even k draw raw 64-bit patterns (every exponent, subnormals, Inf, NaN,
// signed zeros), odd k draw values with exponents in [-64, 63] like a smoother's.
__device__ __forceinline__ double test_operand(unsigned long long seed, long long k, int which)
{
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)k * 2 + which));
    if ((k & 1) == 0) return __longlong_as_double((long long)h);
    const unsigned long long man = h & 0x000FFFFFFFFFFFFFull, sign = h & 0x8000000000000000ull;
    const long long ex = 1023 + (long long)((h >> 52) & 127) - 64;
    return __longlong_as_double((long long)(sign | ((unsigned long long)ex << 52) | man));
}

__global__ void r_check_division(long long n, unsigned long long seed, unsigned long long *bad)
{
    unsigned long long local = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const double a = test_operand(seed, k, 0), b = test_operand(seed, k, 1);
        const double want = a / b, got = div_by(a, make_recip(b));
        const bool same = __double_as_longlong(want) == __double_as_longlong(got) || (want != want && got != got);
        local += same ? 0 : 1;
    }
    if (local) atomicAdd(bad, local);
}

cudaError_t raw_check_division(long long n, unsigned long long seed, unsigned long long *bad, cudaStream_t s)
{
    r_check_division<<<148 * 8, BLOCK, 0, s>>>(n, seed, bad);
    return cudaGetLastError();
}

}  // namespace mg
