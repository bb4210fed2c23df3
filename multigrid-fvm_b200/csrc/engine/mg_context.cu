// mg_context.cu — the C ABI of include/mgfvm.h on top of the engine's kernels.
//
// A context owns every level of every case of a batch in one device pool, builds
// the launch schedule of one V-cycle (Version-6-26-04.c:195-249) once, captures it
// in a CUDA graph and replays that graph; the stop rule is evaluated on the device
// at the end of every cycle, so the host only polls per-case flags every
// `sync_every` cycles and a converged case costs nothing but early-exiting blocks.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "mg_adjoint.cuh"
#include "mg_init.cuh"
#include "mg_kernels.cuh"
#include "mg_tangent.cuh"
#include "mgfvm_host.h"

#include <cudaTypedefs.h>

using namespace mg;

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return mgfvm_fail(MGFVM_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                              __FILE__, __LINE__);                                               \
    } while (0)

#define RC(call)                   \
    do {                           \
        int r_ = (call);           \
        if (r_ != MGFVM_OK) return r_; \
    } while (0)

static_assert(PFAN_LAST == mg::PFAN_END, "fan-list end marker differs between host and device");
static const int TAIL_AUTO_CELLS = 0;   // automatic choice: grid kernels on every level (measured fastest)
static const int HIST_INITIAL = 4096;

struct mgfvm_ctx {
    int device = 0;
    mgfvm_options opt{};
    int ncases = 0;
    int maxng = 0;
    Sched sched{};
    std::vector<mgfvm_config> cfg;
    std::vector<std::vector<int>> obs;
    std::vector<std::vector<double>> profile;
    std::vector<mgfvm_obstacle_prog> progs;   // ncases * MAXLEV
    std::vector<CaseDev> hc;
    std::vector<CaseState> hs;
    std::vector<InitDev> hinit;
    CaseDev *dc = nullptr;
    CaseState *ds = nullptr;
    InitDev *dinit = nullptr;
    char *pool = nullptr;
    size_t pool_bytes = 0;
    double *hist = nullptr;
    int hist_cap = 0;
    double *dprofile = nullptr;
    int *dobs = nullptr;
    int *hflags = nullptr;                    // pinned readback of the per-case done flags, two sets
    size_t hflags_bytes = 0;
    cudaEvent_t eflag[2] = {nullptr, nullptr};  // completion of each set's copy
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<Launch> cyc;
    std::vector<int> maxcells;                // per level: max npx*npy over cases
    int last_eq[MAXLEV];                      // per level: equation of the visible coefficient set
    mgfvm_tuning tune{};                      // per-level schedule choices (0: default)
    long long launches = 0;
    long long h2d = 0, d2h = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double last_ms = 0.0;
    // tangent contexts (opt.tangent): derivative storage and each case's direction
    char *tpool = nullptr;
    std::vector<size_t> tcase_off, tcase_bytes;   // per case: its part of tpool
    std::vector<CaseTan> ht;
    CaseTan *dt = nullptr;
    std::vector<int> dir_kind, dir_index;
    // tensor maps of the V-cycle's TMA-staged smoother launches (host copy, device table)
    std::vector<SmoothMap> hmaps;
    SmoothMap *dmaps = nullptr;
    std::vector<int> tail0;                   // per case: first one-CTA-kernel level chosen at creation
    std::vector<void *> pooled;               // buffers taken from the device's memory pool
    // the last mgfvm_adjoint: per case J and its gradient (nfy inlet faces, amuf, prsc)
    int adj_cycles = -1;
    std::vector<double> adj_J, adj_gamuf, adj_gprsc;
    std::vector<char> adj_bad;                // the case turned non-finite within the cycles
    std::vector<std::vector<double>> adj_gin;
};

static inline int npx_of(const mgfvm_config &c, int ig) { return c.nfx / (1 << ig) + 2; }
static inline int npy_of(const mgfvm_config &c, int ig) { return c.nfy / (1 << ig) + 2; }
static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static inline int nblk(long long n) { return (int)std::max<long long>(1, (n + BLOCK - 1) / BLOCK); }

// ------------------------------------------------------------------ schedule
namespace {

// cuTensorMapEncodeTiled from the driver (through the runtime: no link to libcuda), or
// nullptr where the driver does not provide it
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        cudaGetLastError();
    }
    return fn;
}

// The two tensor maps of a TMA-staged smoother launch on level L with a bw x bh box:
// the level's first NSLOTS_LEVEL slot arrays as an (x, y, slot) tensor.  False where
// the layout does not allow it (slots not at one stride, a row not a multiple of 16
// bytes) or the encoder refuses.
static bool encode_smooth_maps(const LevelDev &L, int bw, int bh, SmoothMap &m)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || !L.f[0] || !L.f[1] || (bw & 1) || bw > 256 || bh > 256) return false;
    const char *base = (const char *)L.f[0];
    const long long stride = (const char *)L.f[1] - base;
    for (int s = 0; s < NSLOTS_LEVEL; ++s)
        if (!L.f[s] || (const char *)L.f[s] - base != s * stride) return false;
    const long long row = (long long)L.npx * (long long)sizeof(double);
    if (row % 16 || stride % 16 || stride < row * L.npy || ((uintptr_t)base & 15)) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)L.npx, (cuuint64_t)L.npy, (cuuint64_t)NSLOTS_LEVEL};
    const cuuint64_t strides[2] = {(cuuint64_t)row, (cuuint64_t)stride};
    const cuuint32_t boxc[3] = {(cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)NCOEF};
    const cuuint32_t boxf[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1u};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    return enc(&m.coef, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, boxc, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
           enc(&m.field, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, boxf, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct Builder {
    mgfvm_ctx *x;
    std::vector<Launch> *out;
    std::vector<SmoothMap> *maps = nullptr;               // where TMA-staged launches may be emitted
    std::map<std::tuple<int, int, int>, int> map_index{};   // (level, bw, bh) -> first map of its cases

    // index of the per-case tensor maps of a (level, box) shape, or -1 where some case's
    // level cannot be staged by TMA
    int smooth_maps(int ig, int bw, int bh)
    {
        const auto key = std::make_tuple(ig, bw, bh);
        auto it = map_index.find(key);
        if (it != map_index.end()) return it->second;
        const int base = (int)maps->size();
        std::vector<SmoothMap> m(x->ncases);
        bool ok = true;
        for (int c = 0; c < x->ncases && ok; ++c) {
            std::memset(&m[c], 0, sizeof(SmoothMap));
            if (ig < x->cfg[c].ngrid) ok = encode_smooth_maps(x->hc[c].lv[ig], bw, bh, m[c]);
        }
        const int idx = ok ? base : -1;
        if (ok) maps->insert(maps->end(), m.begin(), m.end());
        map_index[key] = idx;
        return idx;
    }

    bool any(int ig, int mode) const
    {
        for (const CaseDev &C : x->hc)
            if (mode_active(C, ig, mode)) return true;
        return false;
    }
    Launch &add(int kernel, int ig, int mode, long long cells, int a0 = 0, int a1 = 0, int a2 = 0, int a3 = 0)
    {
        Launch L{};
        L.kernel = kernel; L.ig = ig; L.mode = mode; L.a0 = a0; L.a1 = a1; L.a2 = a2; L.a3 = a3;
        L.grid = dim3(nblk(cells), x->ncases);
        L.block = BLOCK;
        out->push_back(L);
        return out->back();
    }
    long long cells(int ig) const { return ig < (int)x->maxcells.size() ? x->maxcells[ig] : 0; }
    long long tiles(int ig, int tile) const
    {
        long long m = 0;
        for (const mgfvm_config &c : x->cfg)
            if (ig < c.ngrid) {
                const long long w = npx_of(c, ig) - 2, h = npy_of(c, ig) - 2;
                m = std::max(m, ((w + tile - 1) / tile) * ((h + tile - 1) / tile));
            }
        return std::max<long long>(m, 1);
    }
    // Whether one CTA per (case, equation) holds the level: its padded grid has at
    // most SMOOTH_BLOCK vertical cell pairs in every case.
    bool whole_level(int ig, int &mx, int &my) const
    {
        mx = my = 0;
        for (const mgfvm_config &c : x->cfg)
            if (ig < c.ngrid) {
                mx = std::max(mx, npx_of(c, ig));
                my = std::max(my, npy_of(c, ig));
            }
        return mx > 0 && mx * ((my + 1) / 2) <= SMOOTH_BLOCK;
    }
    // Whether a cluster of G <= BAND_MAX_CTAS CTAs per case holds the level in bands of
    // rows (k_band_visit): one thread per interior column and vertical cell pair of a
    // band, the band and its halo rows in shared memory, for the largest case.
    bool band_level(int ig, int &G, int &block, int &smem) const
    {
        int mx = 0, my = 0;
        for (const mgfvm_config &c : x->cfg)
            if (ig < c.ngrid) {
                mx = std::max(mx, npx_of(c, ig));
                my = std::max(my, npy_of(c, ig));
            }
        if (mx < 3 || my < 3) return false;
        const int wc = mx - 2, rows = my - 2;
        const int b0 = (2 * SMOOTH_BLOCK / wc) & ~1;   // rows of a band that SMOOTH_BLOCK threads cover
        if (b0 < 2) return false;
        G = (rows + b0 - 1) / b0;
        if (G > BAND_MAX_CTAS) return false;
        const int b = band_rows(my, G);
        block = round32(wc * (b / 2));
        smem = (x->sched.isolve == MGFVM_JACOBI ? 2 : 1) * (b + 2) * mx * (int)sizeof(double);
        return block <= SMOOTH_BLOCK && smem <= BAND_SMEM_MAX;
    }
    static int round32(int n) { return std::max(32, (n + 31) / 32 * 32); }
    int min_ngrid() const
    {
        int m = MAXLEV;
        for (const mgfvm_config &c : x->cfg) m = std::min(m, c.ngrid);
        return m;
    }
    // `nsw` sweeps of the equations in `mask`.  A level that fits one CTA runs every
    // unit (half-sweep of red-black GS, sweep of Jacobi) in one in-place launch;
    // otherwise the units go in an even number of tile launches of at most the level's
    // cap each, alternating field -> buffer -> field (a single launch copies back).
    // `tmp_ok`: the next kernel can take the result from the ping-pong buffers, so an
    // odd number of tile launches needs no copy back.  Returns whether it is left there.
    // Mixed precision runs on the V-cycle's levels smoothed in tiles, every level but
    // the coarsest (a whole level one CTA holds, and a level of band visits, stays FP64:
    // its visits are latency-bound single launches): FP32 operands and corrections
    // (k_smooth_f32).
    bool f32_level(int ig, int mode) const
    {
        int mx, my, G, blk, smem;
        return x->opt.precision == MGFVM_PREC_MIXED && mode != M_OP && ig < min_ngrid() - 1 &&
               !whole_level(ig, mx, my) && !band_visits(ig, mode, G, blk, smem);
    }
    // Whether the visits to level ig run as band visits (k_band_visit, FP64 in either
    // precision): the level fits a cluster and the tuning asks for them, or leaves it
    // to the default, which takes them for batches of at least BAND_MIN_CASES cases
    // that all have the level at one size (a launch is shaped for its largest case, so
    // smaller ones would leave most of their clusters' threads idle).
    bool band_visits(int ig, int mode, int &G, int &blk, int &smem) const
    {
        const int isolve = x->sched.isolve, t = x->tune.band_visit[ig];
        int mx, my;
        return mode != M_OP && x->sched.nswpp > 0 && t != 1 &&
               (isolve == MGFVM_JACOBI || isolve == MGFVM_GAUSS_SEIDEL) && !whole_level(ig, mx, my) &&
               band_level(ig, G, blk, smem) &&
               (t == 2 || (x->ncases >= BAND_MIN_CASES && one_size(ig, mx, my)));
    }
    // every case that has level ig has it at mx x my
    bool one_size(int ig, int mx, int my) const
    {
        for (const mgfvm_config &c : x->cfg)
            if (ig < c.ngrid && (npx_of(c, ig) != mx || npy_of(c, ig) != my)) return false;
        return true;
    }
    int f32_buf = 0;   // the FP32 correction buffer the last F32 smoothing call ended in
    bool smooth(int ig, int mode, int mask, int nsw, bool tmp_ok = false)
    {
        const int isolve = x->sched.isolve;
        const int units = isolve == MGFVM_GAUSS_SEIDEL ? 2 * nsw : nsw;
        if (units <= 0 || (isolve != MGFVM_JACOBI && isolve != MGFVM_GAUSS_SEIDEL)) return false;
        const int neq = __builtin_popcount((unsigned)mask);
        const int bufs = isolve == MGFVM_JACOBI ? 2 : 1;
        const int kern = K_SMOOTH;
        auto smem_for = [&](int cells) { return bufs * cells * (int)sizeof(double); };
        if (f32_level(ig, mode)) {
            // launches of at most the level's cap of units; the correction passes between
            // them in FP32 and the last adds it to the field, so any count works
            const int tt = x->tune.smooth_threads[ig];
            const int nt = tt == SMOOTH_BLOCK / 2 || tt == SMOOTH_BLOCK / 4 ? tt : SMOOTH_BLOCK;
            const int most = (smooth_pairs_side(0, nt) - MIN_TILE) / 2;
            const int cap = std::min(most, x->tune.smooth_units[ig] > 0 ? x->tune.smooth_units[ig] : MAX_UNITS);
            const int chunks = (units + cap - 1) / cap;
            const int hmax = (units + chunks - 1) / chunks;
            const int tile = smooth_pairs_side(hmax, nt);
            const int side = tile + 2 * hmax;
            int u0 = 0;
            for (int c = 0; c < chunks; ++c) {
                const int nu = units / chunks + (c < units % chunks ? 1 : 0);
                // bit 8: a later launch reads its operands before waiting for the one before it
                const int flags = (c == 0 ? 1 : 0) | (c == chunks - 1 ? 2 : 0) | ((c & 1) ? 4 : 0) |
                                  (c > 0 && x->sched.pdl ? 8 : 0);
                Launch &L = add(K_SMOOTH_F32, ig, mode, 0, mask, u0, nu, flags);
                L.a4 = tile;
                L.grid = dim3((unsigned)tiles(ig, tile), x->ncases, neq);
                L.block = std::min(nt, round32(side * ((side + 1) / 2)));
                L.smem = bufs * side * side * (int)sizeof(float);
                u0 += nu;
            }
            f32_buf = chunks & 1;
            return false;
        }
        int mx, my;
        if (whole_level(ig, mx, my)) {
            Launch &L = add(kern, ig, mode, 0, mask, 0, units, 2);
            L.a4 = std::max(mx, my);
            L.grid = dim3(1, x->ncases, neq);
            L.block = round32(mx * ((my + 1) / 2));
            L.smem = smem_for(mx * my);
            return false;
        }
        const int tt = x->tune.smooth_threads[ig];
        const int nt = tt == SMOOTH_BLOCK / 2 || tt == SMOOTH_BLOCK / 4 ? tt : SMOOTH_BLOCK;
        const int most = (smooth_pairs_side(0, nt) - MIN_TILE) / 2;   // units that leave a MIN_TILE tile
        const int cap = std::min(most, x->tune.smooth_units[ig] > 0 ? x->tune.smooth_units[ig] : MAX_UNITS);
        int chunks = (units + cap - 1) / cap;
        if ((chunks & 1) && units >= chunks + 1 && !tmp_ok) ++chunks;
        const int hmax = (units + chunks - 1) / chunks;
        const int tile = smooth_pairs_side(hmax, nt);
        const int side = tile + 2 * hmax;
        // TMA staging: a box one column wider than the region where it starts at an odd x
        const int bw = (side + 2) & ~1, bh = side;
        const int tma_smem = (NCOEF + 1 + bufs - 1) * bw * bh * (int)sizeof(double);
        const int mi = maps && kern == K_SMOOTH && mode != M_OP && x->tune.smooth_tma[ig] == 2 &&
                               tma_smem <= SMOOTH_TMA_SMEM_MAX
                           ? smooth_maps(ig, bw, bh)
                           : -1;
        int u0 = 0;
        for (int c = 0; c < chunks; ++c) {
            const int nu = units / chunks + (c < units % chunks ? 1 : 0);
            // a later launch reads its coefficients before waiting for the one before it
            const int early = mi < 0 && c > 0 && x->sched.pdl ? 4 : 0;
            Launch &L = add(mi >= 0 ? K_SMOOTH_TMA : kern, ig, mode, 0, mask, u0, nu, (c & 1) | early);
            L.a4 = tile;
            L.grid = dim3((unsigned)tiles(ig, tile), x->ncases, neq);
            L.block = std::min(nt, round32(side * ((side + 1) / 2)));
            L.smem = mi >= 0 ? tma_smem : smem_for(side * side);
            if (mi >= 0) { L.bw = bw; L.bh = bh; L.map = mi; }
            u0 += nu;
        }
        if (chunks & 1) {
            if (tmp_ok) return true;
            Launch &L = add(K_COPY, ig, mode, cells(ig), mask);
            L.grid.z = neq;
        }
        return false;
    }
    void pfix(int ig, int mode)
    {
        int maxcopy = 0, haz = 0;
        for (int c = 0; c < x->ncases; ++c) {
            if (!mode_active(x->hc[c], ig, mode)) continue;
            const mgfvm_obstacle_prog &P = x->progs[c * MAXLEV + ig];
            maxcopy = std::max(maxcopy, P.ncopy);
            haz |= P.hazard;
        }
        if (maxcopy == 0) return;
        if (haz) { add(K_PFIX, ig, mode, maxcopy, 0); add(K_PFIX, ig, mode, maxcopy, 1); }
        else add(K_PFIX, ig, mode, maxcopy, 2);
    }
    // pbound + outflow (bits as k_bound); skipped when no case has such a boundary
    void bound(int ig, int mode, int bits)
    {
        if (!bound_needed(bits)) return;
        Launch &L = add(K_BOUND, ig, mode, 1, bits);
        L.grid = dim3(1, x->ncases);
    }
    // Can outflow run inside update on this level?  Not if pbound (periodic) or the
    // obstacle pressure copy sits between them on the outlet columns for any case.
    bool outflow_fusable(int ig, int mode, bool pfix_in_update) const
    {
        for (int c = 0; c < x->ncases; ++c) {
            const CaseDev &C = x->hc[c];
            if (!mode_active(C, ig, mode)) continue;
            if (C.ibc_xm == 3 || C.ibc_ym == 3) return false;
            if (!pfix_in_update && x->progs[(size_t)c * MAXLEV + ig].touches_outlet) return false;
        }
        return true;
    }
    // Can update do the obstacle pressure copy itself?  Every active case's copy program
    // on the level is empty or has no chained copies (fan lists built).
    bool pfix_fusable(int ig, int mode) const
    {
        if (x->tune.update_pfix[ig] == 1) return false;
        for (int c = 0; c < x->ncases; ++c) {
            if (!mode_active(x->hc[c], ig, mode)) continue;
            const LevelDev &L = x->hc[c].lv[ig];
            if (L.ncopy > 0 && !L.pcode) return false;
        }
        return true;
    }
    // Whether the launch about to be added follows a smoother launch (or the copy back
    // of its buffers), with programmatic dependent launch on: masserror+coefp and update
    // then read the operands that smoothers do not write before waiting for it.
    bool after_smoother(int mode) const
    {
        if (!x->sched.pdl || mode == M_OP || out->empty()) return false;
        const int k = out->back().kernel;
        return k == K_SMOOTH || k == K_SMOOTH_F32 || k == K_SMOOTH_TMA || k == K_COPY;
    }
    // returns the update's fuse bits (0: outflow still to do)
    // `bound_bits` != 0: pbound/outflow follow the obstacle pressure copy (k_bound bits);
    // when both have work they run as one kernel, one CTA per case.
    // `uvsc_in_tmp`: the preceding u, v, sc smoothing left its results in the buffers
    int solve_pp(int ig, int mode, bool reduce, int fuse, int bound_bits = 0, bool uvsc_in_tmp = false)
    {
        // mixed precision: p' operands and p' itself in FP32 (p' needs a smoothing to be set)
        const bool f32 = f32_level(ig, mode) && x->sched.nswpp > 0;
        const int jac = x->sched.isolve == MGFVM_JACOBI ? 4 : 0;
        add(K_MASS_COEFP, ig, mode, cells(ig), reduce ? 1 : 0,
            (uvsc_in_tmp ? 1 : 0) | (f32 ? 2 | jac : 0) | (after_smoother(mode) ? 8 : 0));
        const bool chain = mode != M_OP && x->tune.odd_chunks[ig] != 1;
        if (smooth(ig, mode, 1 << EQ_PP, x->sched.nswpp, chain)) fuse |= 8;
        if (f32) fuse |= 16 | (f32_buf ? 32 : 0);
        add(K_UPDATE, ig, mode, cells(ig) + 2, fuse | (after_smoother(mode) ? 64 : 0));
        return after_update(ig, mode, fuse, bound_bits);
    }
    // the obstacle pressure copy (unless update did it: fuse bit 4) and pbound/outflow
    int after_update(int ig, int mode, int fuse, int bound_bits)
    {
        if (fuse & 4) {                       // the copy ran inside update
            if (bound_bits) bound(ig, mode, bound_bits);
            return fuse;
        }
        if (bound_bits && bound_needed(bound_bits) && pfix_needed(ig, mode)) {
            Launch &L = add(K_PFIX_BOUND, ig, mode, 1, bound_bits);
            L.grid = dim3(1, x->ncases);
            L.block = PFIX_BOUND_BLOCK;
            return fuse;
        }
        pfix(ig, mode);
        if (bound_bits) bound(ig, mode, bound_bits);
        return fuse;
    }
    bool pfix_needed(int ig, int mode) const
    {
        for (int c = 0; c < x->ncases; ++c)
            if (mode_active(x->hc[c], ig, mode) && x->progs[c * MAXLEV + ig].ncopy > 0) return true;
        return false;
    }
    bool bound_needed(int bits) const
    {
        bool need = false;
        for (const CaseDev &C : x->hc)
            need |= ((bits & 1) && (C.ibc_xm == 3 || C.ibc_ym == 3)) || ((bits & 6) && C.ibc_xp == 4);
        return need;
    }
    // One SIMPLE step (down leg :201-207, up leg :235-244).  u, v and sc depend only
    // on the visit-start fluxes, so they are assembled together and smoothed in the
    // same launches; the scalar's outflow ghost moves with its equation.
    static int asm_bits(bool down) { return A_FLUX | A_U | A_V | A_SC | (down ? A_SC_OUTFLOW : 0); }
    // Assembly and restriction run one thread per (cell, equation) — 3 slices, each
    // with a third of the dependent loads — unless tuned to one thread per cell.
    static int slices(int, int knob) { return knob == 1 ? 1 : 3; }
    // the assembly bits of a down-leg (or up-leg) step on level ig, with the FP32
    // operands of a mixed-precision level
    int asm_what(int ig, int mode, bool down) const
    {
        if (!f32_level(ig, mode)) return asm_bits(down);
        return asm_bits(down) | A_F32 | (x->sched.isolve == MGFVM_JACOBI ? A_JAC : 0);
    }
    void step(int ig, int mode, bool down, bool reduce, bool asm_done = false)
    {
        int mx, my;
        const int isolve = x->sched.isolve;
        const int ppu = isolve == MGFVM_GAUSS_SEIDEL ? 2 * x->sched.nswpp : x->sched.nswpp;
        const int mu = isolve == MGFVM_GAUSS_SEIDEL ? 2 * x->sched.nswpm : x->sched.nswpm;
        if (mode != M_OP && ppu > 0 && x->tune.pp_level[ig] != 1 &&
            (isolve == MGFVM_JACOBI || isolve == MGFVM_GAUSS_SEIDEL) && whole_level(ig, mx, my)) {
            // the whole visit (assembly, u/v/sc smoothing, p' and update) in one launch
            const bool pfx = pfix_fusable(ig, mode);
            const int fuse = outflow_fusable(ig, mode, pfx) ? (down ? 1 : 3) : 0;
            const int what = asm_done ? 0 : (int)asm_bits(down);
            const bool visit = what != 0 || mu > 0;
            // the pressure copy and pbound / outflow left after update run in the same
            // CTA (pp_level_tail) instead of the launches after_update would add
            const int bb = fuse ? 0 : (down ? 3 : 7);
            const int tail = (!pfx && pfix_needed(ig, mode) ? 128 : 0) | (bb && bound_needed(bb) ? bb << 8 : 0);
            Launch &L = add(visit ? K_LEVEL_VISIT : K_PP_LEVEL, ig, mode, 0, ppu, reduce ? 1 : 0,
                            fuse | (pfx ? 4 : 0) | tail, what);
            L.a4 = std::max(mu, 0);
            L.grid = dim3(visit ? 3 : 1, x->ncases);
            L.block = round32(mx * ((my + 1) / 2));
            L.smem = (isolve == MGFVM_JACOBI ? 2 : 1) * mx * my * (int)sizeof(double);
            return;
        }
        int G, blk, smem;
        if (band_visits(ig, mode, G, blk, smem)) {
            // the whole visit in one launch of a cluster of G CTAs per case
            const bool pfx = pfix_fusable(ig, mode);
            const int fuse = outflow_fusable(ig, mode, pfx) ? (down ? 1 : 3) : 0;
            Launch &L = add(K_BAND_VISIT, ig, mode, 0, ppu, reduce ? 1 : 0, fuse | (pfx ? 4 : 0),
                            asm_done ? 0 : (int)asm_bits(down));
            L.a4 = std::max(mu, 0);
            L.grid = dim3(G, x->ncases);
            L.block = blk;
            L.smem = smem;
            after_update(ig, mode, fuse | (pfx ? 4 : 0), fuse ? 0 : (down ? 3 : 7));
            return;
        }
        if (!asm_done) {
            Launch &L = add(K_ASM, ig, mode, cells(ig), asm_what(ig, mode, down), 1);
            L.grid.z = slices(ig, x->tune.asm_slices[ig]);
        }
        const bool in_tmp = smooth(ig, mode, (1 << EQ_U) | (1 << EQ_V) | (1 << EQ_SC), x->sched.nswpm,
                                   x->tune.odd_chunks[ig] != 1);
        const bool pfx = pfix_fusable(ig, mode);
        const int fuse = outflow_fusable(ig, mode, pfx) ? (down ? 1 : 3) : 0;
        solve_pp(ig, mode, reduce, fuse | (pfx ? 4 : 0), fuse ? 0 : (down ? 3 : 7), in_tmp);
    }
    // :211-220
    // `coarse_asm`: also run the coarse level's down-leg assembly (see k_restrict)
    void restrict_(int ig, int mode_f, bool coarse_asm = false)
    {
        const int z = slices(ig, x->tune.restrict_slices[ig]);
        add(K_RESTV_FLUXES, ig, mode_f, cells(ig)).grid.z = z;
        Launch &L = add(K_RESTRICT, ig, mode_f, cells(ig + 1), coarse_asm ? asm_what(ig + 1, M_DOWN, true) : 0);
        L.grid.z = z;
    }
    // :230-233
    // In a V-cycle the gather may form the coarse corrections from the R(x_f) that the
    // restriction saved (the fine level has not changed since), unless tuned off.
    void prolong(int ig, int mode)
    {
        const bool fused = mode == M_PROLONG && x->tune.prol_fused[ig] != 1;
        if (!fused) add(K_PROL_CORR, ig, mode, cells(ig + 1));
        add(K_PROL_APPLY, ig, mode, cells(ig), fused ? 1 : 0);
    }
    // The first level of the coarse cluster launch (k_coarse_cycle, when the tuning asks
    // for it): the first level one CTA per case holds, when every level from there down
    // is run by the V-cycle's
    // grid kernels (no one-CTA coarse kernel, no tangent), takes whole-level visits
    // (pp_level), the smoother is GS or Jacobi and p' is smoothed; x->maxng when there
    // is none.
    int coarse_from() const
    {
        if (x->tune.coarse_cluster != 2 || x->opt.tangent || x->sched.nswpp <= 0 ||
            (x->sched.isolve != MGFVM_JACOBI && x->sched.isolve != MGFVM_GAUSS_SEIDEL))
            return x->maxng;
        for (const CaseDev &C : x->hc)
            if (C.tail < C.ngrid) return x->maxng;
        for (int ig = 0; ig < x->maxng; ++ig) {
            int mx, my;
            if (!whole_level(ig, mx, my)) continue;
            for (int k = ig; k < x->maxng; ++k)
                if (x->tune.pp_level[k] == 1) return x->maxng;   // whole-level visits turned off
            return ig;
        }
        return x->maxng;
    }
    void cycle()
    {
        bool asm_done = false;
        const int c0 = coarse_from();
        for (int ig = 0; ig < c0; ++ig) {
            if (any(ig, M_DOWN)) step(ig, M_DOWN, true, ig == 0, asm_done);
            asm_done = false;
            if (ig + 1 < c0 && any(ig, M_RESTRICT)) {
                asm_done = any(ig + 1, M_DOWN);
                restrict_(ig, M_RESTRICT, asm_done);
            }
        }
        if (c0 < x->maxng) {
            // the rest of the down leg, the coarse levels and the up leg back into c0 - 1
            int mx, my;
            whole_level(c0, mx, my);
            const int isolve = x->sched.isolve;
            Launch L{};
            L.kernel = K_COARSE_CYCLE;
            L.ig = c0;
            L.a0 = c0;
            L.a1 = isolve == MGFVM_GAUSS_SEIDEL ? 2 * x->sched.nswpp : x->sched.nswpp;
            L.a2 = std::max(0, isolve == MGFVM_GAUSS_SEIDEL ? 2 * x->sched.nswpm : x->sched.nswpm);
            L.grid = dim3(3, x->ncases);
            L.block = SMOOTH_BLOCK;
            L.smem = (isolve == MGFVM_JACOBI ? 2 : 1) * mx * my * (int)sizeof(double);
            out->push_back(L);
            if (c0 >= 2 && any(c0 - 1, M_PROLONG)) step(c0 - 1, M_UP, false, false);
        }
        bool tail = false;
        for (const CaseDev &C : x->hc) tail |= C.tail < C.ngrid;
        if (tail) {
            // shared memory: every equation of the largest coarse-kernel level at once
            long long need = 0;
            for (int c = 0; c < x->ncases; ++c) {
                const CaseDev &C = x->hc[c];
                if (C.tail < C.ngrid)
                    need = std::max<long long>(need, 24LL * npx_of(x->cfg[c], C.tail) * npy_of(x->cfg[c], C.tail) *
                                                         (long long)sizeof(double));
            }
            Launch L{};
            L.kernel = x->opt.tangent ? K_TAIL_TAN : K_TAIL; L.grid = dim3(x->ncases); L.block = TAIL_BLOCK;
            L.smem = x->opt.tangent ? 0 : (int)std::min<long long>(need, TAIL_SMEM_MAX);
            out->push_back(L);
        }
        for (int ig = std::min(x->maxng, c0) - 1; ig > 0; --ig) {
            if (!any(ig - 1, M_PROLONG)) continue;
            prolong(ig - 1, M_PROLONG);
            if (ig != 1) step(ig - 1, M_UP, false, false);
        }
        // the final prolongation into level 0 can carry the end-of-cycle norms when
        // every case reaches level 0 through it
        bool fuse_end = !out->empty() && out->back().kernel == K_PROL_APPLY && out->back().ig == 0;
        for (const CaseDev &C : x->hc) fuse_end &= C.ngrid >= 2 && C.tail >= 1;
        if (fuse_end) {
            out->back().kernel = K_PROL_APPLY_END;
            return;
        }
        Launch L{};
        L.kernel = K_ENDCYCLE;
        long long n0 = 0;
        for (const mgfvm_config &c : x->cfg)
            n0 = std::max<long long>(n0, (long long)(npx_of(c, 0) - 2) * (npy_of(c, 0) - 2));
        L.grid = dim3(nblk(n0), x->ncases);
        L.block = BLOCK;
        out->push_back(L);
    }
    void op(int op, int ig)
    {
        switch (op) {
        case MGFVM_OP_FLUXES: add(K_FLUXES, ig, M_OP, cells(ig)); break;
        case MGFVM_OP_SOLVE_U:
            add(K_ASM, ig, M_OP, cells(ig), A_U, 0);
            smooth(ig, M_OP, 1 << EQ_U, x->sched.nswpm);
            break;
        case MGFVM_OP_SOLVE_V:
            add(K_ASM, ig, M_OP, cells(ig), A_V, 0);
            smooth(ig, M_OP, 1 << EQ_V, x->sched.nswpm);
            break;
        case MGFVM_OP_SOLVE_PP: solve_pp(ig, M_OP, true, 0); break;
        case MGFVM_OP_PBOUND: bound(ig, M_OP, 1); break;
        case MGFVM_OP_OUTFLOW: bound(ig, M_OP, 6); break;
        case MGFVM_OP_SOLVE_SC:
            add(K_ASM, ig, M_OP, cells(ig), A_SC, 0);
            smooth(ig, M_OP, 1 << EQ_SC, x->sched.nswpm);
            break;
        case MGFVM_OP_RESTRICT: restrict_(ig, M_OP_PAIR); break;
        case MGFVM_OP_PROLONG: prolong(ig, M_OP_PAIR); break;
        case MGFVM_OP_SMOOTH_U: smooth(ig, M_OP, 1 << EQ_U, x->sched.nswpm); break;
        case MGFVM_OP_SMOOTH_V: smooth(ig, M_OP, 1 << EQ_V, x->sched.nswpm); break;
        case MGFVM_OP_SMOOTH_PP: smooth(ig, M_OP, 1 << EQ_PP, x->sched.nswpp); break;
        case MGFVM_OP_SMOOTH_SC: smooth(ig, M_OP, 1 << EQ_SC, x->sched.nswpm); break;
        default: break;
        }
    }
};

// Equation whose coefficient set a single-step op leaves as "the" coefficient arrays
// (the reference has one set that every assembly overwrites); -1: unchanged.
int op_equation(int op)
{
    switch (op) {
    case MGFVM_OP_SOLVE_U: return EQ_U;
    case MGFVM_OP_SOLVE_V: return EQ_V;
    case MGFVM_OP_SOLVE_PP: return EQ_PP;
    case MGFVM_OP_SOLVE_SC: return EQ_SC;
    default: return -1;
    }
}

// Slot holding the reference field `f` on a level whose last assembled equation is `eq`.
int field_slot(int f, int eq)
{
    switch (f) {
    case MGFVM_F_U: return S_U;
    case MGFVM_F_V: return S_V;
    case MGFVM_F_P: return S_P;
    case MGFVM_F_PP: return S_PP;
    case MGFVM_F_SC: return S_SC;
    case MGFVM_F_SU: return co_slot(eq, CK_SU);
    case MGFVM_F_RS: return S_RS;
    case MGFVM_F_RESU: return S_RESU;
    case MGFVM_F_RESV: return S_RESV;
    case MGFVM_F_RESSC: return S_RESSC;
    case MGFVM_F_C: return S_C;
    case MGFVM_F_AW: return co_slot(eq, CK_AW);
    case MGFVM_F_AE: return co_slot(eq, CK_AE);
    case MGFVM_F_AS: return co_slot(eq, CK_AS);
    case MGFVM_F_AN: return co_slot(eq, CK_AN);
    case MGFVM_F_AP: return co_slot(eq, CK_AP);
    case MGFVM_F_APU: return S_APU;
    case MGFVM_F_APV: return S_APV;
    case MGFVM_F_SPU: return S_SPU;
    case MGFVM_F_SPV: return S_SPV;
    case MGFVM_F_SPSC: return S_SPSC;
    case MGFVM_F_CX: return S_CX;
    case MGFVM_F_CY: return S_CY;
    case MGFVM_F_AREAX: return S_AREAX;
    case MGFVM_F_AREAY: return S_AREAY;
    default: return -1;
    }
}

int run_list(mgfvm_ctx *x, const std::vector<Launch> &v)
{
    for (const Launch &L : v) {
        cudaError_t e = launch_one(L, x->dc, x->ds, x->dt, x->sched, x->stream);
        if (e != cudaSuccess)
            return mgfvm_fail(MGFVM_ECUDA, "kernel %d at level %d failed to launch: %s", L.kernel, L.ig,
                              cudaGetErrorString(e));
    }
    x->launches += (long long)v.size();
    return MGFVM_OK;
}

int pull(mgfvm_ctx *x)
{
    CK(cudaStreamSynchronize(x->stream));
    CK(cudaMemcpy(x->hs.data(), x->ds, sizeof(CaseState) * x->ncases, cudaMemcpyDeviceToHost));
    x->d2h += (long long)sizeof(CaseState) * x->ncases;
    return MGFVM_OK;
}

int push(mgfvm_ctx *x)
{
    CK(cudaMemcpy(x->dc, x->hc.data(), sizeof(CaseDev) * x->ncases, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(x->ds, x->hs.data(), sizeof(CaseState) * x->ncases, cudaMemcpyHostToDevice));
    x->h2d += (long long)(sizeof(CaseDev) + sizeof(CaseState)) * x->ncases;
    return MGFVM_OK;
}

// A context's device buffers (state pool, derivative storage, histories, case tables,
// the autotuner's backup) come from one stream-ordered memory pool per device that
// keeps up to KEEP_BYTES reserved after they are released, so programs that create and
// release contexts in a loop reuse that memory instead of mapping and unmapping it, and
// releasing a context calls no cudaFree (which waits for the whole device).  Allocation
// waits for the context stream, so the memory is usable from any stream when it
// returns.
static const unsigned long long KEEP_BYTES = 4ull << 30;
static cudaMemPool_t device_pool(int device)
{
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t mp = nullptr;
    if (cudaMemPoolCreate(&mp, &props) != cudaSuccess) {
        cudaGetLastError();
        mp = nullptr;
    } else {
        unsigned long long keep = KEEP_BYTES;
        cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pools[device] = mp;
    return mp;
}

// Small pinned host buffers (the stop-flag readbacks) are kept for reuse once a context
// releases them: pinning and unpinning host memory costs milliseconds per context.
static std::mutex pinned_mu;
static std::multimap<size_t, void *> pinned_cache;
static void *pinned_get(size_t bytes)
{
    {
        std::lock_guard<std::mutex> lock(pinned_mu);
        auto it = pinned_cache.lower_bound(bytes);
        if (it != pinned_cache.end() && it->first == bytes) {
            void *p = it->second;
            pinned_cache.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}
static void pinned_put(void *p, size_t bytes)
{
    std::lock_guard<std::mutex> lock(pinned_mu);
    pinned_cache.emplace(bytes, p);
}

static cudaError_t ctx_malloc(mgfvm_ctx *x, void **p, size_t bytes)
{
    cudaMemPool_t mp = device_pool(x->device);
    if (mp) {
        cudaError_t e = cudaMallocFromPoolAsync(p, bytes, mp, x->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
        if (e == cudaSuccess && ((uintptr_t)*p & 255) == 0) {
            x->pooled.push_back(*p);
            return cudaSuccess;
        }
        if (e == cudaSuccess) {          // not 256-byte aligned: take the plain allocator
            cudaFreeAsync(*p, x->stream);
            cudaStreamSynchronize(x->stream);
        } else if (e == cudaErrorMemoryAllocation) {
            *p = nullptr;
            return e;
        }
        cudaGetLastError();
    }
    return cudaMalloc(p, bytes);
}

static void ctx_free(mgfvm_ctx *x, void *p)
{
    if (!p) return;
    auto it = std::find(x->pooled.begin(), x->pooled.end(), p);
    if (it == x->pooled.end()) {
        cudaFree(p);
        return;
    }
    x->pooled.erase(it);
    // returned to the pool in stream order (the callers have drained the stream)
    if (!x->stream || cudaFreeAsync(p, x->stream) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
    }
}

int ensure_hist(mgfvm_ctx *x, int need)
{
    if (need <= x->hist_cap) return MGFVM_OK;
    int cap = std::max(HIST_INITIAL, x->hist_cap);
    while (cap < need) cap *= 2;
    RC(pull(x));
    double *h = nullptr;
    CK(ctx_malloc(x, (void **)&h, sizeof(double) * 2 * (size_t)cap * x->ncases));
    CK(cudaMemset(h, 0, sizeof(double) * 2 * (size_t)cap * x->ncases));
    if (x->hist && x->hist_cap > 0)
        CK(cudaMemcpy2D(h, sizeof(double) * cap, x->hist, sizeof(double) * x->hist_cap,
                        sizeof(double) * x->hist_cap, 2 * (size_t)x->ncases, cudaMemcpyDeviceToDevice));
    if (x->hist) ctx_free(x, x->hist);
    x->hist = h;
    x->hist_cap = cap;
    for (int c = 0; c < x->ncases; ++c) {
        x->hc[c].hist_err = h + (size_t)(2 * c) * cap;
        x->hc[c].hist_delta = h + (size_t)(2 * c + 1) * cap;
        x->hc[c].hist_cap = cap;
    }
    return push(x);
}

int build_graph(mgfvm_ctx *x)
{
    if (x->gexec) return MGFVM_OK;
    CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
    for (const Launch &L : x->cyc) {
        cudaError_t e = launch_one(L, x->dc, x->ds, x->dt, x->sched, x->stream);
        if (e != cudaSuccess) {
            cudaGraph_t g;
            cudaStreamEndCapture(x->stream, &g);
            if (g) cudaGraphDestroy(g);
            return mgfvm_fail(MGFVM_ECUDA, "graph capture: %s", cudaGetErrorString(e));
        }
    }
    CK(cudaStreamEndCapture(x->stream, &x->graph));
    CK(cudaGraphInstantiate(&x->gexec, x->graph, 0));
    return MGFVM_OK;
}

int run_cycles(mgfvm_ctx *x, int n)
{
    for (int ig = 0; ig < MAXLEV; ++ig) x->last_eq[ig] = EQ_SC;
    if (x->opt.use_graph) {
        RC(build_graph(x));
        for (int k = 0; k < n; ++k) CK(cudaGraphLaunch(x->gexec, x->stream));
        x->launches += (long long)n * (long long)x->cyc.size();
    } else {
        for (int k = 0; k < n; ++k) RC(run_list(x, x->cyc));
    }
    return MGFVM_OK;
}

int set_controls(mgfvm_ctx *x, int stop, double fp_tol)
{
    RC(pull(x));
    for (CaseDev &C : x->hc) {
        C.stop_enabled = stop;
        C.fp_tol = fp_tol;
    }
    for (CaseState &S : x->hs) S.done = 0;
    return push(x);
}

// Derivative storage of a tangent context: every slot tangent_slot() admits, on every
// level of every case, plus each pressure-copy buffer; zero until seeded.
int alloc_tangent(mgfvm_ctx *x)
{
    size_t off = 0;
    auto take = [&](size_t bytes) { off = align_up(off, 256); size_t o = off; off += std::max<size_t>(bytes, 8); return o; };
    std::vector<std::vector<size_t>> offs(x->ncases);
    x->tcase_off.assign(x->ncases, 0);
    x->tcase_bytes.assign(x->ncases, 0);
    for (int c = 0; c < x->ncases; ++c) {
        const mgfvm_config &g = x->cfg[c];
        x->tcase_off[c] = align_up(off, 256);
        for (int ig = 0; ig < g.ngrid; ++ig) {
            const size_t n = (size_t)npx_of(g, ig) * npy_of(g, ig);
            for (int s = 0; s < NSLOTS; ++s) offs[c].push_back(tangent_slot(s) ? take(n * sizeof(double)) : (size_t)-1);
            const int nc = x->progs[(size_t)c * MAXLEV + ig].ncopy;
            offs[c].push_back(take((size_t)std::max(nc, 1) * sizeof(double)));
        }
        x->tcase_bytes[c] = align_up(off, 256) - x->tcase_off[c];
    }
    const size_t bytes = align_up(off, 256);
    cudaError_t me = ctx_malloc(x, (void **)&x->tpool, bytes);
    if (me != cudaSuccess)
        return mgfvm_fail(me == cudaErrorMemoryAllocation ? MGFVM_ENOMEM : MGFVM_ECUDA,
                          "derivative storage of %zu bytes: %s", bytes, cudaGetErrorString(me));
    CK(cudaMemset(x->tpool, 0, bytes));
    x->ht.assign(x->ncases, CaseTan{});
    for (int c = 0; c < x->ncases; ++c) {
        size_t k = 0;
        for (int ig = 0; ig < x->cfg[c].ngrid; ++ig) {
            LevelTan &D = x->ht[c].lv[ig];
            for (int s = 0; s < NSLOTS; ++s, ++k) D.t[s] = offs[c][k] == (size_t)-1 ? nullptr : (double *)(x->tpool + offs[c][k]);
            D.pbuf_t = (double *)(x->tpool + offs[c][k++]);
        }
    }
    x->dir_kind.assign(x->ncases, MGFVM_DIR_NONE);
    x->dir_index.assign(x->ncases, 0);
    CK(ctx_malloc(x, (void **)&x->dt, sizeof(CaseTan) * x->ncases));
    CK(cudaMemcpy(x->dt, x->ht.data(), sizeof(CaseTan) * x->ncases, cudaMemcpyHostToDevice));
    x->h2d += (long long)sizeof(CaseTan) * x->ncases;
    return MGFVM_OK;
}

// Zero case c's derivatives and seed its direction: the level-0 inlet face (i = 0,
// row index + 1) with the coarse faces that rest_geom averages from it (rest_geom
// :1391-1473, as k_rest_geom), or the derivative of every level's amu and amusc =
// amuf / prsc (coefsc :867) with respect to amuf or prsc.
int seed_tangent(mgfvm_ctx *x, int c)
{
    CK(cudaMemsetAsync(x->tpool + x->tcase_off[c], 0, x->tcase_bytes[c], x->stream));
    const mgfvm_config &g = x->cfg[c];
    const int kind = x->dir_kind[c], idx = x->dir_index[c];
    for (int ig = 0; ig < g.ngrid; ++ig) {
        LevelTan &D = x->ht[c].lv[ig];
        D.amu_t = kind == MGFVM_DIR_AMUF ? 1.0 : 0.0;
        D.amusc_t = kind == MGFVM_DIR_AMUF ? 1.0 / g.prsc : kind == MGFVM_DIR_PRSC ? -g.amuf / (g.prsc * g.prsc) : 0.0;
    }
    if (kind == MGFVM_DIR_INLET) {
        std::vector<double> col(npy_of(g, 0), 0.0);
        col[idx + 1] = 1.0;
        for (int ig = 0; ig < g.ngrid; ++ig) {
            const int npx = npx_of(g, ig), npy = npy_of(g, ig);
            if (ig > 0) {
                std::vector<double> cc(npy, 0.0);
                for (int jc = 1; jc <= npy - 2; ++jc) cc[jc] = 0.5 * (col[2 * jc] + col[2 * jc - 1]);
                col.swap(cc);
            }
            CK(cudaMemcpy2DAsync(x->ht[c].lv[ig].t[S_U], sizeof(double) * npx, col.data(), sizeof(double),
                                 sizeof(double), npy, cudaMemcpyHostToDevice, x->stream));
            x->h2d += (long long)(sizeof(double) * npy);
        }
    }
    CK(cudaMemcpyAsync(x->dt + c, &x->ht[c], sizeof(CaseTan), cudaMemcpyHostToDevice, x->stream));
    x->h2d += (long long)sizeof(CaseTan);
    CK(cudaStreamSynchronize(x->stream));
    return MGFVM_OK;
}

// The V-cycle's launch list, and the device table of tensor maps its TMA-staged
// smoother launches read (without that table, those launches are plain tile launches).
int build_cycle(mgfvm_ctx *x)
{
    x->cyc.clear();
    x->hmaps.clear();
    if (x->dmaps) {
        cudaStreamSynchronize(x->stream);
        ctx_free(x, x->dmaps);
        x->dmaps = nullptr;
    }
    {
        Builder b{x, &x->cyc, &x->hmaps};
        b.cycle();
    }
    if (x->hmaps.empty()) return MGFVM_OK;
    cudaError_t e = ctx_malloc(x, (void **)&x->dmaps, sizeof(SmoothMap) * x->hmaps.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(x->dmaps, x->hmaps.data(), sizeof(SmoothMap) * x->hmaps.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (x->dmaps) ctx_free(x, x->dmaps);
        x->dmaps = nullptr;
        x->cyc.clear();
        x->hmaps.clear();
        Builder b{x, &x->cyc};
        b.cycle();
        return MGFVM_OK;
    }
    x->h2d += (long long)(sizeof(SmoothMap) * x->hmaps.size());
    for (Launch &L : x->cyc)
        if (L.kernel == K_SMOOTH_TMA) L.ptr = x->dmaps + L.map;
    return MGFVM_OK;
}

int init_state(mgfvm_ctx *x, int only_case)
{
    for (int c = 0; c < x->ncases; ++c) {
        if (only_case >= 0 && c != only_case) continue;
        x->hs[c] = CaseState{};
        x->hc[c].stop_enabled = 0;
    }
    RC(push(x));
    int max_obs = 0, max_npy = 0;
    for (int c = 0; c < x->ncases; ++c) {
        if (only_case >= 0 && c != only_case) continue;
        max_obs = std::max(max_obs, x->cfg[c].nobs);
        max_npy = std::max(max_npy, npy_of(x->cfg[c], 0));
    }
    CaseDev *dc = x->dc + (only_case >= 0 ? only_case : 0);
    InitDev *di = x->dinit + (only_case >= 0 ? only_case : 0);
    const int n = only_case >= 0 ? 1 : x->ncases;
    cudaError_t e = launch_init(dc, di, n, x->maxng, x->maxcells.data(), max_obs, max_npy, x->stream);
    if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "init kernels: %s", cudaGetErrorString(e));
    x->launches += 3LL * x->maxng + 1 + (x->maxng - 1);
    CK(cudaStreamSynchronize(x->stream));
    if (x->opt.tangent)
        for (int c = 0; c < x->ncases; ++c)
            if (only_case < 0 || c == only_case) RC(seed_tangent(x, c));
    return MGFVM_OK;
}

int upload_profiles(mgfvm_ctx *x)
{
    size_t tot = 0;
    for (auto &p : x->profile) tot += p.size();
    if (x->dprofile) { ctx_free(x, x->dprofile); x->dprofile = nullptr; }
    if (tot) {
        CK(ctx_malloc(x, (void **)&x->dprofile, sizeof(double) * tot));
    }
    size_t off = 0;
    for (int c = 0; c < x->ncases; ++c) {
        auto &p = x->profile[c];
        x->hinit[c].profile = p.empty() ? nullptr : x->dprofile + off;
        x->hinit[c].nprofile = (int)p.size();
        if (!p.empty()) CK(cudaMemcpy(x->dprofile + off, p.data(), sizeof(double) * p.size(), cudaMemcpyHostToDevice));
        x->h2d += (long long)(sizeof(double) * p.size());
        off += p.size();
    }
    CK(cudaMemcpy(x->dinit, x->hinit.data(), sizeof(InitDev) * x->ncases, cudaMemcpyHostToDevice));
    x->h2d += (long long)sizeof(InitDev) * x->ncases;
    return MGFVM_OK;
}

void destroy_all(mgfvm_ctx *x)
{
    if (!x) return;
    if (x->device >= 0) cudaSetDevice(x->device);
    if (x->stream) cudaStreamSynchronize(x->stream);
    if (x->gexec) cudaGraphExecDestroy(x->gexec);
    if (x->graph) cudaGraphDestroy(x->graph);
    if (x->pool) ctx_free(x, x->pool);
    if (x->tpool) ctx_free(x, x->tpool);
    if (x->dmaps) ctx_free(x, x->dmaps);
    if (x->dt) ctx_free(x, x->dt);
    if (x->hist) ctx_free(x, x->hist);
    if (x->dprofile) ctx_free(x, x->dprofile);
    if (x->dobs) ctx_free(x, x->dobs);
    if (x->dc) ctx_free(x, x->dc);
    if (x->ds) ctx_free(x, x->ds);
    if (x->dinit) ctx_free(x, x->dinit);
    if (x->hflags) pinned_put(x->hflags, x->hflags_bytes);
    for (cudaEvent_t &e : x->eflag)
        if (e) cudaEventDestroy(e);
    if (x->e0) cudaEventDestroy(x->e0);
    if (x->e1) cudaEventDestroy(x->e1);
    if (x->stream) cudaStreamDestroy(x->stream);
    for (auto &p : x->progs) mgfvm_free_obstacle_prog(&p);
    delete x;
}

int check_ctx(mgfvm_ctx *x)
{
    if (!x) return mgfvm_fail(MGFVM_EINVAL, "null context");
    CK(cudaSetDevice(x->device));
    return MGFVM_OK;
}

int check_case_level(mgfvm_ctx *x, int icase, int level)
{
    if (icase < 0 || icase >= x->ncases) return mgfvm_fail(MGFVM_EINVAL, "case %d outside [0, %d)", icase, x->ncases);
    if (level < 0 || level >= x->cfg[icase].ngrid)
        return mgfvm_fail(MGFVM_EINVAL, "level %d outside [0, %d)", level, x->cfg[icase].ngrid);
    return MGFVM_OK;
}

int create_impl(const mgfvm_config *cases, int ncases, const mgfvm_options *opt_in, mgfvm_ctx *x)
{
    mgfvm_options opt;
    if (opt_in) opt = *opt_in; else mgfvm_options_default(&opt);
    if (opt.sync_every < 1) opt.sync_every = 1;
    if (opt.precision != MGFVM_PREC_FP64 && opt.precision != MGFVM_PREC_MIXED)
        return mgfvm_fail(MGFVM_EINVAL, "unknown precision %d", opt.precision);
    if (opt.tangent && opt.precision != MGFVM_PREC_FP64)
        return mgfvm_fail(MGFVM_EINVAL, "derivatives are taken of the FP64 V-cycle only");
    x->opt = opt;
    x->device = opt.device;
    x->ncases = ncases;
    for (int c = 0; c < ncases; ++c) RC(mgfvm_config_validate(&cases[c]));
    for (int c = 1; c < ncases; ++c)
        if (cases[c].isolve != cases[0].isolve || cases[c].nswpm != cases[0].nswpm ||
            cases[c].nswpp != cases[0].nswpp)
            return mgfvm_fail(MGFVM_EINVAL, "case %d: isolve/nswpm/nswpp differ from case 0; a batch "
                                            "shares one smoothing schedule", c);
    x->sched.isolve = cases[0].isolve;
    x->sched.nswpm = cases[0].nswpm;
    x->sched.nswpp = cases[0].nswpp;
    x->sched.tma_wait_polls = TMA_WAIT_POLLS;
    x->sched.pdl = true;
    x->cfg.assign(cases, cases + ncases);
    x->obs.resize(ncases);
    x->profile.resize(ncases);
    for (int c = 0; c < ncases; ++c) {
        x->obs[c].assign(cases[c].obs, cases[c].obs + 4 * (size_t)cases[c].nobs);
        x->cfg[c].obs = x->obs[c].empty() ? nullptr : x->obs[c].data();
        x->cfg[c].dpdxm = 0.0;   // never read by the reference (:33), so always 0 there
        x->cfg[c].dpdym = 0.0;
        x->maxng = std::max(x->maxng, cases[c].ngrid);
    }
    if (x->maxng > MAXLEV) return mgfvm_fail(MGFVM_EINVAL, "ngrid above %d", MAXLEV);
    x->maxcells.assign(x->maxng, 0);
    for (int c = 0; c < ncases; ++c)
        for (int ig = 0; ig < x->cfg[c].ngrid; ++ig)
            x->maxcells[ig] = std::max(x->maxcells[ig], npx_of(x->cfg[c], ig) * npy_of(x->cfg[c], ig));

    // obstacle programs (host)
    x->progs.assign((size_t)ncases * MAXLEV, mgfvm_obstacle_prog{});
    for (int c = 0; c < ncases; ++c)
        for (int ig = 0; ig < x->cfg[c].ngrid; ++ig)
            RC(mgfvm_build_obstacle_prog(&x->cfg[c], ig, &x->progs[(size_t)c * MAXLEV + ig]));

    CK(cudaSetDevice(x->device));
    CK(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&x->e0));
    CK(cudaEventCreate(&x->e1));
    x->hflags_bytes = sizeof(int) * 2 * (size_t)ncases;
    x->hflags = (int *)pinned_get(x->hflags_bytes);
    if (!x->hflags) return mgfvm_fail(MGFVM_ENOMEM, "pinned host memory for %d flags", 2 * ncases);
    for (cudaEvent_t &e : x->eflag) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));

    // pool layout: pass 0 sizes, pass 1 assigns
    x->hc.assign(ncases, CaseDev{});
    x->hs.assign(ncases, CaseState{});
    std::vector<size_t> off_slots;
    size_t off = 0;
    auto take = [&](size_t bytes) { off = align_up(off, 256); size_t o = off; off += std::max<size_t>(bytes, 8); return o; };
    struct Pend { int c, ig; size_t slot[NSLOTS]; size_t tag, seq, pdst, psrc, pbuf, pcode, pfan; };
    std::vector<Pend> pend;
    std::vector<size_t> part_off(ncases), cnt_off(ncases);
    for (int c = 0; c < ncases; ++c) {
        const mgfvm_config &g = x->cfg[c];
        for (int ig = 0; ig < g.ngrid; ++ig) {
            Pend p{};
            p.c = c; p.ig = ig;
            const size_t n = (size_t)npx_of(g, ig) * npy_of(g, ig);
            const int ns = ig == 0 ? NSLOTS : NSLOTS_LEVEL;
            for (int s = 0; s < NSLOTS; ++s) p.slot[s] = s < ns ? take(n * sizeof(double)) : (size_t)-1;
            p.tag = take(n * sizeof(int));
            const mgfvm_obstacle_prog &P = x->progs[(size_t)c * MAXLEV + ig];
            p.seq = P.nseq ? take(n * sizeof(unsigned)) : (size_t)-1;
            p.pdst = P.ncopy ? take(P.ncopy * sizeof(int)) : (size_t)-1;
            p.psrc = P.ncopy ? take(P.ncopy * sizeof(int)) : (size_t)-1;
            p.pbuf = P.ncopy ? take(P.ncopy * sizeof(double)) : (size_t)-1;
            const bool fan = P.ncopy && P.fan;
            p.pcode = fan ? take(n * sizeof(int)) : (size_t)-1;
            p.pfan = fan ? take(2 * (size_t)P.ncopy * sizeof(int)) : (size_t)-1;
            pend.push_back(p);
        }
        const long long n0 = (long long)(npx_of(g, 0) - 2) * (npy_of(g, 0) - 2);
        part_off[c] = take((size_t)std::max(nblk(n0), 64) * RED_STRIDE * sizeof(double));
        cnt_off[c] = take(16 * sizeof(unsigned));
    }
    const size_t pool_bytes = align_up(off, 256);
    x->pool_bytes = pool_bytes;
    cudaError_t me = ctx_malloc(x, (void **)&x->pool, pool_bytes);
    if (me != cudaSuccess)
        return mgfvm_fail(me == cudaErrorMemoryAllocation ? MGFVM_ENOMEM : MGFVM_ECUDA,
                          "device pool of %zu bytes: %s", pool_bytes, cudaGetErrorString(me));
    CK(cudaMemset(x->pool, 0, pool_bytes));

    for (int c = 0; c < ncases; ++c) {
        CaseDev &C = x->hc[c];
        const mgfvm_config &g = x->cfg[c];
        C.relxm = g.relxm; C.relxp = g.relxp; C.sc_obs = g.sc_obs;
        C.dpdxm = g.dpdxm; C.dpdym = g.dpdym; C.convergence = g.convergence;
        C.ibc_xm = g.ibc_xm; C.ibc_xp = g.ibc_xp; C.ibc_ym = g.ibc_ym; C.ibc_yp = g.ibc_yp;
        C.ngrid = g.ngrid;
        int tail = g.ngrid;
        if (opt.tangent) tail = 0;     // the tangent V-cycle runs in the one-CTA kernel
        else if (opt.tail_level >= 0) tail = std::min(opt.tail_level, g.ngrid);
        else
            for (int ig = 0; ig < g.ngrid; ++ig)
                if (npx_of(g, ig) * npy_of(g, ig) <= TAIL_AUTO_CELLS) { tail = ig; break; }
        C.tail = tail;
        x->tail0.push_back(tail);
        C.partials = (double *)(x->pool + part_off[c]);
        C.counters = (unsigned *)(x->pool + cnt_off[c]);
    }
    for (const Pend &p : pend) {
        CaseDev &C = x->hc[p.c];
        LevelDev &L = C.lv[p.ig];
        const mgfvm_config &g = x->cfg[p.c];
        L.npx = npx_of(g, p.ig);
        L.npy = npy_of(g, p.ig);
        L.dx = g.xl / (L.npx - 2);       // AllocateMemorySoA :413-414
        L.dy = g.yl / (L.npy - 2);
        L.amu = g.amuf;
        L.amusc = g.amuf / g.prsc;       // coefsc :867
        for (int s = 0; s < NSLOTS; ++s) L.f[s] = p.slot[s] == (size_t)-1 ? nullptr : (double *)(x->pool + p.slot[s]);
        L.tag = (int *)(x->pool + p.tag);
        const mgfvm_obstacle_prog &P = x->progs[(size_t)p.c * MAXLEV + p.ig];
        L.ncopy = P.ncopy;
        L.hazard = P.hazard;
        L.seq = nullptr; L.pdst = nullptr; L.psrc = nullptr; L.pbuf = nullptr;
        L.pcode = nullptr; L.pfan = nullptr;
        if (P.nseq) {
            const size_t n = (size_t)L.npx * L.npy;
            std::vector<unsigned> dense(n, 0u);
            for (int k = 0; k < P.nseq; ++k) dense[P.cells[k]] = P.codes[k];
            unsigned *d = (unsigned *)(x->pool + p.seq);
            CK(cudaMemcpy(d, dense.data(), n * sizeof(unsigned), cudaMemcpyHostToDevice));
            x->h2d += (long long)(n * sizeof(unsigned));
            L.seq = d;
        }
        if (P.ncopy) {
            int *dd = (int *)(x->pool + p.pdst), *ds = (int *)(x->pool + p.psrc);
            CK(cudaMemcpy(dd, P.dst, P.ncopy * sizeof(int), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ds, P.src, P.ncopy * sizeof(int), cudaMemcpyHostToDevice));
            x->h2d += 2LL * P.ncopy * (long long)sizeof(int);
            L.pdst = dd; L.psrc = ds;
            L.pbuf = (double *)(x->pool + p.pbuf);
        }
        if (p.pcode != (size_t)-1) {
            // per cell: PCODE_DST when the copy writes it, 1 + its first fan entry when
            // its update thread performs copies
            const size_t n = (size_t)L.npx * L.npy;
            std::vector<int> code(n, 0);
            for (int k = 0; k < P.ncopy; ++k) {
                code[P.fan[2 * k] & ~PFAN_LAST] |= PCODE_DST;
                if (k == 0 || P.owners[k] != P.owners[k - 1]) code[P.owners[k]] |= k + 1;
            }
            int *dc = (int *)(x->pool + p.pcode), *df = (int *)(x->pool + p.pfan);
            CK(cudaMemcpy(dc, code.data(), n * sizeof(int), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(df, P.fan, 2 * (size_t)P.ncopy * sizeof(int), cudaMemcpyHostToDevice));
            x->h2d += (long long)(n + 2 * (size_t)P.ncopy) * (long long)sizeof(int);
            L.pcode = dc;
            L.pfan = df;
        }
    }

    // init parameters
    size_t nobs_tot = 0;
    for (int c = 0; c < ncases; ++c) nobs_tot += x->obs[c].size();
    if (nobs_tot) CK(ctx_malloc(x, (void **)&x->dobs, sizeof(int) * nobs_tot));
    x->hinit.assign(ncases, InitDev{});
    size_t ooff = 0;
    for (int c = 0; c < ncases; ++c) {
        const mgfvm_config &g = x->cfg[c];
        InitDev &P = x->hinit[c];
        P.guess[0] = g.u_guess; P.guess[1] = g.v_guess; P.guess[2] = g.p_guess; P.guess[3] = g.sc_guess;
        const double bc[4][4] = {{g.u_xm, g.v_xm, g.p_xm, g.sc_xm}, {g.u_xp, g.v_xp, g.p_xp, g.sc_xp},
                                 {g.u_ym, g.v_ym, g.p_ym, g.sc_ym}, {g.u_yp, g.v_yp, g.p_yp, g.sc_yp}};
        std::memcpy(P.bc, bc, sizeof bc);
        P.sc_obs = g.sc_obs;
        P.ig_obs = g.ig_obs; P.ibeg_obs = g.ibeg_obs; P.nobs = g.nobs;
        P.obs = nullptr;
        if (g.nobs) {
            CK(cudaMemcpy(x->dobs + ooff, x->obs[c].data(), sizeof(int) * x->obs[c].size(), cudaMemcpyHostToDevice));
            x->h2d += (long long)(sizeof(int) * x->obs[c].size());
            P.obs = x->dobs + ooff;
            ooff += x->obs[c].size();
        }
        P.ig_inlt = g.ig_inlt; P.ninlt = g.ninlt; P.ig_outlt = g.ig_outlt; P.noutlt = g.noutlt;
        for (int k = 0; k < MGFVM_MAX_PORTS; ++k) {
            P.jf_in[k] = g.jfinlt[k]; P.jl_in[k] = g.jlinlt[k];
            P.jf_out[k] = g.jfoutlt[k]; P.jl_out[k] = g.jloutlt[k];
            P.in_val[k][0] = g.uinlt[k]; P.in_val[k][1] = g.vinlt[k]; P.in_val[k][2] = g.scinlt[k];
            P.out_val[k][0] = g.uoutlt[k]; P.out_val[k][1] = g.voutlt[k]; P.out_val[k][2] = g.scoutlt[k];
        }
    }
    CK(ctx_malloc(x, (void **)&x->dc, sizeof(CaseDev) * ncases));
    CK(ctx_malloc(x, (void **)&x->ds, sizeof(CaseState) * ncases));
    CK(ctx_malloc(x, (void **)&x->dinit, sizeof(InitDev) * ncases));
    RC(upload_profiles(x));
    // histories
    x->hist_cap = 0;
    RC(push(x));
    RC(ensure_hist(x, HIST_INITIAL));
    for (int ig = 0; ig < MAXLEV; ++ig) x->last_eq[ig] = EQ_SC;
    CK(configure_kernels());
    if (opt.tangent) RC(alloc_tangent(x));
    RC(init_state(x, -1));
    return build_cycle(x);
}

}  // namespace

// =================================================================== C ABI
extern "C" {

int mgfvm_create(const mgfvm_config *cases, int ncases, const mgfvm_options *opt, mgfvm_ctx **out)
{
    mgfvm_clear_error();
    if (!out) return mgfvm_fail(MGFVM_EINVAL, "null output pointer");
    *out = nullptr;
    if (!cases || ncases < 1) return mgfvm_fail(MGFVM_EINVAL, "need at least one case");
    mgfvm_ctx *x = new (std::nothrow) mgfvm_ctx();
    if (!x) return mgfvm_fail(MGFVM_ENOMEM, "out of host memory");
    int rc = create_impl(cases, ncases, opt, x);
    if (rc != MGFVM_OK) {
        std::string msg = mgfvm_last_error();
        destroy_all(x);
        return mgfvm_fail(rc, "%s", msg.c_str());
    }
    *out = x;
    return MGFVM_OK;
}

int mgfvm_destroy(mgfvm_ctx *x)
{
    destroy_all(x);
    return MGFVM_OK;
}

int mgfvm_reset(mgfvm_ctx *x)
{
    RC(check_ctx(x));
    RC(pull(x));
    return init_state(x, -1);
}

int mgfvm_set_inlet_profile(mgfvm_ctx *x, int icase, const double *u, int n)
{
    RC(check_ctx(x));
    if (icase < 0 || icase >= x->ncases) return mgfvm_fail(MGFVM_EINVAL, "case %d out of range", icase);
    if (n < 0 || (n > 0 && !u)) return mgfvm_fail(MGFVM_EINVAL, "bad inlet profile");
    RC(pull(x));
    x->profile[icase].assign(u, u + n);
    RC(upload_profiles(x));
    return init_state(x, icase);
}

// A kernel found its launch shape too small for its tile (a schedule bug): fail loudly.
static int check_status(mgfvm_ctx *x)
{
    for (int c = 0; c < x->ncases; ++c) {
        if (x->hs[c].status & CASE_BAD_LAUNCH)
            return mgfvm_fail(MGFVM_ECUDA, "case %d: a smoother launch was too small for its tile", c);
        if (x->hs[c].status & CASE_WAIT_TIMEOUT)
            return mgfvm_fail(MGFVM_ETIMEOUT,
                              "a smoother CTA of case %d gave up waiting for its TMA loads: the results of every "
                              "case from this call are invalid; mgfvm_reset returns the context to a defined state",
                              c);
    }
    return MGFVM_OK;
}

int mgfvm_cycle(mgfvm_ctx *x, int ncycles)
{
    RC(check_ctx(x));
    if (ncycles < 0) return mgfvm_fail(MGFVM_EINVAL, "negative cycle count");
    RC(pull(x));
    int need = 0;
    for (const CaseState &S : x->hs) need = std::max(need, S.ncyc + ncycles);
    RC(ensure_hist(x, need));
    RC(set_controls(x, 0, 0.0));
    CK(cudaEventRecord(x->e0, x->stream));
    RC(run_cycles(x, ncycles));
    CK(cudaEventRecord(x->e1, x->stream));
    CK(cudaEventSynchronize(x->e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, x->e0, x->e1));
    x->last_ms = ms;
    CK(cudaGetLastError());
    RC(pull(x));
    return check_status(x);
}

int mgfvm_solve(mgfvm_ctx *x, int max_cycles, double fp_tol, int *cycles_out)
{
    RC(check_ctx(x));
    if (max_cycles < 0) return mgfvm_fail(MGFVM_EINVAL, "negative cycle limit");
    RC(pull(x));
    std::vector<int> start(x->ncases);
    int need = 0;
    for (int c = 0; c < x->ncases; ++c) {
        start[c] = x->hs[c].ncyc;
        need = std::max(need, x->hs[c].ncyc + max_cycles);
    }
    RC(ensure_hist(x, need));
    RC(set_controls(x, 1, fp_tol));
    CK(cudaEventRecord(x->e0, x->stream));
    // Chunks of sync_every cycles, each followed by a copy of the stop flags; the next
    // chunk is queued before the host looks at the previous chunk's flags, so the GPU
    // never waits for the host.  Once every case has stopped, a chunk already queued
    // runs as cycles in which every kernel skips its stopped case.
    int run = 0, issued = 0;
    auto issue = [&]() -> int {
        const int n = std::min(x->opt.sync_every, max_cycles - run);
        RC(run_cycles(x, n));
        run += n;
        int *f = x->hflags + (size_t)(issued & 1) * x->ncases;
        CK(cudaMemcpy2DAsync(f, sizeof(int), &x->ds[0].done, sizeof(CaseState), sizeof(int), x->ncases,
                             cudaMemcpyDeviceToHost, x->stream));
        CK(cudaEventRecord(x->eflag[issued & 1], x->stream));
        x->d2h += (long long)sizeof(int) * x->ncases;
        ++issued;
        return MGFVM_OK;
    };
    if (run < max_cycles) RC(issue());
    for (int k = 0; k < issued; ++k) {
        if (run < max_cycles) RC(issue());
        CK(cudaEventSynchronize(x->eflag[k & 1]));
        const int *f = x->hflags + (size_t)(k & 1) * x->ncases;
        bool all = true;
        for (int c = 0; c < x->ncases; ++c) all &= f[c] != 0;
        if (all) break;
    }
    CK(cudaEventRecord(x->e1, x->stream));
    CK(cudaEventSynchronize(x->e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, x->e0, x->e1));
    x->last_ms = ms;
    RC(pull(x));
    int nonfinite = 0;
    for (int c = 0; c < x->ncases; ++c) {
        if (cycles_out) cycles_out[c] = x->hs[c].ncyc - start[c];
        if (x->hs[c].status & CASE_NONFINITE) nonfinite = 1;
    }
    if (nonfinite) return mgfvm_fail(MGFVM_ENONFINITE, "a case's mass error or fixed-point change became NaN/Inf");
    return check_status(x);
}

int mgfvm_history(mgfvm_ctx *x, int icase, double *err, double *delta, int cap, int *n_out)
{
    RC(check_ctx(x));
    if (icase < 0 || icase >= x->ncases) return mgfvm_fail(MGFVM_EINVAL, "case %d out of range", icase);
    RC(pull(x));
    const int n = std::min(x->hs[icase].ncyc, x->hist_cap);
    if (n_out) *n_out = x->hs[icase].ncyc;
    const int m = std::min(n, std::max(cap, 0));
    if (err && m) CK(cudaMemcpy(err, x->hc[icase].hist_err, sizeof(double) * m, cudaMemcpyDeviceToHost));
    if (delta && m) CK(cudaMemcpy(delta, x->hc[icase].hist_delta, sizeof(double) * m, cudaMemcpyDeviceToHost));
    x->d2h += (long long)sizeof(double) * m * ((err ? 1 : 0) + (delta ? 1 : 0));
    return MGFVM_OK;
}

int mgfvm_num_levels(mgfvm_ctx *x, int icase, int *ngrid)
{
    if (!x || icase < 0 || icase >= x->ncases || !ngrid) return mgfvm_fail(MGFVM_EINVAL, "bad arguments");
    *ngrid = x->cfg[icase].ngrid;
    return MGFVM_OK;
}

int mgfvm_level_dims(mgfvm_ctx *x, int icase, int level, int *npx, int *npy)
{
    if (!x) return mgfvm_fail(MGFVM_EINVAL, "null context");
    RC(check_case_level(x, icase, level));
    if (npx) *npx = npx_of(x->cfg[icase], level);
    if (npy) *npy = npy_of(x->cfg[icase], level);
    return MGFVM_OK;
}

int mgfvm_get_field(mgfvm_ctx *x, int icase, int level, int field, double *out)
{
    RC(check_ctx(x));
    RC(check_case_level(x, icase, level));
    if (field < 0 || field >= MGFVM_NFIELDS || !out) return mgfvm_fail(MGFVM_EINVAL, "bad field %d", field);
    CK(cudaStreamSynchronize(x->stream));
    const LevelDev &L = x->hc[icase].lv[level];
    CK(cudaMemcpy(out, L.f[field_slot(field, x->last_eq[level])], sizeof(double) * L.npx * L.npy,
                  cudaMemcpyDeviceToHost));
    x->d2h += (long long)sizeof(double) * L.npx * L.npy;
    return MGFVM_OK;
}

int mgfvm_field_device_ptr(mgfvm_ctx *x, int icase, int level, int field, double **ptr, int *npx, int *npy)
{
    RC(check_ctx(x));
    RC(check_case_level(x, icase, level));
    if (field < 0 || field >= MGFVM_NFIELDS || !ptr) return mgfvm_fail(MGFVM_EINVAL, "bad field %d", field);
    const LevelDev &L = x->hc[icase].lv[level];
    *ptr = L.f[field_slot(field, x->last_eq[level])];
    if (npx) *npx = L.npx;
    if (npy) *npy = L.npy;
    return MGFVM_OK;
}

int mgfvm_set_field(mgfvm_ctx *x, int icase, int level, int field, const double *in)
{
    RC(check_ctx(x));
    if (x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "%s: not available in a tangent context (it would change the state without its derivatives)", __func__);
    RC(check_case_level(x, icase, level));
    if (field < 0 || field >= MGFVM_NFIELDS || !in) return mgfvm_fail(MGFVM_EINVAL, "bad field %d", field);
    CK(cudaStreamSynchronize(x->stream));
    const LevelDev &L = x->hc[icase].lv[level];
    CK(cudaMemcpy(L.f[field_slot(field, x->last_eq[level])], in, sizeof(double) * L.npx * L.npy,
                  cudaMemcpyHostToDevice));
    x->h2d += (long long)sizeof(double) * L.npx * L.npy;
    return MGFVM_OK;
}

int mgfvm_get_tag(mgfvm_ctx *x, int icase, int level, int *out)
{
    RC(check_ctx(x));
    RC(check_case_level(x, icase, level));
    if (!out) return mgfvm_fail(MGFVM_EINVAL, "null output");
    CK(cudaStreamSynchronize(x->stream));
    const LevelDev &L = x->hc[icase].lv[level];
    CK(cudaMemcpy(out, L.tag, sizeof(int) * L.npx * L.npy, cudaMemcpyDeviceToHost));
    x->d2h += (long long)sizeof(int) * L.npx * L.npy;
    return MGFVM_OK;
}

int mgfvm_get_obstacle_ranges(mgfvm_ctx *x, int icase, int level, int *out)
{
    if (!x) return mgfvm_fail(MGFVM_EINVAL, "null context");
    RC(check_case_level(x, icase, level));
    for (int k = 0; k < x->cfg[icase].nobs; ++k) mgfvm_obstacle_range(&x->cfg[icase], k, level, &out[4 * k]);
    return MGFVM_OK;
}

int mgfvm_op(mgfvm_ctx *x, int op, int level)
{
    RC(check_ctx(x));
    if (x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "%s: not available in a tangent context (it would change the state without its derivatives)", __func__);
    if (op < 0 || op >= MGFVM_NOPS) return mgfvm_fail(MGFVM_EINVAL, "unknown op %d", op);
    if (level < 0 || level >= x->maxng) return mgfvm_fail(MGFVM_EINVAL, "level %d out of range", level);
    if ((op == MGFVM_OP_RESTRICT || op == MGFVM_OP_PROLONG) && level + 1 >= x->maxng)
        return mgfvm_fail(MGFVM_EINVAL, "transfer from level %d needs level %d", level, level + 1);
    RC(set_controls(x, 0, 0.0));
    std::vector<Launch> v;
    Builder b{x, &v};
    b.op(op, level);
    RC(run_list(x, v));
    CK(cudaStreamSynchronize(x->stream));
    if (op_equation(op) >= 0) x->last_eq[level] = op_equation(op);
    return MGFVM_OK;
}

int mgfvm_kernel_launches(mgfvm_ctx *x, long long *out)
{
    if (!x || !out) return mgfvm_fail(MGFVM_EINVAL, "bad arguments");
    *out = x->launches;
    return MGFVM_OK;
}

int mgfvm_last_elapsed_ms(mgfvm_ctx *x, double *ms)
{
    if (!x || !ms) return mgfvm_fail(MGFVM_EINVAL, "bad arguments");
    *ms = x->last_ms;
    return MGFVM_OK;
}

int mgfvm_stream(mgfvm_ctx *x, void **stream)
{
    if (!x || !stream) return mgfvm_fail(MGFVM_EINVAL, "bad arguments");
    *stream = (void *)x->stream;
    return MGFVM_OK;
}

int mgfvm_time_op(mgfvm_ctx *x, int op, int level, int reps, double *ms_total, int *launches)
{
    RC(check_ctx(x));
    if (x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "%s: not available in a tangent context (it would change the state without its derivatives)", __func__);
    if (op < 0 || op >= MGFVM_NOPS || reps < 1) return mgfvm_fail(MGFVM_EINVAL, "bad op %d or reps %d", op, reps);
    if (level < 0 || level >= x->maxng) return mgfvm_fail(MGFVM_EINVAL, "level %d out of range", level);
    if ((op == MGFVM_OP_RESTRICT || op == MGFVM_OP_PROLONG) && level + 1 >= x->maxng)
        return mgfvm_fail(MGFVM_EINVAL, "transfer from level %d needs level %d", level, level + 1);
    RC(set_controls(x, 0, 0.0));
    std::vector<Launch> v;
    Builder b{x, &v};
    b.op(op, level);
    // the op's launches are captured once into a graph and the graph is replayed, so
    // the host's launch rate does not pace short kernels (as in a V-cycle)
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
    for (const Launch &L : v) {
        cudaError_t e = launch_one(L, x->dc, x->ds, x->dt, x->sched, x->stream);
        if (e != cudaSuccess) {
            cudaStreamEndCapture(x->stream, &g);
            if (g) cudaGraphDestroy(g);
            return mgfvm_fail(MGFVM_ECUDA, "time_op capture: %s", cudaGetErrorString(e));
        }
    }
    CK(cudaStreamEndCapture(x->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(ge, x->stream);          // warm the graph
    if (e == cudaSuccess) e = cudaEventRecord(x->e0, x->stream);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = cudaGraphLaunch(ge, x->stream);
    if (e == cudaSuccess) e = cudaEventRecord(x->e1, x->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(x->e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, x->e0, x->e1);
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "time_op: %s", cudaGetErrorString(e));
    x->launches += (long long)v.size() * (reps + 1);
    if (ms_total) *ms_total = ms;
    if (launches) *launches = (int)v.size() * reps;
    return MGFVM_OK;
}

static bool tuning_valid(const mgfvm_tuning &t)
{
    for (int ig = 0; ig < MGFVM_MAX_LEVELS; ++ig) {
        if (t.smooth_units[ig] < 0 || t.smooth_units[ig] > 64) return false;
        if (t.smooth_threads[ig] != 0 && t.smooth_threads[ig] != SMOOTH_BLOCK && t.smooth_threads[ig] != SMOOTH_BLOCK / 2 &&
            t.smooth_threads[ig] != SMOOTH_BLOCK / 4)
            return false;
        for (int v : {t.asm_slices[ig], t.restrict_slices[ig]})
            if (v != 0 && v != 1 && v != 3) return false;
        if (t.update_pfix[ig] < 0 || t.update_pfix[ig] > 2) return false;
        if (t.odd_chunks[ig] < 0 || t.odd_chunks[ig] > 2) return false;
        if (t.pp_level[ig] < 0 || t.pp_level[ig] > 2) return false;
        if (t.smooth_tma[ig] < 0 || t.smooth_tma[ig] > 2) return false;
        if (t.coarse_kernel[ig] < 0 || t.coarse_kernel[ig] > 2) return false;
        if (t.prol_fused[ig] < 0 || t.prol_fused[ig] > 2) return false;
        if (t.band_visit[ig] < 0 || t.band_visit[ig] > 2) return false;
    }
    return t.tma_first_wait >= -1 && t.pdl >= 0 && t.pdl <= 2 && t.coarse_cluster >= 0 && t.coarse_cluster <= 2;
}

// The first level of the one-CTA coarse kernel from x->tune.coarse_kernel (the first
// level marked 2), else as chosen at creation; written to the cases where it changes.
static int apply_tail(mgfvm_ctx *x)
{
    int from = -1;
    for (int ig = 0; ig < MGFVM_MAX_LEVELS && from < 0; ++ig)
        if (x->tune.coarse_kernel[ig] == 2) from = ig;
    bool change = false;
    for (int c = 0; c < x->ncases; ++c) {
        const int t = x->opt.tangent ? 0 : from >= 0 ? std::min(from, x->cfg[c].ngrid) : x->tail0[c];
        change |= x->hc[c].tail != t;
    }
    if (!change) return MGFVM_OK;
    RC(pull(x));
    for (int c = 0; c < x->ncases; ++c)
        x->hc[c].tail = x->opt.tangent ? 0 : from >= 0 ? std::min(from, x->cfg[c].ngrid) : x->tail0[c];
    return push(x);
}

// Drop the captured graph and rebuild the V-cycle's launch list from x->tune.
static int rebuild_schedule(mgfvm_ctx *x)
{
    if (x->gexec) cudaGraphExecDestroy(x->gexec);
    if (x->graph) cudaGraphDestroy(x->graph);
    x->gexec = nullptr;
    x->graph = nullptr;
    RC(apply_tail(x));
    return build_cycle(x);
}

// Milliseconds per graph-replayed V-cycle (best of two runs of n), stop rule off.
static int time_schedule(mgfvm_ctx *x, int n, double *ms)
{
    RC(build_graph(x));
    CK(cudaGraphLaunch(x->gexec, x->stream));
    double best = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
        CK(cudaEventRecord(x->e0, x->stream));
        for (int k = 0; k < n; ++k) CK(cudaGraphLaunch(x->gexec, x->stream));
        CK(cudaEventRecord(x->e1, x->stream));
        CK(cudaEventSynchronize(x->e1));
        float t = 0;
        CK(cudaEventElapsedTime(&t, x->e0, x->e1));
        best = std::min(best, (double)t / n);
    }
    x->launches += (long long)(2 * n + 1) * (long long)x->cyc.size();
    *ms = best;
    return MGFVM_OK;
}

int mgfvm_get_tuning(mgfvm_ctx *x, mgfvm_tuning *t)
{
    RC(check_ctx(x));
    if (!t) return mgfvm_fail(MGFVM_EINVAL, "null tuning");
    *t = x->tune;
    return MGFVM_OK;
}

int mgfvm_set_tuning(mgfvm_ctx *x, const mgfvm_tuning *t)
{
    RC(check_ctx(x));
    if (!t || !tuning_valid(*t)) return mgfvm_fail(MGFVM_EINVAL, "tuning values outside the allowed sets");
    x->tune = *t;
    x->sched.tma_wait_polls = t->tma_first_wait == 0 ? TMA_WAIT_POLLS : std::max(0, t->tma_first_wait);
    x->sched.pdl = t->pdl != 1;
    return rebuild_schedule(x);
}

int mgfvm_autotune(mgfvm_ctx *x, int cycles, mgfvm_tuning *chosen, double *ms_before, double *ms_after)
{
    RC(check_ctx(x));
    if (x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "%s: not available in a tangent context (it would change the state without its derivatives)", __func__);
    if (cycles < 1) return mgfvm_fail(MGFVM_EINVAL, "cycles must be >= 1");
    RC(pull(x));
    const std::vector<CaseState> saved = x->hs;
    char *backup = nullptr;
    cudaError_t me = ctx_malloc(x, (void **)&backup, x->pool_bytes);
    if (me != cudaSuccess)
        return mgfvm_fail(me == cudaErrorMemoryAllocation ? MGFVM_ENOMEM : MGFVM_ECUDA,
                          "autotune state backup of %zu bytes: %s", x->pool_bytes, cudaGetErrorString(me));
    int rc = MGFVM_OK;
    double t0 = 0.0, best = 0.0;
    auto trial = [&](double *ms) -> int {
        x->hs = saved;                  // histories and flags as before every trial
        RC(push(x));
        return time_schedule(x, cycles, ms);
    };
    do {
        if (cudaMemcpyAsync(backup, x->pool, x->pool_bytes, cudaMemcpyDeviceToDevice, x->stream) != cudaSuccess) {
            rc = mgfvm_fail(MGFVM_ECUDA, "autotune: state backup failed");
            break;
        }
        if ((rc = set_controls(x, 0, 0.0)) != MGFVM_OK) break;
        if ((rc = trial(&t0)) != MGFVM_OK) break;
        best = t0;
        Builder probe{x, nullptr};
        // coordinate descent, level by level, one knob at a time
        for (int ig = 0; ig < x->maxng && rc == MGFVM_OK; ++ig) {
            std::vector<std::vector<int>> knobs;   // {kind, value0, value1}
            int mx, my;
            if (!probe.whole_level(ig, mx, my)) {
                static const int opts[][2] = {{SMOOTH_BLOCK, 10}, {SMOOTH_BLOCK, 4}, {SMOOTH_BLOCK, 6}, {SMOOTH_BLOCK, 16},
                                              {SMOOTH_BLOCK / 2, 4}, {SMOOTH_BLOCK / 2, 6}, {SMOOTH_BLOCK / 2, 10},
                                              {SMOOTH_BLOCK / 4, 3}, {SMOOTH_BLOCK / 4, 5}};
                for (auto &o : opts) knobs.push_back({0, o[0], o[1]});
            }
            if (!probe.whole_level(ig, mx, my)) knobs.push_back({3, 2, 0});
            int bg, bb, bs;
            if (!probe.whole_level(ig, mx, my) && probe.band_level(ig, bg, bb, bs)) {
                knobs.push_back({6, 1, 0});
                knobs.push_back({6, 2, 0});
            }
            if (ig >= 1 && ig >= x->maxng - 3) knobs.push_back({4, 2, 0});   // one-CTA kernel from here down
            if (ig + 1 < x->maxng) knobs.push_back({5, 1, 0});                 // separate correction kernel
            if (ig == 0) knobs.push_back({7, x->tune.coarse_cluster == 2 ? 1 : 2, 0});   // coarse cluster launch
            knobs.push_back({1, 1, 0});
            knobs.push_back({1, 3, 0});
            if (ig + 1 < x->maxng) {
                knobs.push_back({2, 1, 0});
                knobs.push_back({2, 3, 0});
            }
            for (const auto &k : knobs) {
                mgfvm_tuning keep = x->tune, cand = x->tune;
                if (k[0] == 0) { cand.smooth_threads[ig] = k[1]; cand.smooth_units[ig] = k[2]; }
                if (k[0] == 1) cand.asm_slices[ig] = k[1];
                if (k[0] == 2) cand.restrict_slices[ig] = k[1];
                if (k[0] == 3) cand.smooth_tma[ig] = k[1];
                if (k[0] == 4) cand.coarse_kernel[ig] = k[1];
                if (k[0] == 5) cand.prol_fused[ig] = k[1];
                if (k[0] == 6) cand.band_visit[ig] = k[1];
                if (k[0] == 7) cand.coarse_cluster = k[1];
                if (memcmp(&cand, &keep, sizeof cand) == 0) continue;
                x->tune = cand;
                rebuild_schedule(x);
                double t = 0.0;
                if ((rc = trial(&t)) != MGFVM_OK) break;
                if (t < best * 0.99) best = t;
                else {
                    x->tune = keep;
                    rebuild_schedule(x);
                }
            }
        }
    } while (0);
    // restore the batch exactly as it was
    cudaError_t e = cudaMemcpyAsync(x->pool, backup, x->pool_bytes, cudaMemcpyDeviceToDevice, x->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
    ctx_free(x, backup);
    x->hs = saved;
    const int rp = push(x);
    if (rc != MGFVM_OK) return rc;
    if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "autotune: state restore failed: %s", cudaGetErrorString(e));
    if (rp != MGFVM_OK) return rp;
    if (chosen) *chosen = x->tune;
    if (ms_before) *ms_before = t0;
    if (ms_after) *ms_after = best;
    return MGFVM_OK;
}

int mgfvm_profile_cycle(mgfvm_ctx *x, double *ms, int *kernel, int *level, int cap, int *n_out)
{
    RC(check_ctx(x));
    RC(pull(x));
    RC(ensure_hist(x, x->hs[0].ncyc + 1));
    RC(set_controls(x, 0, 0.0));
    const int n = (int)x->cyc.size();
    std::vector<cudaEvent_t> ev(n + 1);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    CK(cudaEventRecord(ev[0], x->stream));
    for (int k = 0; k < n; ++k) {
        cudaError_t e = launch_one(x->cyc[k], x->dc, x->ds, x->dt, x->sched, x->stream);
        if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "profile launch %d: %s", k, cudaGetErrorString(e));
        CK(cudaEventRecord(ev[k + 1], x->stream));
    }
    CK(cudaEventSynchronize(ev[n]));
    x->launches += n;
    for (int k = 0; k < n && k < cap; ++k) {
        float t = 0;
        CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
        if (ms) ms[k] = t;
        if (kernel) kernel[k] = x->cyc[k].kernel;
        if (level) level[k] = x->cyc[k].ig;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (n_out) *n_out = n;
    return MGFVM_OK;
}

int mgfvm_transfer_bytes(mgfvm_ctx *x, long long *h2d, long long *d2h)
{
    if (!x) return mgfvm_fail(MGFVM_EINVAL, "null context");
    if (h2d) *h2d = x->h2d;
    if (d2h) *d2h = x->d2h;
    return MGFVM_OK;
}

// ----------------------------------------------- raw-pointer entry points
static int check_raw(const void *const *ptrs, int n, int npx, int npy, int nx, int ny)
{
    for (int k = 0; k < n; ++k)
        if (!ptrs[k]) return mgfvm_fail(MGFVM_EINVAL, "null device pointer");
    if (npx < 3 || npy < 3 || nx < 1 || ny < 1 || nx > npx - 1 || ny > npy - 1)
        return mgfvm_fail(MGFVM_EINVAL, "extent nx=%d ny=%d does not fit a %d x %d level", nx, ny, npx, npy);
    return MGFVM_OK;
}

int mgfvm_jacobi_f64(const double *aw, const double *ae, const double *as, const double *an, const double *ap,
                     const double *su, double *phi, double *scratch, int npx, int npy, int nx, int ny, int nsw,
                     void *stream)
{
    const void *p[] = {aw, ae, as, an, ap, su, phi, scratch};
    RC(check_raw(p, 8, npx, npy, nx, ny));
    if (nsw < 0) return mgfvm_fail(MGFVM_EINVAL, "negative sweep count");
    CK(mg::raw_jacobi(aw, ae, as, an, ap, su, phi, scratch, npx, npy, nx, ny, nsw, (cudaStream_t)stream));
    return MGFVM_OK;
}

int mgfvm_rbgs_f64(const double *aw, const double *ae, const double *as, const double *an, const double *ap,
                   const double *su, double *phi, int npx, int npy, int nx, int ny, int nsw, void *stream)
{
    const void *p[] = {aw, ae, as, an, ap, su, phi};
    RC(check_raw(p, 7, npx, npy, nx, ny));
    if (nsw < 0) return mgfvm_fail(MGFVM_EINVAL, "negative sweep count");
    CK(mg::raw_rbgs(aw, ae, as, an, ap, su, phi, npx, npy, nx, ny, nsw, (cudaStream_t)stream));
    return MGFVM_OK;
}

size_t mgfvm_masserror_scratch_doubles(int npx, int npy)
{
    return mg::raw_masserror_blocks(npx, npy) * RED_STRIDE + 1;
}

int mgfvm_masserror_f64(const double *u, const double *v, const double *areax, const double *areay, double *su,
                        double *pp, int npx, int npy, double *err_out, double *partials, void *stream)
{
    const void *p[] = {u, v, areax, areay, su, pp, err_out, partials};
    RC(check_raw(p, 8, npx, npy, npx - 1, npy - 1));
    CK(mg::raw_masserror(u, v, areax, areay, su, pp, npx, npy, err_out, partials, (cudaStream_t)stream));
    return MGFVM_OK;
}

int mgfvm_check_division(int device, long long n, unsigned long long seed, long long *mismatches)
{
    if (n < 0 || !mismatches) return mgfvm_fail(MGFVM_EINVAL, "bad count or null output");
    CK(cudaSetDevice(device));
    unsigned long long *bad = nullptr, h = 0;
    CK(cudaMalloc(&bad, sizeof *bad));
    cudaError_t e = cudaMemset(bad, 0, sizeof *bad);
    if (e == cudaSuccess) e = mg::raw_check_division(n, seed, bad, 0);
    if (e == cudaSuccess) e = cudaMemcpy(&h, bad, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(bad);
    if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "division self-test: %s", cudaGetErrorString(e));
    *mismatches = (long long)h;
    return MGFVM_OK;
}

// ------------------------------------------------------------ derivatives
int mgfvm_set_direction(mgfvm_ctx *x, int icase, int kind, int index)
{
    RC(check_ctx(x));
    if (!x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "not a tangent context (mgfvm_options.tangent)");
    if (icase < 0 || icase >= x->ncases) return mgfvm_fail(MGFVM_EINVAL, "case %d out of range", icase);
    if (kind < MGFVM_DIR_NONE || kind > MGFVM_DIR_PRSC) return mgfvm_fail(MGFVM_EINVAL, "unknown direction %d", kind);
    if (kind == MGFVM_DIR_INLET && (index < 0 || index >= x->cfg[icase].nfy))
        return mgfvm_fail(MGFVM_EINVAL, "inlet face %d outside [0, %d)", index, x->cfg[icase].nfy);
    RC(pull(x));
    x->dir_kind[icase] = kind;
    x->dir_index[icase] = kind == MGFVM_DIR_INLET ? index : 0;
    return init_state(x, icase);
}

int mgfvm_get_tangent(mgfvm_ctx *x, int icase, int level, int field, double *out)
{
    RC(check_ctx(x));
    if (!x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "not a tangent context (mgfvm_options.tangent)");
    RC(check_case_level(x, icase, level));
    if (field < 0 || field >= MGFVM_NFIELDS || !out) return mgfvm_fail(MGFVM_EINVAL, "bad field %d", field);
    CK(cudaStreamSynchronize(x->stream));
    const LevelDev &L = x->hc[icase].lv[level];
    const double *t = x->ht[icase].lv[level].t[field_slot(field, x->last_eq[level])];
    const size_t n = (size_t)L.npx * L.npy;
    if (!t) {
        std::fill(out, out + n, 0.0);   // geometry and obstacle sources do not depend on the parameters
        return MGFVM_OK;
    }
    CK(cudaMemcpy(out, t, sizeof(double) * n, cudaMemcpyDeviceToHost));
    x->d2h += (long long)(sizeof(double) * n);
    return MGFVM_OK;
}

// J of the level-0 state (and its derivative from the tangent fields): row means over
// the interior rows j = 1 .. npy-2, summed in row order.
static void objective_of(const double *p, const double *sc, int npx, int npy, double *J)
{
    double sin = 0.0, sout = 0.0, ssc = 0.0;
    for (int j = 1; j <= npy - 2; ++j) {
        sin += p[(size_t)j * npx + 1];
        sout += p[(size_t)j * npx + npx - 2];
        ssc += sc[(size_t)j * npx + npx - 1];
    }
    const double ny = (double)(npy - 2);
    *J = (sin / ny - sout / ny) + ssc / ny;
}

int mgfvm_objective(mgfvm_ctx *x, int icase, double *J, double *dJ)
{
    RC(check_ctx(x));
    RC(check_case_level(x, icase, 0));
    if (dJ && !x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "dJ needs a tangent context (mgfvm_options.tangent)");
    const LevelDev &L = x->hc[icase].lv[0];
    const size_t n = (size_t)L.npx * L.npy;
    std::vector<double> p(n), sc(n);
    if (J) {
        RC(mgfvm_get_field(x, icase, 0, MGFVM_F_P, p.data()));
        RC(mgfvm_get_field(x, icase, 0, MGFVM_F_SC, sc.data()));
        objective_of(p.data(), sc.data(), L.npx, L.npy, J);
    }
    if (dJ) {
        RC(mgfvm_get_tangent(x, icase, 0, MGFVM_F_P, p.data()));
        RC(mgfvm_get_tangent(x, icase, 0, MGFVM_F_SC, sc.data()));
        objective_of(p.data(), sc.data(), L.npx, L.npy, dJ);
    }
    return MGFVM_OK;
}

int mgfvm_gradient(const mgfvm_config *cfg, const double *inlet_u, int n_inlet, int ncycles, int device,
                   double *J, double *dJ_dinlet, double *dJ_damuf, double *dJ_dprsc)
{
    mgfvm_clear_error();
    if (!cfg || ncycles < 0 || n_inlet < 0 || (n_inlet > 0 && !inlet_u))
        return mgfvm_fail(MGFVM_EINVAL, "bad gradient arguments");
    const int nf = cfg->nfy, ndir = nf + 2;
    mgfvm_options opt;
    mgfvm_options_default(&opt);
    opt.device = device;
    opt.tangent = 1;
    // directions in batches: all at once where the device holds them (or at most
    // MGFVM_GRADIENT_BATCH, when set), else halved until a batch fits
    int chunk = ndir;
    if (const char *env = std::getenv("MGFVM_GRADIENT_BATCH")) {
        const int cap = std::atoi(env);
        if (cap >= 1) chunk = std::min(chunk, cap);
    }
    for (int d0 = 0; d0 < ndir;) {
        const int n = std::min(chunk, ndir - d0);
        std::vector<mgfvm_config> cases(n, *cfg);
        mgfvm_ctx *x = nullptr;
        int rc = mgfvm_create(cases.data(), n, &opt, &x);
        if (rc == MGFVM_ENOMEM && chunk > 1) {
            cudaGetLastError();   // the failed allocation's error must not reach the next batch's checks
            chunk = (chunk + 1) / 2;
            continue;
        }
        RC(rc);
        do {
            for (int c = 0; c < n; ++c) {
                const int d = d0 + c;
                x->profile[c].assign(inlet_u, inlet_u + n_inlet);
                x->dir_kind[c] = d < nf ? MGFVM_DIR_INLET : d == nf ? MGFVM_DIR_AMUF : MGFVM_DIR_PRSC;
                x->dir_index[c] = d < nf ? d : 0;
            }
            if ((rc = upload_profiles(x)) != MGFVM_OK) break;
            if ((rc = init_state(x, -1)) != MGFVM_OK) break;
            if ((rc = mgfvm_cycle(x, ncycles)) != MGFVM_OK) break;
            if (d0 == 0 && J && (rc = mgfvm_objective(x, 0, J, nullptr)) != MGFVM_OK) break;
            for (int c = 0; c < n && rc == MGFVM_OK; ++c) {
                const int d = d0 + c;
                double *dst = d < nf ? (dJ_dinlet ? dJ_dinlet + d : nullptr) : d == nf ? dJ_damuf : dJ_dprsc;
                if (dst) rc = mgfvm_objective(x, c, nullptr, dst);
            }
        } while (0);
        mgfvm_destroy(x);
        RC(rc);
        d0 += n;
    }
    return MGFVM_OK;
}

// ------------------------------------------------------------------ adjoint
// Reverse mode of `ncycles` V-cycles from the initial state (mg_adjoint.cuh): the
// forward run keeps the u, v, p, sc arrays of every level (all a cycle reads of the
// previous cycles' results) at the start of every m-th cycle, m ~ sqrt(ncycles); the
// reverse sweep then takes the segments last to first, re-runs each from its
// checkpoint keeping the start of every one of its cycles, and runs the taped cycle
// and its transpose for those cycles last to first.  Memory: (ncycles/m + m) copies
// of those arrays, one cycle's tape and one set of adjoint arrays per case.
int mgfvm_adjoint(mgfvm_ctx *x, int ncycles)
{
    RC(check_ctx(x));
    if (x->opt.tangent) return mgfvm_fail(MGFVM_EINVAL, "mgfvm_adjoint: not available in a tangent context");
    if (x->opt.precision != MGFVM_PREC_FP64)
        return mgfvm_fail(MGFVM_EUNSUPPORTED, "mgfvm_adjoint: FP64 contexts only");
    if (ncycles < 0) return mgfvm_fail(MGFVM_EINVAL, "negative cycle count");
    const int n = x->ncases;
    // the phase programs and their tapes
    std::vector<std::vector<Phase>> progs(n);
    std::vector<long long> tape_n(n), tape_off(n), prog_off(n), live_off(n);
    long long tape_tot = 0, prog_tot = 0, live_tot = 0;
    for (int c = 0; c < n; ++c) {
        if (!build_adj_program(x->hc[c], x->sched, progs[c], tape_n[c]))
            return mgfvm_fail(MGFVM_EUNSUPPORTED, "mgfvm_adjoint: case %d has periodic boundaries (not covered)", c);
        tape_off[c] = tape_tot;
        tape_tot += (tape_n[c] + 31) / 32 * 32;
        prog_off[c] = prog_tot;
        prog_tot += (long long)progs[c].size();
        live_off[c] = live_tot;
        for (int ig = 0; ig < x->cfg[c].ngrid; ++ig) live_tot += 4LL * npx_of(x->cfg[c], ig) * npy_of(x->cfg[c], ig);
    }
    RC(pull(x));
    if (!x->tpool) RC(alloc_tangent(x));     // the adjoint arrays: the derivative storage's layout
    const int m = std::max(1, (int)std::ceil(std::sqrt((double)std::max(ncycles, 1))));
    const int nseg = (ncycles + m - 1) / m;
    // device buffers
    Phase *dprog = nullptr;
    CaseAdj *dadj = nullptr;
    double *tape = nullptr, *pacc = nullptr, *ckpt = nullptr, *seg = nullptr, *fin = nullptr;
    long long *dlive = nullptr;
    const size_t pacc_n = (size_t)n * 2 * MAXLEV;
    std::vector<void **> bufs = {(void **)&dprog, (void **)&dadj, (void **)&tape, (void **)&pacc, (void **)&ckpt,
                                 (void **)&seg, (void **)&fin, (void **)&dlive};
    const size_t sizes[] = {sizeof(Phase) * (size_t)std::max<long long>(prog_tot, 1), sizeof(CaseAdj) * (size_t)n,
                            sizeof(double) * (size_t)std::max<long long>(tape_tot, 1), sizeof(double) * pacc_n,
                            sizeof(double) * (size_t)live_tot * std::max(nseg, 1), sizeof(double) * (size_t)live_tot * m,
                            sizeof(double) * (size_t)live_tot, sizeof(long long) * (size_t)n};
    auto release = [&]() {
        cudaStreamSynchronize(x->stream);
        for (void **b : bufs)
            if (*b) {
                ctx_free(x, *b);
                *b = nullptr;
            }
    };
    for (size_t k = 0; k < bufs.size(); ++k) {
        cudaError_t me = ctx_malloc(x, bufs[k], sizes[k]);
        if (me != cudaSuccess) {
            *bufs[k] = nullptr;
            release();
            cudaGetLastError();
            return mgfvm_fail(me == cudaErrorMemoryAllocation ? MGFVM_ENOMEM : MGFVM_ECUDA,
                              "mgfvm_adjoint: %zu bytes of checkpoints, tape or programs: %s", sizes[k],
                              cudaGetErrorString(me));
        }
    }
    int rc = MGFVM_OK;
    std::vector<CaseState> hs_final;
    const int maxng = x->maxng, maxcells = *std::max_element(x->maxcells.begin(), x->maxcells.end());
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device);
    int cluster = adj_cluster_size(n, std::max(sms, 1));
    if (const char *env = std::getenv("MGFVM_ADJOINT_CLUSTER")) {
        const int v = std::atoi(env);
        if (v == 1 || v == 2 || v == 4 || v == 8) cluster = v;
    }
    auto live = [&](double *buf, int dir) -> int {
        cudaError_t e = launch_live_copy(x->dc, dlive, buf, n, maxcells, maxng, dir, x->stream);
        if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "checkpoint copy: %s", cudaGetErrorString(e));
        return MGFVM_OK;
    };
    do {
        // programs, per-case descriptors
        std::vector<Phase> flat;
        flat.reserve((size_t)prog_tot);
        for (auto &pg : progs) flat.insert(flat.end(), pg.begin(), pg.end());
        std::vector<CaseAdj> ha(n);
        const char *gen = std::getenv("MGFVM_ADJOINT_GENERIC");
        const int generic = gen && std::atoi(gen) == 1 ? 1 : 0;
        for (int c = 0; c < n; ++c)
            ha[c] = CaseAdj{dprog + prog_off[c], (int)progs[c].size(), tape + tape_off[c], pacc + (size_t)c * 2 * MAXLEV,
                            generic};
        if (cudaMemcpy(dprog, flat.data(), sizeof(Phase) * flat.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dadj, ha.data(), sizeof(CaseAdj) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dlive, live_off.data(), sizeof(long long) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(pacc, 0, sizeof(double) * pacc_n) != cudaSuccess) {
            rc = mgfvm_fail(MGFVM_ECUDA, "mgfvm_adjoint: upload: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        x->h2d += (long long)(sizeof(Phase) * flat.size() + sizeof(CaseAdj) * n + sizeof(long long) * n);
        // forward: from the initial state, checkpoints at the start of every m-th cycle
        if ((rc = init_state(x, -1)) != MGFVM_OK) break;
        if ((rc = ensure_hist(x, ncycles)) != MGFVM_OK) break;
        if ((rc = set_controls(x, 0, 0.0)) != MGFVM_OK) break;
        if (cudaEventRecord(x->e0, x->stream) != cudaSuccess) { rc = mgfvm_fail(MGFVM_ECUDA, "event"); break; }
        for (int sgi = 0; sgi < nseg && rc == MGFVM_OK; ++sgi) {
            rc = live(ckpt + (size_t)sgi * live_tot, 0);
            if (rc == MGFVM_OK) rc = run_cycles(x, std::min(m, ncycles - sgi * m));
        }
        if (rc != MGFVM_OK || (rc = live(fin, 0)) != MGFVM_OK) break;
        if ((rc = pull(x)) != MGFVM_OK || (rc = check_status(x)) != MGFVM_OK) break;
        hs_final = x->hs;
        // J of every case, and its adjoint seed on level 0 (zero elsewhere)
        x->adj_J.assign(n, 0.0);
        x->adj_bad.assign(n, 0);
        CK(cudaMemsetAsync(x->tpool, 0, x->tcase_off.empty() ? 0 : x->tcase_off.back() + x->tcase_bytes.back(),
                           x->stream));
        for (int c = 0; c < n && rc == MGFVM_OK; ++c) {
            const LevelDev &L = x->hc[c].lv[0];
            const size_t cells = (size_t)L.npx * L.npy;
            std::vector<double> p(cells), sc(cells), bp(cells, 0.0), bsc(cells, 0.0);
            if ((rc = mgfvm_get_field(x, c, 0, MGFVM_F_P, p.data())) != MGFVM_OK) break;
            if ((rc = mgfvm_get_field(x, c, 0, MGFVM_F_SC, sc.data())) != MGFVM_OK) break;
            // a case whose iteration diverged (the reference's does on the same inputs) has
            // no derivative; its transpose runs on non-finite values without touching the
            // other cases, and its gradient is reported as such
            bool finite = true;
            for (size_t k = 0; k < cells; ++k) finite &= std::isfinite(p[k]) && std::isfinite(sc[k]);
            x->adj_bad[c] = !finite;
            objective_of(p.data(), sc.data(), L.npx, L.npy, &x->adj_J[c]);
            const double ny = (double)(L.npy - 2);
            for (int j = 1; j <= L.npy - 2; ++j) {
                bp[(size_t)j * L.npx + 1] += 1.0 / ny;
                bp[(size_t)j * L.npx + L.npx - 2] += -1.0 / ny;
                bsc[(size_t)j * L.npx + L.npx - 1] += 1.0 / ny;
            }
            const LevelTan &B = x->ht[c].lv[0];
            if (cudaMemcpy(B.t[S_P], bp.data(), sizeof(double) * cells, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(B.t[S_SC], bsc.data(), sizeof(double) * cells, cudaMemcpyHostToDevice) != cudaSuccess) {
                rc = mgfvm_fail(MGFVM_ECUDA, "mgfvm_adjoint: seed: %s", cudaGetErrorString(cudaGetLastError()));
                break;
            }
            x->h2d += (long long)(2 * sizeof(double) * cells);
        }
        if (rc != MGFVM_OK) break;
        // reverse: segments last to first
        for (int sgi = nseg - 1; sgi >= 0 && rc == MGFVM_OK; --sgi) {
            const int cnt = std::min(m, ncycles - sgi * m);
            rc = live(ckpt + (size_t)sgi * live_tot, 1);
            for (int k = 0; k < cnt && rc == MGFVM_OK; ++k) {
                rc = live(seg + (size_t)k * live_tot, 0);
                if (rc == MGFVM_OK && k + 1 < cnt) rc = run_cycles(x, 1);
            }
            for (int k = cnt - 1; k >= 0 && rc == MGFVM_OK; --k) {
                rc = live(seg + (size_t)k * live_tot, 1);
                if (rc != MGFVM_OK) break;
                cudaError_t e = launch_adj_cycle(x->dc, x->ds, x->dt, dadj, n, cluster, x->stream);
                if (e != cudaSuccess) rc = mgfvm_fail(MGFVM_ECUDA, "adjoint cycle: %s", cudaGetErrorString(e));
                x->launches += 1;
            }
        }
        if (rc != MGFVM_OK) break;
        if (cudaEventRecord(x->e1, x->stream) != cudaSuccess || cudaEventSynchronize(x->e1) != cudaSuccess) {
            rc = mgfvm_fail(MGFVM_ECUDA, "mgfvm_adjoint: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, x->e0, x->e1);
        x->last_ms = ms;
        if ((rc = pull(x)) != MGFVM_OK) break;
        for (int c = 0; c < n; ++c)
            if (x->hs[c].status & CASE_TAPE_ESCAPE) {
                rc = mgfvm_fail(MGFVM_ECUDA, "mgfvm_adjoint: a phase of case %d wrote outside its tape", c);
                break;
            }
        if (rc != MGFVM_OK || (rc = check_status(x)) != MGFVM_OK) break;
        // gradients: the adjoint of the initial state through the parameters' seeding
        // (the inlet face value and the coarse faces rest_geom averages from it; amu and
        // amusc = amuf / prsc on every level)
        std::vector<double> hp(pacc_n);
        CK(cudaMemcpy(hp.data(), pacc, sizeof(double) * pacc_n, cudaMemcpyDeviceToHost));
        x->d2h += (long long)(sizeof(double) * pacc_n);
        x->adj_gin.assign(n, {});
        x->adj_gamuf.assign(n, 0.0);
        x->adj_gprsc.assign(n, 0.0);
        for (int c = 0; c < n && rc == MGFVM_OK; ++c) {
            const mgfvm_config &g = x->cfg[c];
            std::vector<std::vector<double>> col(g.ngrid);
            for (int ig = 0; ig < g.ngrid; ++ig) {
                const int npx = npx_of(g, ig), npy = npy_of(g, ig);
                col[ig].assign(npy, 0.0);
                if (cudaMemcpy2D(col[ig].data(), sizeof(double), x->ht[c].lv[ig].t[S_U], sizeof(double) * npx,
                                 sizeof(double), npy, cudaMemcpyDeviceToHost) != cudaSuccess) {
                    rc = mgfvm_fail(MGFVM_ECUDA, "mgfvm_adjoint: %s", cudaGetErrorString(cudaGetLastError()));
                    break;
                }
                x->d2h += (long long)(sizeof(double) * npy);
            }
            if (rc != MGFVM_OK) break;
            std::vector<double> acc = col[g.ngrid - 1];
            for (int ig = g.ngrid - 1; ig > 0; --ig) {
                std::vector<double> fine = col[ig - 1];
                for (int jc = 1; jc <= (int)acc.size() - 2; ++jc) {
                    fine[2 * jc] += 0.5 * acc[jc];
                    fine[2 * jc - 1] += 0.5 * acc[jc];
                }
                acc.swap(fine);
            }
            x->adj_gin[c].assign(acc.begin() + 1, acc.begin() + 1 + g.nfy);
            double ga = 0.0, gs = 0.0;
            for (int ig = 0; ig < g.ngrid; ++ig) {
                const double bamu = hp[(size_t)c * 2 * MAXLEV + 2 * ig], bamusc = hp[(size_t)c * 2 * MAXLEV + 2 * ig + 1];
                ga += bamu + bamusc * (1.0 / g.prsc);
                gs += bamusc * (-g.amuf / (g.prsc * g.prsc));
            }
            x->adj_gamuf[c] = ga;
            x->adj_gprsc[c] = gs;
        }
        if (rc != MGFVM_OK) break;
        // leave u, v, p, sc and the histories as the forward run left them
        if ((rc = live(fin, 1)) != MGFVM_OK) break;
        x->hs = hs_final;
        rc = push(x);
        if (rc == MGFVM_OK) x->adj_cycles = ncycles;
    } while (0);
    release();
    return rc;
}

int mgfvm_adjoint_gradient(mgfvm_ctx *x, int icase, double *J, double *dJ_dinlet, double *dJ_damuf, double *dJ_dprsc)
{
    RC(check_ctx(x));
    if (icase < 0 || icase >= x->ncases) return mgfvm_fail(MGFVM_EINVAL, "case %d out of range", icase);
    if (x->adj_cycles < 0 || (int)x->adj_J.size() != x->ncases)
        return mgfvm_fail(MGFVM_EINVAL, "mgfvm_adjoint_gradient: no mgfvm_adjoint has run on this context");
    const bool bad = x->adj_bad[icase] != 0;
    const double nan = std::nan("");
    if (J) *J = x->adj_J[icase];
    if (dJ_dinlet) {
        if (bad) std::fill(dJ_dinlet, dJ_dinlet + x->adj_gin[icase].size(), nan);
        else std::copy(x->adj_gin[icase].begin(), x->adj_gin[icase].end(), dJ_dinlet);
    }
    if (dJ_damuf) *dJ_damuf = bad ? nan : x->adj_gamuf[icase];
    if (dJ_dprsc) *dJ_dprsc = bad ? nan : x->adj_gprsc[icase];
    if (bad)
        return mgfvm_fail(MGFVM_ENONFINITE, "case %d turned non-finite within the %d cycles: no gradient", icase,
                          x->adj_cycles);
    return MGFVM_OK;
}

}  // extern "C"
