// mg_init.cu — device construction of the initial state of every case:
// init (Version-6-26-04.c:546-676) and rest_geom (:1391-1473).
//
// The reference runs these once on the host.  Here they run on the device so a
// batch of hundreds of cases is never materialised in host memory:
//   k_init_fill      every array's default, then the four boundary loops (:581-612)
//                    applied per cell in the reference's order (x-, x+, y-, y+);
//   k_init_obstacles the obstacle loop (:616-641); all its writes are constants, so
//                    any write order gives the same result;
//   k_init_ports     discrete inlets then outlets (:645-674), one thread per row
//                    walking the lists in order so overlapping entries resolve as in
//                    the reference;
//   k_init_profile   the optional per-face inlet profile (before rest_geom);
//   k_rest_geom      one coarse level from its fine level: face areas, then the
//                    x- and x+ boundary u, v (the three loops touch disjoint cells,
//                    and levels run finest first as in the reference).
#include "mg_init.cuh"

namespace mg {

__global__ void k_init_fill(const CaseDev *__restrict__ cs, const InitDev *in, int ig)
{
    const CaseDev &C = cs[blockIdx.y];
    if (ig >= C.ngrid) return;
    const InitDev &P = in[blockIdx.y];
    const LevelDev &L = C.lv[ig];
    const int nx = L.npx, ny = L.npy;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nx * ny) return;
    const int i = t % nx, j = t / nx;
    double u = P.guess[0], v = P.guess[1], p = P.guess[2], sc = P.guess[3];
    if (i == 0) { u = P.bc[0][0]; v = P.bc[0][1]; p = P.bc[0][2]; sc = P.bc[0][3]; }
    if (i == nx - 1) { v = P.bc[1][1]; p = P.bc[1][2]; sc = P.bc[1][3]; }
    if (i == nx - 2) { u = P.bc[1][0]; }
    if (j == 0) { u = P.bc[2][0]; v = P.bc[2][1]; p = P.bc[2][2]; sc = P.bc[2][3]; }
    if (j == ny - 1) { u = P.bc[3][0]; v = P.bc[3][1]; p = P.bc[3][2]; sc = P.bc[3][3]; }
    MGF(L, S_U)[t] = u; MGF(L, S_V)[t] = v; MGF(L, S_P)[t] = p; MGF(L, S_SC)[t] = sc;
    const int zero_slots[] = {S_PP, S_RS, S_RESU, S_RESV, S_RESSC, S_C, S_SPU, S_SPV, S_SPSC, S_CX, S_CY,
                              S_TMP0, S_TMP1, S_TMP2, S_CU, S_CV, S_CP};
    for (int k = 0; k < (int)(sizeof zero_slots / sizeof zero_slots[0]); ++k) MGF(L, zero_slots[k])[t] = 0.0;
    for (int s = S_CO; s < NSLOTS_LEVEL; ++s) MGF(L, s)[t] = 0.0;
    MGF(L, S_APU)[t] = 1.0e30;
    MGF(L, S_APV)[t] = 1.0e30;
    MGF(L, S_AREAX)[t] = L.dy;
    MGF(L, S_AREAY)[t] = L.dx;
    L.tag[t] = 1;
    if (ig == 0)
        for (int s = S_PREV_U; s <= S_PREV_SC; ++s) MGF(L, s)[t] = 0.0;
}

// AllocateMemorySoA's level mapping of obstacle k (:470-476); only called for ig < ig_obs.
__device__ __forceinline__ void obstacle_range(const InitDev &P, int k, int ig, int r[4])
{
    const int fac = 1 << (P.ig_obs - 1 - ig);
    const int *o = &P.obs[4 * k];
    r[0] = (o[0] + P.ibeg_obs - 1) * fac + 1;
    r[1] = (o[1] + P.ibeg_obs) * fac;
    r[2] = (o[2] - 1) * fac + 1;
    r[3] = o[3] * fac;
}

__global__ void k_init_obstacles(const CaseDev *__restrict__ cs, const InitDev *in, int ig)
{
    const CaseDev &C = cs[blockIdx.y];
    const InitDev &P = in[blockIdx.y];
    const int k = blockIdx.x;
    if (ig >= C.ngrid || ig >= P.ig_obs || k >= P.nobs) return;
    const LevelDev &L = C.lv[ig];
    const int nx = L.npx;
    int r[4];
    obstacle_range(P, k, ig, r);
    const int wi = r[1] - r[0] + 1, wj = r[3] - r[2] + 1;
    if (wi <= 0 || wj <= 0) return;
    for (int t = threadIdx.x; t < wi * wj; t += blockDim.x) {
        const int i = r[0] + t % wi, j = r[2] + t / wi, q = j * nx + i;
        MGF(L, S_U)[q] = 0.0; MGF(L, S_V)[q] = 0.0;
        MGF(L, S_U)[q - 1] = 0.0; MGF(L, S_V)[q - nx] = 0.0;
        MGF(L, S_SPU)[q] = 1.0e30; MGF(L, S_SPV)[q] = 1.0e30;
        MGF(L, S_SPU)[q - 1] = 1.0e30; MGF(L, S_SPV)[q - nx] = 1.0e30;
        MGF(L, S_SPSC)[q] = 1.0e30;
        L.tag[q] = 0;
        MGF(L, S_SC)[q] = P.sc_obs;
    }
}

__global__ void k_init_ports(const CaseDev *__restrict__ cs, const InitDev *in, int ig)
{
    const CaseDev &C = cs[blockIdx.y];
    const InitDev &P = in[blockIdx.y];
    if (ig >= C.ngrid) return;
    const LevelDev &L = C.lv[ig];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L.npy) return;
    const int nx = L.npx;
    if (ig < P.ig_inlt) {
        const int fac = 1 << (P.ig_inlt - 1 - ig);
        for (int k = 0; k < P.ninlt; ++k) {
            const int js = (P.jf_in[k] - 1) * fac + 1, je = P.jl_in[k] * fac;
            if (j >= js && j <= je) {
                const int q = j * nx;
                MGF(L, S_U)[q] = P.in_val[k][0]; MGF(L, S_V)[q] = P.in_val[k][1]; MGF(L, S_SC)[q] = P.in_val[k][2];
            }
        }
    }
    if (ig < P.ig_outlt) {
        const int fac = 1 << (P.ig_outlt - 1 - ig);
        for (int k = 0; k < P.noutlt; ++k) {
            const int js = (P.jf_out[k] - 1) * fac + 1, je = P.jl_out[k] * fac;
            if (j >= js && j <= je) {
                const int q = j * nx + nx - 2;
                MGF(L, S_U)[q] = P.out_val[k][0]; MGF(L, S_V)[q] = P.out_val[k][1]; MGF(L, S_SC)[q + 1] = P.out_val[k][2];
            }
        }
    }
}

__global__ void k_init_profile(const CaseDev *__restrict__ cs, const InitDev *in)
{
    const CaseDev &C = cs[blockIdx.y];
    const InitDev &P = in[blockIdx.y];
    if (!P.profile || P.nprofile <= 0) return;
    const LevelDev &L = C.lv[0];
    const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (j > P.nprofile || j >= L.npy - 1) return;
    MGF(L, S_U)[j * L.npx] = P.profile[j - 1];
}

__global__ void k_rest_geom(const CaseDev *__restrict__ cs, int ig)
{
    const CaseDev &C = cs[blockIdx.y];
    if (ig >= C.ngrid || ig < 1) return;
    const LevelDev &F = C.lv[ig - 1], &K = C.lv[ig];
    const int nxf = F.npx, nxc = K.npx, nyc = K.npy;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nxc * nyc) return;
    const int ic = t % nxc, jc = t / nxc, q = 2 * jc * nxf + 2 * ic;
    if (jc >= 1 && jc <= nyc - 2 && ic <= nxc - 2)
        MGF(K, S_AREAX)[t] = MGF(F, S_AREAX)[q] + MGF(F, S_AREAX)[q - nxf];
    if (jc <= nyc - 2 && ic >= 1 && ic <= nxc - 2)
        MGF(K, S_AREAY)[t] = MGF(F, S_AREAY)[q] + MGF(F, S_AREAY)[q - 1];
    if (jc >= 1 && jc <= nyc - 2 && ic == 0) {
        MGF(K, S_U)[t] = 0.5 * (MGF(F, S_U)[q] + MGF(F, S_U)[q - nxf]);
        MGF(K, S_V)[t] = 0.5 * (MGF(F, S_V)[q] + MGF(F, S_V)[q - 1]);
    }
    if (jc >= 1 && jc <= nyc - 2 && ic == nxc - 2) {
        MGF(K, S_U)[t] = 0.5 * (MGF(F, S_U)[q] + MGF(F, S_U)[q - nxf]);
        MGF(K, S_V)[t] = 0.5 * (MGF(F, S_V)[q] + MGF(F, S_V)[q - 1]);
    }
}

cudaError_t launch_init(CaseDev *dcases, const InitDev *dinit, int ncases, int maxng, const int *max_cells,
                        int max_obs, int max_npy, cudaStream_t s)
{
    const int B = 256;
    for (int ig = 0; ig < maxng; ++ig) {
        dim3 g((max_cells[ig] + B - 1) / B, ncases);
        k_init_fill<<<g, B, 0, s>>>(dcases, dinit, ig);
        if (max_obs > 0) k_init_obstacles<<<dim3(max_obs, ncases), 128, 0, s>>>(dcases, dinit, ig);
        k_init_ports<<<dim3((max_npy + B - 1) / B, ncases), B, 0, s>>>(dcases, dinit, ig);
    }
    k_init_profile<<<dim3((max_npy + B - 1) / B, ncases), B, 0, s>>>(dcases, dinit);
    for (int ig = 1; ig < maxng; ++ig) {
        dim3 g((max_cells[ig] + B - 1) / B, ncases);
        k_rest_geom<<<g, B, 0, s>>>(dcases, ig);
    }
    return cudaGetLastError();
}

}  // namespace mg
