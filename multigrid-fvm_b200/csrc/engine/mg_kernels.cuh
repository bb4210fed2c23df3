// mg_kernels.cuh — host-side launchers of the engine's kernels.
#pragma once

#include "mg_common.cuh"

namespace mg {

// One kernel launch of the V-cycle schedule.
enum KernelId {
    K_FLUXES = 0, K_MOM_U, K_MOM_V, K_MASS_COEFP, K_UPDATE, K_PFIX, K_PERIODIC, K_OUTFLOW,
    K_SC, K_JACOBI, K_JACOBI_COPYBACK, K_GS, K_RESTV, K_RESTRICT, K_PROL_CORR, K_PROL_APPLY,
    K_TAIL, K_ENDCYCLE, K_NKERNELS
};

struct Launch {
    int kernel;     // KernelId
    int ig;         // level (fine level for transfers)
    int mode;       // enum Mode
    int a0, a1, a2; // kernel-specific: equation, sweep/colour, flags
    dim3 grid;
    int block;
};

struct Sched {
    int isolve, nswpm, nswpp;
};

// Launch one schedule entry on `stream`; returns the CUDA error of the launch.
cudaError_t launch_one(const Launch &L, CaseDev *dcases, const Sched &S, cudaStream_t stream);

// Kernels of the raw-pointer entry points.
cudaError_t raw_jacobi(const double *aw, const double *ae, const double *as, const double *an,
                       const double *ap, const double *su, double *phi, double *scratch, int npx,
                       int npy, int nx, int ny, int nsw, cudaStream_t s);
cudaError_t raw_rbgs(const double *aw, const double *ae, const double *as, const double *an,
                     const double *ap, const double *su, double *phi, int npx, int npy, int nx,
                     int ny, int nsw, cudaStream_t s);
cudaError_t raw_masserror(const double *u, const double *v, const double *ax, const double *ay,
                          double *su, double *pp, int npx, int npy, double *err_out,
                          double *partials, cudaStream_t s);
size_t raw_masserror_blocks(int npx, int npy);

constexpr int BLOCK = 256;
constexpr int TAIL_BLOCK = 512;

}  // namespace mg
