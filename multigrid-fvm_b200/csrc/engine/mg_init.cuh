// mg_init.cuh — per-case parameters of the device-side initial state.
#pragma once

#include "mg_cells.cuh"

namespace mg {

struct InitDev {
    double guess[4];          // u, v, p, sc initial guess (InputData line 8)
    double bc[4][4];          // x-, x+, y-, y+ boundary (u, v, p, sc) (lines 4-7)
    double sc_obs;
    int ig_obs, ibeg_obs, nobs;
    const int *obs;           // 4*nobs pattern.txt rectangles
    int ig_inlt, ninlt, ig_outlt, noutlt;
    int jf_in[MGFVM_MAX_PORTS], jl_in[MGFVM_MAX_PORTS];
    int jf_out[MGFVM_MAX_PORTS], jl_out[MGFVM_MAX_PORTS];
    double in_val[MGFVM_MAX_PORTS][3], out_val[MGFVM_MAX_PORTS][3];
    const double *profile;    // optional level-0 inlet u profile
    int nprofile;
};

cudaError_t launch_init(CaseDev *dcases, const InitDev *dinit, int ncases, int maxng, const int *max_cells,
                        int max_obs, int max_npy, cudaStream_t s);

}  // namespace mg
