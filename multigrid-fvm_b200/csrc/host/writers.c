/*
 * writers.c — the reference's output files, byte for byte.
 *
 * mgfvm_write_vtk restates write_vtk_2d_cc (Version-6-26-04.c:2261-2363): legacy
 * ASCII VTK of the level-0 interior with cell-centred velocity (face averages),
 * pressure, scalar and an obstacle flag, all with `%f`, followed by the three
 * diagnostic stdout lines (mean |velocity|, mean x-velocity, tortuosity).  The
 * obstacle flag is rasterised once instead of testing every rectangle per cell.
 *
 * mgfvm_write_convergence restates write_convergence_data_file (:2544-2558),
 * including its quirks: it writes the first `nconverged` entries (the index of the
 * last cycle run, so the last cycle's entry is not written) and reports `nvcycle`
 * records in its message.
 */
#include "mgfvm_host.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int mgfvm_write_vtk(const char *path, const mgfvm_config *c, int nx, int ny, const double *u,
                    const double *v, const double *p, const double *sc, const int *obs_ranges,
                    int iter, double diag_out[3])
{
    const int I = nx - 2, J = ny - 2, N = I * J;
    const double dx = c->xl / (nx - 2), dy = c->yl / (ny - 2);
    double sum_vx = 0.0, sum_mag = 0.0;
    FILE *fp = fopen(path, "w");
    if (!fp) {
        perror("fopen");
        return mgfvm_fail(MGFVM_EIO, "cannot open %s for writing", path);
    }
    fprintf(fp, "# vtk DataFile Version 3.0\n");
    fprintf(fp, "2D SIMPLE output iter %d\n", iter);
    fprintf(fp, "ASCII\n");
    fprintf(fp, "DATASET STRUCTURED_GRID\n");
    fprintf(fp, "DIMENSIONS %d %d 1\n", I, J);
    fprintf(fp, "POINTS %d float\n", N);
    for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) {
            double x = (i - 0.5) * dx;
            double y = (j - 0.5) * dy;
            fprintf(fp, "%f %f 0.0\n", x, y);
        }
    fprintf(fp, "\nPOINT_DATA %d\n", N);
    fprintf(fp, "VECTORS Velocity float\n");
    for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) {
            int q = j * nx + i;
            double ucc = 0.5 * (u[q] + u[q - 1]);
            double vcc = 0.5 * (v[q] + v[q - nx]);
            sum_vx += ucc;
            sum_mag += sqrt(ucc * ucc + vcc * vcc);
            fprintf(fp, "%f %f 0.0\n", ucc, vcc);
        }
    fprintf(fp, "\nSCALARS P float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) fprintf(fp, "%f\n", p[j * nx + i]);
    fprintf(fp, "\nSCALARS SC float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (int j = 1; j <= J; ++j)
        for (int i = 1; i <= I; ++i) fprintf(fp, "%f\n", sc[j * nx + i]);
    fprintf(fp, "\nSCALARS OBS float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    if (c->nobs > 0) {
        unsigned char *mask = (unsigned char *)calloc((size_t)nx * ny, 1);
        if (!mask) { fclose(fp); return mgfvm_fail(MGFVM_ENOMEM, "vtk obstacle mask"); }
        for (int k = 0; k < c->nobs; ++k) {
            const int *r = &obs_ranges[4 * k];
            for (int j = r[2] > 1 ? r[2] : 1; j <= r[3] && j <= J; ++j)
                for (int i = r[0] > 1 ? r[0] : 1; i <= r[1] && i <= I; ++i) mask[j * nx + i] = 1;
        }
        for (int j = 1; j <= J; ++j)
            for (int i = 1; i <= I; ++i) fprintf(fp, "%f\n", mask[j * nx + i] ? 1.0 : 0.0);
        free(mask);
    }
    fclose(fp);
    printf("Average velocity magnitude at iter %d: %e\n", iter, sum_mag / N);
    printf("Average x-velocity at iter %d: %e\n", iter, sum_vx / N);
    printf("Tortuosity at iter %d: %e\n", iter, (sum_mag) / (sum_vx));
    if (diag_out) {
        diag_out[0] = sum_mag / N;
        diag_out[1] = sum_vx / N;
        diag_out[2] = sum_mag / sum_vx;
    }
    return MGFVM_OK;
}

int mgfvm_write_convergence(const char *path, const double *hist, int nconverged, int nvcycle,
                            int verbose)
{
    FILE *fp = fopen(path, "w");
    if (!fp) {
        fprintf(stderr, "ERROR: Could not open convergence_data file %s for writing.\n", path);
        return mgfvm_fail(MGFVM_EIO, "cannot open %s for writing", path);
    }
    fprintf(fp, "Iteration,convergence_data\n");
    for (int i = 0; i < nconverged; i++) fprintf(fp, "%d,%e\n", i + 1, hist[i]);
    fclose(fp);
    if (verbose) printf("Successfully wrote %d convergence_data records to %s\n", nvcycle, path);
    return MGFVM_OK;
}
