/*
 * A C program that uses libffs_lbm.so through include/ffs_lbm.h only (no
 * Python, no torch): it creates a D2Q9 channel with a cylinder given as a
 * device surface, starts it in uniform flow, steps it, and checks the
 * density, the flow downstream, the status word and the drag on the
 * cylinder; then it steps the same cylinder as the surface of a volume mesh
 * through the coupled entry point.  It is what a
 * C or C++ host (the reference's Simulator2D, a solver of another language
 * through its FFI) does with the library.
 *
 * Exit status 0 on success; the message says what failed otherwise.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "ffs_lbm.h"

#define CHECK(expr)                                                                                                    \
    do {                                                                                                               \
        ffs_status s_ = (expr);                                                                                        \
        if (s_ != FFS_OK) {                                                                                            \
            fprintf(stderr, "%s failed: %s (%s)\n", #expr, ffs_status_string(s_), ffs_last_error());                   \
            return 1;                                                                                                  \
        }                                                                                                              \
    } while (0)

int main(void)
{
    const int nx = 128, ny = 64, nseg = 48, steps = 40;
    const double dx = 0.01;
    ffs_lbm_desc d = {0};
    d.dim = 2;
    d.nx = nx;
    d.ny = ny;
    d.nz = 1;
    d.fluid_viscosity = 0.02;
    d.fluid_density = 1.0;
    d.fluid_dx = dx;
    d.dt = 0.005;
    d.boundary_velocities[0] = 0.04f; /* InletLeft */
    d.storage = FFS_STORAGE_F32;
    ffs_lbm *g = NULL;
    CHECK(ffs_lbm_create(&d, &g));
    if (ffs_abi_version() != FFS_ABI_VERSION) { fprintf(stderr, "ABI version mismatch\n"); return 1; }

    /* walls top and bottom, inlet left, outlet right (LbmNodeFlag values) */
    unsigned char *flags = malloc((size_t)nx * ny);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            unsigned char f = 1;
            if (y == 0 || y == ny - 1) f = 5;
            else if (x == 0) f = 13;
            else if (x == nx - 1) f = 20;
            flags[y * nx + x] = f;
        }
    CHECK(ffs_lbm_set_flags(g, flags, FFS_MEM_HOST, NULL));
    CHECK(ffs_lbm_initialize(g, NULL));

    /* uniform flow at the inlet velocity in every cell: equilibrium moments
     * rho = 1, u = (0.04, 0), pi_xx = ux^2, pi_yy = pi_xy = 0 */
    float *m = malloc(sizeof(float) * 6 * (size_t)nx * ny);
    for (size_t c = 0; c < (size_t)nx * ny; ++c) {
        float *mc = m + 6 * c;
        mc[0] = 1.0f;
        mc[1] = 0.04f;
        mc[2] = 0.0f;
        mc[3] = 0.04f * 0.04f;
        mc[4] = 0.0f;
        mc[5] = 0.0f;
    }
    CHECK(ffs_lbm_set_moments(g, m, FFS_LAYOUT_AOS, FFS_MEM_HOST, FFS_BUF_BOTH, NULL));

    /* a static cylinder: polygon of nseg segments, radius 8 cells at (32, 32) */
    float hv[2 * 48], hu[2 * 48] = {0};
    unsigned int he[2 * 48];
    for (int i = 0; i < nseg; ++i) {
        const double th = 2.0 * 3.14159265358979 * i / nseg;
        hv[2 * i] = (float)((32.0 + 8.0 * cos(th)) * dx);
        hv[2 * i + 1] = (float)((32.0 + 8.0 * sin(th)) * dx);
        he[2 * i] = (unsigned)i;
        he[2 * i + 1] = (unsigned)((i + 1) % nseg);
    }
    float *dv, *du, *dfrc;
    unsigned int *de;
    if (cudaMalloc((void **)&dv, sizeof hv) || cudaMalloc((void **)&du, sizeof hu) ||
        cudaMalloc((void **)&de, sizeof he) || cudaMalloc((void **)&dfrc, sizeof hv)) {
        fprintf(stderr, "cudaMalloc failed\n");
        return 1;
    }
    cudaMemcpy(dv, hv, sizeof hv, cudaMemcpyHostToDevice);
    cudaMemcpy(du, hu, sizeof hu, cudaMemcpyHostToDevice);
    cudaMemcpy(de, he, sizeof he, cudaMemcpyHostToDevice);
    cudaMemset(dfrc, 0, sizeof hv);
    ffs_surface s = {2, dv, du, de, nseg, nseg, dfrc, NULL};

    /* cells inside the polygon become SolidDynamic (about pi * 8^2 of them) */
    CHECK(ffs_lbm_fill_solid(g, &s, NULL));
    CHECK(ffs_lbm_get_flags(g, flags, FFS_MEM_HOST, NULL));
    int inside = 0;
    for (int c = 0; c < nx * ny; ++c) inside += flags[c] == 4;
    if (inside < 180 || inside > 220) { fprintf(stderr, "%d cells inside the cylinder\n", inside); return 1; }

    for (int t = 0; t < steps; ++t) CHECK(ffs_lbm_step(g, &s, NULL));
    uint32_t status = 0;
    CHECK(ffs_lbm_get_status(g, &status, 1, NULL));
    if (status) { fprintf(stderr, "device status %u\n", status); return 1; }

    CHECK(ffs_lbm_get_moments(g, m, FFS_LAYOUT_AOS, FFS_MEM_HOST, FFS_BUF_CURRENT, NULL));
    double rho_min = 1e30, rho_max = -1e30, ux_mean = 0.0;
    int n = 0;
    for (int y = 1; y < ny - 1; ++y)
        for (int x = 80; x < 120; ++x) {
            const float *c = m + 6 * ((size_t)y * nx + x);
            rho_min = fmin(rho_min, c[0]);
            rho_max = fmax(rho_max, c[0]);
            ux_mean += c[1];
            ++n;
        }
    ux_mean /= n;
    float hf[2 * 48];
    cudaMemcpy(hf, dfrc, sizeof hf, cudaMemcpyDeviceToHost);
    double fx = 0.0;
    for (int i = 0; i < nseg; ++i) fx += hf[2 * i];
    printf("rho in [%.6f, %.6f], mean ux downstream %.5f, drag sum %.6g\n", rho_min, rho_max, ux_mean, fx);
    if (!(rho_min > 0.9 && rho_max < 1.1)) { fprintf(stderr, "density out of range\n"); return 1; }
    if (!(ux_mean > 0.0)) { fprintf(stderr, "no flow downstream\n"); return 1; }
    if (!(fx > 0.0)) { fprintf(stderr, "the flow should push the cylinder downstream\n"); return 1; }

    /* The same cylinder as the surface of a "volume mesh" of 2 * nseg
     * vertices (surface vertex i is volume vertex 2 i + 1; the even ones are
     * interior and never reach the fluid), stepped with the coupled entry
     * point: gather, fluid step and force scatter on one stream. */
    float hvv[4 * 48], hvu[4 * 48] = {0};
    unsigned int hmap[48];
    for (int i = 0; i < nseg; ++i) {
        hmap[i] = (unsigned)(2 * i + 1);
        hvv[4 * i] = hvv[4 * i + 1] = 1.0e3f; /* interior vertex far outside the grid */
        hvv[4 * i + 2] = hv[2 * i];
        hvv[4 * i + 3] = hv[2 * i + 1];
    }
    float *dvv, *dvu, *dvf, *dsp, *dsu;
    unsigned int *dmap;
    if (cudaMalloc((void **)&dvv, sizeof hvv) || cudaMalloc((void **)&dvu, sizeof hvu) ||
        cudaMalloc((void **)&dvf, sizeof hvv) || cudaMalloc((void **)&dsp, sizeof hv) ||
        cudaMalloc((void **)&dsu, sizeof hv) || cudaMalloc((void **)&dmap, sizeof hmap)) {
        fprintf(stderr, "cudaMalloc failed\n");
        return 1;
    }
    cudaMemcpy(dvv, hvv, sizeof hvv, cudaMemcpyHostToDevice);
    cudaMemcpy(dvu, hvu, sizeof hvu, cudaMemcpyHostToDevice);
    cudaMemcpy(dmap, hmap, sizeof hmap, cudaMemcpyHostToDevice);
    ffs_volume_surface vs = {0};
    vs.dim = 2;
    vs.num_volume_vertices = 2 * nseg;
    vs.volume_positions = dvv;
    vs.volume_velocities = dvu;
    vs.volume_forces = dvf;
    vs.num_vertices = nseg;
    vs.num_elements = nseg;
    vs.surface_to_volume = dmap;
    vs.elements = de;
    vs.surface_positions = dsp;
    vs.surface_velocities = dsu;
    for (int t = 0; t < 4; ++t) CHECK(ffs_lbm_step_coupled(g, &vs, NULL));
    CHECK(ffs_lbm_get_status(g, &status, 1, NULL));
    if (status) { fprintf(stderr, "device status %u after coupled steps\n", status); return 1; }
    float hvf[4 * 48], hsp[2 * 48];
    cudaMemcpy(hvf, dvf, sizeof hvf, cudaMemcpyDeviceToHost);
    cudaMemcpy(hsp, dsp, sizeof hsp, cudaMemcpyDeviceToHost);
    double vfx = 0.0;
    for (int i = 0; i < nseg; ++i) {
        if (hvf[4 * i] != 0.0f || hvf[4 * i + 1] != 0.0f) { fprintf(stderr, "force on an interior vertex\n"); return 1; }
        if (hsp[2 * i] != hv[2 * i] || hsp[2 * i + 1] != hv[2 * i + 1]) { fprintf(stderr, "gather mismatch\n"); return 1; }
        vfx += hvf[4 * i + 2];
    }
    printf("coupled step: drag on the volume mesh %.6g\n", vfx);
    if (!(vfx > 0.0)) { fprintf(stderr, "no drag scattered to the volume mesh\n"); return 1; }
    cudaFree(dvv); cudaFree(dvu); cudaFree(dvf); cudaFree(dsp); cudaFree(dsu); cudaFree(dmap);

    CHECK(ffs_lbm_destroy(g));
    cudaFree(dv); cudaFree(du); cudaFree(de); cudaFree(dfrc);
    free(flags);
    free(m);
    printf("c abi smoke ok\n");
    return 0;
}
