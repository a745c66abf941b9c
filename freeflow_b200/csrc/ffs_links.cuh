// Moving-boundary links: detection, the sparse update of cells that own
// links, and the per-vertex force reduction.
#pragma once
#include "ffs_common.cuh"

namespace fflbm {

// Sparse link table, rebuilt every step.  A cell that owns at least one link
// gets one open-addressing slot: keys[slot] = cell + 1 and links[slot * Q + l]
// = the smallest (depth, element) key of direction l (~0 if none).  `list`
// holds the occupied slots in claim order; `count` their number.  The sparse
// kernel returns every slot it visits to the empty state, so the table is
// clean again at the end of the step without touching unused slots.
struct LinkTable {
    uint32_t cap = 0;                  // power of two (0: not allocated)
    uint32_t *keys = nullptr;          // [cap]
    unsigned long long *links = nullptr; // [cap * Q]
    uint32_t *list = nullptr;          // [cap]
    uint32_t *count = nullptr;         // [1]
    long long *acc = nullptr;          // [acc_cap * DIM] fixed-point force sums (2^-32 units)
    uint32_t acc_cap = 0;              // vertices
    uint32_t *done = nullptr;          // [1] CTAs of link_cells_kernel that finished (zero between steps)
};

// Surfaces of at most this many force components have their fixed-point
// sums converted by the last CTA of link_cells_kernel instead of a kernel of
// their own: one launch less per step where launches dominate (the 2D
// configurations), one CTA's work where that is cheap.
constexpr long long kFoldForcesMax = 2048;

struct SurfaceArgs {
    const float *V;
    const float *U;
    const uint32_t *E;
    int nv, ne;
    float *forces;
    double *forces64;
    // coupled step: the surface is the boundary of a volume mesh; the step's
    // forces are written to vforces[map[i]] (nvol volume vertices) instead
    const uint32_t *map = nullptr;
    float *vforces = nullptr;
    int nvol = 0;
};

struct StepScalars {
    float cl;       // lattice spacing (physical)
    float ct;       // time step (physical)
    double cf;      // force scale rho_f dx^DIM dx / dt^2
};

// fixed-point scale of the per-vertex force sums
constexpr double kForceScale = 4294967296.0; // 2^32

template <int DIM, typename T>
cudaError_t launch_detect_links(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt, const SurfaceArgs &s,
                                const StepScalars &sc, cudaStream_t st);
// With fold_forces, the last CTA also does launch_finalize_forces's work
// (the caller launches no finalize kernel); lt.done must be allocated.
template <int DIM, typename T>
cudaError_t launch_link_cells(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt, const SurfaceArgs &s,
                              const StepScalars &sc, cudaStream_t st, bool fold_forces = false);
template <int DIM>
cudaError_t launch_finalize_forces(const LinkTable &lt, const SurfaceArgs &s, double cf, cudaStream_t st);
template <int DIM>
cudaError_t launch_reset_links(const LinkTable &lt, uint32_t *flag_words, cudaStream_t st);
// first stage of the coupled step: gathers the surface from the volume
// arrays through the map and zeroes the volume forces
cudaError_t launch_gather_surface(int dim, const float *vpos, const float *vvel, const uint32_t *map, int nv, int nvol,
                                  float *spos, float *svel, float *vforces, uint32_t *status, cudaStream_t st);

template <int DIM>
cudaError_t launch_prepare_flags(uint8_t *flags, uint32_t *wallmask, int nx, int ny, int nz, cudaStream_t st);
template <int DIM, typename T>
cudaError_t launch_initialize(const GridArgs<T> &g, T *other, const float *bcvel, cudaStream_t st);
cudaError_t launch_fill_solid2(uint8_t *flags, int nx, int ny, float cl, const SurfaceArgs &s, cudaStream_t st);
// bits: ny * nz * ceil(nx / 32) words, zero on entry and on return
cudaError_t launch_fill_solid3(uint8_t *flags, uint32_t *bits, int nx, int ny, int nz, float cl, const SurfaceArgs &s,
                               cudaStream_t st);

template <int DIM, typename T>
cudaError_t launch_convert_in(const float *in, bool aos, T *out, uint32_t ncell, Codec c, cudaStream_t st);
template <int DIM, typename T>
cudaError_t launch_convert_out(const T *in, float *out, bool aos, uint32_t ncell, Codec c, cudaStream_t st);

} // namespace fflbm
