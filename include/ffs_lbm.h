/*
 * ffs_lbm.h -- C ABI of the B200 moment-encoded lattice-Boltzmann fluid step.
 *
 * One `ffs_lbm` object is one fluid grid (D2Q9 or D3Q27) resident in device
 * memory, the equivalent of FreeFlow's LbmFlowField2D / LbmFlowField3D plus
 * the step that advances it.  Every entry point takes plain pointers, sizes
 * and a CUDA stream passed as `void *` (a cudaStream_t; NULL = legacy default
 * stream).  Nothing in this header depends on CUDA, C++ or torch headers.
 *
 * Errors: every call returns an ffs_status; nothing throws across the ABI and
 * no device code traps.  Device-side anomalies (non-finite density, link
 * table overflow, force range) are latched in a status word read with
 * ffs_lbm_get_status().  ffs_last_error() describes the last failed call on
 * the calling thread.
 *
 * Each entry point cites, beside its declaration, the FreeFlow interface it
 * replaces (paths relative to that repository).
 */
#ifndef FFS_LBM_H
#define FFS_LBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFS_ABI_VERSION 4

typedef struct ffs_lbm ffs_lbm;

typedef enum {
    FFS_OK = 0,
    FFS_ERR_INVALID_ARGUMENT = 1,
    FFS_ERR_OUT_OF_MEMORY = 2,
    FFS_ERR_CUDA = 3,
    FFS_ERR_CAPACITY = 4,
    FFS_ERR_UNSUPPORTED = 5
} ffs_status;

typedef enum { FFS_STORAGE_F32 = 0, FFS_STORAGE_F16 = 1, FFS_STORAGE_BF16 = 2 } ffs_storage;

/* Moment array layout for get/set.  AOS is the reference's layout
 * (LbmFlowField2D.cpp:29, LbmFlowField3D.cpp:81): NM floats per cell, x
 * fastest, in the order [rho, ux, uy, pixx, piyy, pixy] (D2Q9) or
 * [rho, ux, uy, uz, pixx, piyy, pizz, pixy, piyz, pixz] (D3Q27), where
 * pi_aa = Pi_aa / rho - 1/3 and pi_ab = Pi_ab / rho.  SOA is the same values
 * as NM planes of ncell floats. */
typedef enum { FFS_LAYOUT_AOS = 0, FFS_LAYOUT_SOA = 1 } ffs_layout;
typedef enum { FFS_MEM_HOST = 0, FFS_MEM_DEVICE = 1 } ffs_memory;

/* Which moment buffer a get/set addresses.  The grid ping-pongs between
 * buffer A and buffer B like the reference's m_current_moments /
 * m_next_moments (LbmFlowField2D.hpp:168-171). */
typedef enum {
    FFS_BUF_CURRENT = 0,
    FFS_BUF_NEXT = 1,
    FFS_BUF_A = 2, /* the reference's m_fMom / m_moments_pre */
    FFS_BUF_B = 3,
    FFS_BUF_BOTH = 4 /* set only */
} ffs_buffer;

/* Fluid parameters; field names follow SimulationParameters2D/3D
 * (include/FSI_Simulator/utils/Config.hpp:64-159). */
typedef struct {
    int dim;                       /* 2 (D2Q9) or 3 (D3Q27) */
    int nx, ny, nz;                /* nz ignored for dim == 2 */
    double fluid_viscosity;        /* lattice kinematic viscosity: omega = 1/(3 nu + 1/2) */
    double fluid_density;          /* used only for the force scale Cf */
    double fluid_dx;               /* lattice spacing (surface coordinates are physical) */
    double dt;
    float boundary_velocities[6];  /* [vx_left, vy_down, vx_right, vy_up(, v_front, v_back)] */
    int storage;                   /* ffs_storage */
    int periodic_mask;             /* bit0 x, bit1 y, bit2 z: wrap the streaming halo at
                                      both faces.  0 = the reference's halo, which
                                      wraps at the low face and clamps at the high
                                      face of each axis (FsiCoupling2D.cu:104-105,
                                      FsiCoupling3D.cu:106-108: unsigned index
                                      arithmetic); the bounce-back test always uses
                                      the wrapped neighbour (:163-176, :200-216) */
    int ref_half_populations;      /* D2Q9 only: round reconstructed populations to
                                      binary16 as the reference's __half tile does
                                      (FsiCoupling2D.cu:89,120-128) */
    int ref_2d_wall_stream;        /* D2Q9 only: 1 = walls stream their stored moments
                                      as in the reference's 2D kernel, which computes
                                      the bounce-back value and then overwrites it with
                                      the ordinary pull (FsiCoupling2D.cu:171-224:
                                      is_blocked is set only on the moving-wall path);
                                      0 = bounce-back, as the 3D kernel does */
} ffs_lbm_desc;

/* Surface seen by the fluid step; mirrors SolidGeometryProxy_Device<DIM>
 * (include/FSI_Simulator/core/SolidGeometryProxy_Device.cuh:30-73).  All
 * pointers are DEVICE pointers.  vertices/velocities are DIM floats per
 * vertex (physical units), elements are DIM vertex indices per element
 * (segments in 2D, triangles in 3D).  forces (DIM floats per vertex) is an
 * accumulator: the step ADDS the fluid force (physical units, scaled by
 * Cf = rho_f dx^DIM dx / dt^2) and never clears it, like the reference.
 * forces64, if not NULL, receives the same sum in double. */
typedef struct {
    int dim;
    const float *vertices;
    const float *velocities;
    const uint32_t *elements;
    int num_vertices;
    int num_elements;
    float *forces;
    double *forces64;
} ffs_surface;

/* A surface given as the boundary of a solid's volume mesh: the solid's own
 * vertex arrays plus the surface-to-volume vertex map, as
 * FsiCouplingDataGpu holds them (include/FSI_Simulator/fsi/
 * FsiCouplingDataGpu.cuh:18-30).  All pointers are DEVICE pointers;
 * positions, velocities and forces are DIM floats per vertex.
 *   volume_positions/velocities  the solid's vertices (physical units)
 *   volume_forces                output, see ffs_lbm_step_coupled
 *   surface_to_volume[i]         volume index of surface vertex i
 *   elements                     DIM surface-vertex indices per element
 *   surface_positions/velocities caller-owned arrays of num_vertices
 *                                entries (FsiCouplingDataGpu::
 *                                surface_positions/velocities); the step
 *                                writes the gathered surface there. */
typedef struct {
    int dim;
    int num_volume_vertices;
    const float *volume_positions;
    const float *volume_velocities;
    float *volume_forces;
    int num_vertices;
    int num_elements;
    const uint32_t *surface_to_volume;
    const uint32_t *elements;
    float *surface_positions;
    float *surface_velocities;
} ffs_volume_surface;

/* Replaces the LbmFlowField2D/3D constructors (LbmFlowField2D.cpp:17-40,
 * LbmFlowField3D.cpp:18-41).  All cells start as Fluid with zero moments;
 * call ffs_lbm_set_flags + ffs_lbm_initialize next. */
ffs_status ffs_lbm_create(const ffs_lbm_desc *desc, ffs_lbm **out);

/* Frees every device allocation of the grid (RAII CudaArray destructors). */
ffs_status ffs_lbm_destroy(ffs_lbm *grid);

/* Uploads LbmNodeFlag values, one byte per cell, x fastest (the array
 * LbmInitializer::initializeState2D/3D builds from the JSON boundaries,
 * LbmInitializer2D.cu:103-124).  Recomputes the derived per-cell data the
 * kernels use (bounce-back masks, outlet feeders). */
ffs_status ffs_lbm_set_flags(ffs_lbm *grid, const uint8_t *flags, int memory, void *stream);
ffs_status ffs_lbm_get_flags(ffs_lbm *grid, uint8_t *flags, int memory, void *stream);

/* initialize_state_kernel_2d/3d + LbmFlowField*::reset
 * (LbmInitializer2D.cu:32-95, LbmInitializer3D.cu:33-113): equilibrium
 * moments with rho = 1 and the inlet velocity on inlet nodes, written to both
 * buffers; buffer A becomes current. */
ffs_status ffs_lbm_initialize(ffs_lbm *grid, void *stream);

/* Moment transfer (Simulator2D::getFluidMoment, Simulator2D.hpp:41-43;
 * Simulator3D.hpp:37-39; bindings.cpp:259-266,309-315).  `layout` is
 * ffs_layout, `memory` ffs_memory, `which` ffs_buffer.  Values are always
 * FP32 at the interface, whatever the storage precision.  Host transfers are
 * synchronous; device transfers are ordered on `stream`. */
ffs_status ffs_lbm_set_moments(ffs_lbm *grid, const float *moments, int layout, int memory, int which, void *stream);
ffs_status ffs_lbm_get_moments(ffs_lbm *grid, float *moments, int layout, int memory, int which, void *stream);

/* Pre-allocates the moving-boundary scratch (link table for up to
 * max_link_cells boundary cells, force accumulators for up to max_vertices
 * vertices) so that steps never allocate.  Optional: the first step with a
 * larger surface allocates on demand. */
ffs_status ffs_lbm_reserve_surface(ffs_lbm *grid, int max_vertices, int max_link_cells);

/* One fluid step: fsi_coupling::solveLbmAndFsiStep2D / solveLbmAndFsiStep3D
 * (src/core/FsiCoupling2D.cu:358-432, src/core/FsiCoupling3D.cu:424-484):
 * moving-boundary link detection, the fused stream-reconstruct-collide-
 * re-encode pass, bounce-back, moving-wall links with surface forces, the
 * outlet update, and the buffer swap.  `surface` may be NULL (no solid).
 * Asynchronous on `stream`; no host synchronisation. */
ffs_status ffs_lbm_step(ffs_lbm *grid, const ffs_surface *surface, void *stream);

/* One coupled fluid step as Simulator2D/3D::step runs it (src/core/
 * Simulator2D.cpp:93-107, Simulator3D.cpp:90-101), in one stream and with no
 * host synchronisation:
 *   1. the surface gather of FemScene2D/3D::getSurfaceProxyForFSI
 *      (src/fem/FemScene.cpp:591-605, 1251-1264; updateSurfaceStatesFromVolume,
 *      src/fsi/FsiCouplingKernels.cu:14-57, 93-131): surface_positions/
 *      velocities[i] = volume_positions/velocities[surface_to_volume[i]];
 *   2. the fluid step of ffs_lbm_step on that surface;
 *   3. the solid solver's applyForces (src/fem/VBDSolver.cpp:101-113,
 *      282-297; scatterSurfaceForcesToVolume, FsiCouplingKernels.cu:59-90,
 *      133-178): volume_forces is zeroed, then holds this step's fluid force
 *      (Cf-scaled, physical units) at every mapped volume vertex.
 * The reference synchronises after the gather (on stream 0) and after the
 * scatter; here the three stages are kernels on `stream` and the call can be
 * captured in a CUDA graph (every pointer is read at launch).  A map entry
 * >= num_volume_vertices latches status bit 8 and that vertex is skipped. */
ffs_status ffs_lbm_step_coupled(ffs_lbm *grid, const ffs_volume_surface *surface, void *stream);

/* No counterpart in the reference.  The same step as ffs_lbm_step, with the
 * same results, but it allocates no device memory: its link table and force
 * accumulators live in one fixed array inside this library (8,126,720 bytes
 * per device), for callers that must not allocate while stepping (a fixed,
 * pre-reserved device-memory budget; loops that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree).
 * Limits: at most FFS_NOALLOC_MAX_VERTICES surface vertices (larger surfaces
 * return FFS_ERR_CAPACITY before any work).  FFS_NOALLOC_MAX_LINK_CELLS cells
 * may own links in one step with the table at most half full; past that the
 * step still runs but detection slows as the table fills, and at twice that
 * number the table is full and the step latches status bit 2 (link table
 * overflow, as ffs_lbm_step does with a too-small reservation).
 * The first call on a device looks the array up on that device (set-up): make
 * it before any stream capture.  The address is kept for the process; after
 * a cudaDeviceReset of that device this entry point must not be called again.
 * Every call on a device shares the array and clears it on `stream` first, so
 * calls that overlap in time on one device race: the caller orders them (one
 * stream, or events).  Link detection runs beside the dense pass on the
 * grid's side stream, as in ffs_lbm_step; stage timing
 * (ffs_lbm_profile_enable) records nothing for these steps. */
#define FFS_NOALLOC_MAX_VERTICES 32768
#define FFS_NOALLOC_MAX_LINK_CELLS 16384
ffs_status ffs_lbm_step_noalloc(ffs_lbm *grid, const ffs_surface *surface, void *stream);

/* fsi_coupling::fillSolidFlags2D (FsiCoupling2D.cu:434-464): Fluid cells
 * whose centre lies inside the closed polygon become SolidDynamic, and
 * SolidDynamic cells outside it return to Fluid.  On a D3Q27 grid the same
 * for a closed triangle mesh, by the parity of the triangles that a ray from
 * the cell centre along +x crosses: the 3D inside test of the reference
 * (SolidGeometryProxy_Device<3>::isInside, SolidGeometryProxy_Device.cuh:
 * 231-289, which has no fill of its own), evaluated row by row.  Elements
 * with a vertex index out of range are skipped. */
ffs_status ffs_lbm_fill_solid(ffs_lbm *grid, const ffs_surface *surface, void *stream);

/* Reads (and optionally clears) the device status word; synchronises
 * `stream`.  Bits: 1 a fluid update produced a non-positive or non-finite
 * density or a non-finite velocity, 2 link table overflow, 4 force out of
 * fixed-point range, 8 element index out of range, 16 a staged plane of
 * moments did not reach shared memory within the dense pass's wait limit
 * (the step's results are invalid; not expected to happen). */
ffs_status ffs_lbm_get_status(ffs_lbm *grid, uint32_t *status, int clear, void *stream);

/* Grid facts: cell count, moments per cell, directions, omega, Cf. */
ffs_status ffs_lbm_get_info(ffs_lbm *grid, int64_t *ncell, int *nm, int *q, double *omega, double *cf);

/* Diagnostic: runs only the link detection of a step for `surface` and
 * copies the resulting links, sorted by (cell * Q + direction), to host
 * arrays: cell_dir[k] = cell * Q + direction and key[k] =
 * (uint32(depth * 32768) << 32) | element, the reference's depthIndexCompact
 * key widened to 64 bits.  *count receives the number of links (at most
 * capacity are written).  Leaves no state behind. */
ffs_status ffs_lbm_debug_links(ffs_lbm *grid, const ffs_surface *surface, uint64_t *cell_dir, uint64_t *key,
                               int64_t capacity, int64_t *count, void *stream);

/* Per-stage GPU timing, the non-blocking counterpart of the reference's
 * PROFILE_CUDA_SCOPE (include/FSI_Simulator/utils/Profiler.hpp:21-31,
 * src/utils/Profiler.cpp:107-121, which synchronises in every scope).  While
 * enabled, each step records CUDA events around its stages on the step's
 * stream; ffs_lbm_profile_read() waits for the recorded events and returns
 * the summed milliseconds and launch counts per stage:
 * [0] link detection, [1] dense fused update, [2] link cells, [3] forces.
 * For surfaces of at most 2048 force components the force conversion runs in
 * the last CTA of the link-cell kernel, and [3] records no launch.
 * enable: 0 off; 1 on; 2 on with link detection moved from its side stream
 * onto the step's stream ahead of the dense pass, so that every stage is
 * timed alone (a measurement mode: the step is then slower by the overlap it
 * gives up; results are the same). */
typedef struct {
    double ms[4];
    int64_t launches[4];
} ffs_profile;

ffs_status ffs_lbm_profile_enable(ffs_lbm *grid, int enable);
ffs_status ffs_lbm_profile_read(ffs_lbm *grid, ffs_profile *out, int reset);

const char *ffs_status_string(ffs_status status);
const char *ffs_last_error(void);
int ffs_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FFS_LBM_H */
