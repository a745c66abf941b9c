/*
 * ffs_pool.h -- C ABI of the batched serving path: many independent D2Q9
 * swimmer episodes of uneven grid sizes advanced together on one GPU.
 *
 * FreeFlow serves reinforcement learning by running one Simulator2D per
 * environment process (rl/env.py:163-217): every control step applies an
 * action, advances `itrnum_per_step` fluid steps (Simulator2D::step,
 * src/core/Simulator2D.cpp:100 -> fsi_coupling::solveLbmAndFsiStep2D,
 * src/core/FsiCoupling2D.cu:358-432), downloads the surface forces and
 * velocities after each of them, accumulates the swimming energy
 * (power = sum -F.v, added when positive) and checks for divergence.
 *
 * A pool keeps every admitted episode's state on the device and advances all
 * of them by one control step with one CUDA-graph launch: per substep the
 * swimmer kinematics, link detection, the fused stream/collide pass (one
 * persistent launch over a packed list of tiles of all grids), the moving-
 * wall link cells and the force reduction run once for the whole pool.
 * Outputs per control step (energy, mean force and torque, per-vertex
 * forces of the last substep, status) are reduced on the device.
 *
 * Memory: the pool reserves `budget_bytes` of device memory once, at
 * creation; episodes are admitted into it while their state fits
 * (ffs_pool_admit returns FFS_ERR_CAPACITY otherwise) and evicted to make
 * room.  Admission and eviction never allocate device memory.
 *
 * All device work of a pool runs on the pool's stream, in call order; the
 * host calls are not thread-safe for one pool.  No call traps on the device.
 *
 * This interface has no counterpart in the reference (which has no batched
 * path); its episode semantics follow rl/env.py:163-217 as cited above.
 */
#ifndef FFS_POOL_H
#define FFS_POOL_H

#include <stdint.h>

#include "ffs_lbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ffs_pool ffs_pool;

#define FFS_POOL_MAX_ACTIONS 16
#define FFS_POOL_MAX_SUBSTEPS 64

typedef struct {
    int storage;            /* ffs_storage of every episode's moments (F16 for serving) */
    int64_t budget_bytes;   /* device memory reserved for episode state */
    int max_episodes;       /* admitted at once */
    int substeps;           /* fluid steps per control step (rl/env.py itrnum_per_step), <= 64 */
    int num_actions;        /* actuator values per control step, <= 16 */
    int max_link_cells;     /* link-table capacity over all episodes (0: 2048 per episode) */
    void *stream;           /* cudaStream_t for all pool work; NULL: the pool creates its own */
} ffs_pool_desc;

/* A prescribed travelling-wave swimmer (the kinematic solid): vertex v moves
 * laterally by A_v sin(k x_v - omega t) about its rest position, with
 * A_v = amplitude[v] * (1 + 0.5 a[segment[v]]) for the current action a.
 * sin_kx / cos_kx hold sin(k x_v) and cos(k x_v).  Substep q of the episode
 * is at time t0 + q dt.  All arrays are host memory, copied at admission. */
typedef struct {
    int num_vertices;
    int num_elements;
    const float *rest;         /* (nv, 2) physical rest positions */
    const uint32_t *elements;  /* (ne, 2) boundary segments */
    const float *amplitude;    /* (nv) physical lateral amplitude */
    const float *sin_kx;       /* (nv) */
    const float *cos_kx;       /* (nv) */
    const int32_t *segment;    /* (nv) action index, or -1 for a vertex the actions do not scale */
    double omega;              /* angular frequency of the body wave, rad per time unit */
    double t0;                 /* time of substep 0 */
} ffs_swimmer;

typedef struct {
    ffs_lbm_desc grid;         /* dim must be 2; storage and periodic_mask are taken from the pool */
    const uint8_t *flags;      /* host, nx * ny LbmNodeFlag values, x fastest */
    ffs_swimmer swimmer;
} ffs_episode_desc;

typedef struct {
    double energy;             /* sum over substeps of max(0, sum_v -F_v . U_v) dt (rl/env.py:172-175) */
    double force[2];           /* mean total fluid force over the substeps */
    double torque;             /* mean torque about the rest centroid */
    uint32_t status;           /* ffs_lbm_get_status bits latched during the control step */
    uint32_t pad;
} ffs_pool_output;

typedef struct {
    int64_t budget_bytes, free_bytes, largest_free_bytes;
    int active_episodes;
    int tiles;                 /* dense tiles per substep over all episodes */
    int tile_x, tile_y;        /* tile shape in use (chosen by ffs_pool_tune) */
    int64_t advances;          /* control steps launched */
    int64_t graph_builds;      /* CUDA graphs instantiated */
    int64_t cells;             /* fluid cells over all admitted episodes */
    int64_t tuned_cells;       /* fluid cells of the mix at the last tuning */
    double dense_ms;           /* one dense pass over that mix (CUDA events, mean of 5) */
    int strip;                 /* 1: the dense unit is a strip of tile_x columns and tile_y
                                  rows walked row by row; 0: a tile_x x tile_y tile */
    int pad;
} ffs_pool_info;

ffs_status ffs_pool_create(const ffs_pool_desc *desc, ffs_pool **out);
ffs_status ffs_pool_destroy(ffs_pool *pool);

/* Device bytes an episode would take in this pool (admission arithmetic). */
ffs_status ffs_pool_episode_bytes(const ffs_pool *pool, const ffs_episode_desc *ep, int64_t *bytes);

/* Copies the episode in, initialises its fluid to rest (LbmInitializer2D),
 * and returns its slot.  FFS_ERR_CAPACITY: no free slot or not enough free
 * memory in the budget (nothing changed; retry after an eviction). */
ffs_status ffs_pool_admit(ffs_pool *pool, const ffs_episode_desc *ep, int *slot);

/* Frees the slot and its memory; takes effect for the next control step. */
ffs_status ffs_pool_evict(ffs_pool *pool, int slot);

/* Action of the slot's next control step (rl/env.py process_action); the
 * previous action is kept until replaced.  n <= num_actions. */
ffs_status ffs_pool_set_action(ffs_pool *pool, int slot, const float *actions, int n);

/* ffs_pool_set_action for n slots in one call: actions holds n rows of
 * num_actions values.  Nothing changes if a slot is invalid. */
ffs_status ffs_pool_set_actions(ffs_pool *pool, int n, const int *slots, const float *actions);

/* Launches one control step of every admitted episode; returns without
 * waiting.  The first call after the mix changed re-uploads the tile table;
 * the first call (and ffs_pool_tune) builds the CUDA graph.  The pinned
 * parameter and output buffers are double-buffered, so the call does not
 * wait for the previous control step: it waits only while the step before
 * that still holds the buffer it refills.  A caller may therefore enqueue
 * the next control step before collecting the previous one (with actions
 * that do not depend on its outputs); collect then returns the newer. */
ffs_status ffs_pool_advance(ffs_pool *pool);

/* Waits for the latest control step and returns the slot's outputs.
 * forces (optional): the slot's per-vertex fluid forces of the last
 * substep, (nv, 2) doubles. */
ffs_status ffs_pool_collect(ffs_pool *pool, int slot, ffs_pool_output *out, double *forces);

/* ffs_pool_collect of n slots' output records in one call (waits once). */
ffs_status ffs_pool_collect_many(ffs_pool *pool, int n, const int *slots, ffs_pool_output *out);

/* Current moments of the slot in the reference AoS layout (nx*ny*6 floats,
 * host memory); synchronous.  For tests and inspection. */
ffs_status ffs_pool_get_moments(ffs_pool *pool, int slot, float *moments);

/* Times the candidate tile shapes of the dense pass on the current mix and
 * keeps the fastest (a project autotuner; rebuilds the graph). */
ffs_status ffs_pool_tune(ffs_pool *pool);

ffs_status ffs_pool_get_info(const ffs_pool *pool, ffs_pool_info *info);

/* The swimmer's surface at substep q under `actions`, computed on the host
 * with the same IEEE operations as the pool's device kinematics (so a
 * single-grid run can be fed exactly the same surface). */
ffs_status ffs_swimmer_surface(const ffs_swimmer *sw, const float *actions, int num_actions, int64_t q, double dt,
                               float *vertices, float *velocities);

#ifdef __cplusplus
}
#endif

#endif /* FFS_POOL_H */
