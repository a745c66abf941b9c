// Device-side tables of the serving pool (include/ffs_pool.h) and the
// launchers of its batched kernels (ffs_batch2d.cu).
#pragma once
#include "ffs_common.cuh"
#include "ffs_links.cuh"

namespace fflbm {

constexpr int kPoolMaxSlots = 1000;          // cell keys: slot * 2^22 + cell + 1 < 2^32
constexpr uint32_t kPoolCellStride = 1u << 22; // cells per episode at most
constexpr int kPoolMaxActions = 16;
constexpr int kPoolMaxSubsteps = 64;

// One admitted episode, as the batched kernels see it.  Every pointer lies
// in the pool's arena.
struct PoolEpisode {
    int nx, ny;
    uint32_t ncell;
    uint32_t cell_base;   // slot * kPoolCellStride: key base in the pool link table
    float omega;          // LBM relaxation rate
    float cl, ct;         // dx, dt
    double cf;            // force scale rho_f dx^2 dx / dt^2
    Codec codec;
    void *mom[2];         // moment buffers A and B (SoA planes)
    uint8_t *flags;       // padded to a multiple of 4 bytes
    uint32_t *wallmask;
    uint32_t *status;
    int nv, ne;
    const float *rest, *amp, *sin_kx, *cos_kx;
    const int32_t *segment;
    const uint32_t *elements;
    float *V, *U;         // surface of the current substep
    long long *acc;       // fixed-point force sums of one substep
    double *force;        // (nv, 2) forces of the last substep
    double *sums;         // [energy, fx, fy, torque] over the control step
    float wave_omega;     // swimmer angular frequency (float)
    float cx0, cy0;       // torque centre: rest centroid
};

// Per active episode (in active-table order), per control step: the action
// and the sin/cos of omega t of each substep, computed on the host in double
// and rounded to float.
struct PoolParams {
    float actions[kPoolMaxActions];
    float sb[kPoolMaxSubsteps];
    float cb[kPoolMaxSubsteps];
};

// The admitted episodes in admission order with prefix sums of their dense
// tiles, elements and vertices.  Kernels read the count from device memory,
// so one captured graph serves every mix.
struct PoolActive {
    uint32_t n;
    uint32_t pad[3];
    uint32_t slot[kPoolMaxSlots];
    uint32_t tiles_x[kPoolMaxSlots];
    uint32_t tile_prefix[kPoolMaxSlots + 1];
    uint32_t elem_prefix[kPoolMaxSlots + 1];
    uint32_t vert_prefix[kPoolMaxSlots + 1];
};

// Output record of one slot (layout of ffs_pool_output).
struct PoolOutput {
    double energy;
    double force[2];
    double torque;
    uint32_t status;
    uint32_t pad;
};

// Travelling-wave swimmer vertex: the same IEEE single operations on the
// host and on the device (no contraction), so a single-grid run can be fed
// exactly the surface the pool computes.
#ifdef __CUDA_ARCH__
#define FFS_MUL(a, b) __fmul_rn((a), (b))
#define FFS_ADD(a, b) __fadd_rn((a), (b))
#define FFS_SUB(a, b) __fsub_rn((a), (b))
#else
#define FFS_MUL(a, b) ((float)((float)(a) * (float)(b)))
#define FFS_ADD(a, b) ((float)((float)(a) + (float)(b)))
#define FFS_SUB(a, b) ((float)((float)(a) - (float)(b)))
#endif
__host__ __device__ inline void swimmer_vertex(float rx, float ry, float amp, float sk, float ck, int seg,
                                               const float *actions, float sb, float cb, float wave_omega,
                                               float &x, float &y, float &vx, float &vy)
{
    const float a = seg >= 0 ? actions[seg] : 0.0f;
    const float A = FFS_MUL(amp, FFS_ADD(1.0f, FFS_MUL(0.5f, a)));
    const float sn = FFS_SUB(FFS_MUL(sk, cb), FFS_MUL(ck, sb)); // sin(k x - omega t)
    const float cs = FFS_ADD(FFS_MUL(ck, cb), FFS_MUL(sk, sb)); // cos(k x - omega t)
    x = rx;
    y = FFS_ADD(ry, FFS_MUL(A, sn));
    vx = 0.0f;
    vy = -FFS_MUL(FFS_MUL(A, wave_omega), cs);
}
#undef FFS_MUL
#undef FFS_ADD
#undef FFS_SUB

// Work units of the batched dense pass (the autotuner's candidates): tiles
// of tx x ty cells, one thread per cell (pool_dense_kernel), or strips of tx
// columns and ty rows walked row by row by tx + 2 threads (pool_strip_kernel).
struct PoolTileShape {
    int tx, ty;
    bool strip;
};
constexpr int kPoolNumShapes = 8;
constexpr PoolTileShape kPoolShapes[kPoolNumShapes] = {{32, 4, false},  {32, 8, false},  {64, 4, false},
                                                       {32, 16, false}, {64, 8, false},  {62, 32, true},
                                                       {126, 32, true}, {126, 64, true}};

cudaError_t launch_pool_kinematics(const PoolEpisode *eps, const PoolParams *prm, const PoolActive *act, int substep,
                                   int grid, cudaStream_t st);
template <typename T>
cudaError_t launch_pool_detect(const PoolEpisode *eps, const PoolActive *act, const LinkTable &lt, uint32_t *owner,
                               int parity, int grid, cudaStream_t st);
template <typename T>
cudaError_t launch_pool_dense(const PoolEpisode *eps, const PoolActive *act, int parity, int shape, int grid,
                              cudaStream_t st);
template <typename T>
int pool_dense_blocks_per_sm(int shape);
template <typename T>
int pool_link_cells_blocks_per_sm();
template <typename T>
cudaError_t launch_pool_link_cells(const PoolEpisode *eps, const LinkTable &lt, const uint32_t *owner, int parity,
                                   int grid, cudaStream_t st);
cudaError_t launch_pool_finalize(const PoolEpisode *eps, const PoolActive *act, const LinkTable &lt, int grid,
                                 cudaStream_t st);
cudaError_t launch_pool_outputs(const PoolEpisode *eps, const PoolActive *act, PoolOutput *out, int substeps,
                                cudaStream_t st);

} // namespace fflbm
