// Batched D2Q9 kernels of the serving pool: every kernel covers all admitted
// episodes of the pool in one launch.
//
// Work items are numbered across episodes through the prefix sums of the
// active table (dense tiles, surface elements, surface vertices); an item
// finds its episode by a binary search over at most kPoolMaxSlots prefixes.
// The per-item bodies are the single-grid ones (dense2d_tile or the same
// per-cell code in strips, detect_element2_warp, link_cell_update), so a pool
// episode computes bit for bit what the same
// grid computes alone through ffs_lbm_step.  The grids are persistent
// (a fixed number of CTAs striding over a count read from device memory), so
// one captured CUDA graph serves every mix of episodes.
//
// Reference: one Simulator2D per environment process, each step through
// fsi_coupling::solveLbmAndFsiStep2D (src/core/FsiCoupling2D.cu:358-432);
// the environment loop is rl/env.py:163-217.
#include "ffs_links_dev.cuh"
#include "ffs_pool.cuh"

namespace fflbm {

namespace {

// Index of the active entry whose range [prefix[i], prefix[i+1]) holds t.
__device__ __forceinline__ int owner_of(const uint32_t *prefix, int n, uint32_t t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename T> __device__ __forceinline__ GridArgs<T> episode_args(const PoolEpisode &e, int parity)
{
    GridArgs<T> g;
    g.nx = e.nx;
    g.ny = e.ny;
    g.nz = 1;
    g.ncell = e.ncell;
    g.periodic = 0;
    g.half_pops = 0;
    g.wall_stream = 0;
    g.omega = e.omega;
    g.codec = e.codec;
    g.src = static_cast<const T *>(e.mom[parity]);
    g.dst = static_cast<T *>(e.mom[parity ^ 1]);
    g.flags = e.flags;
    g.wallmask = e.wallmask;
    g.status = e.status;
    return g;
}

__device__ __forceinline__ SurfaceArgs episode_surface(const PoolEpisode &e)
{
    SurfaceArgs s{};
    s.V = e.V;
    s.U = e.U;
    s.E = e.elements;
    s.nv = e.nv;
    s.ne = e.ne;
    s.forces = nullptr;
    s.forces64 = nullptr;
    return s;
}

} // namespace

// ------------------------------------------------------------ kinematics
__global__ void pool_kinematics_kernel(const PoolEpisode *eps, const PoolParams *prm, const PoolActive *act,
                                       int substep)
{
    const int n = (int)act->n;
    if (n == 0) return;
    const uint32_t total = act->vert_prefix[n];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int a = owner_of(act->vert_prefix, n, t);
        const uint32_t s = act->slot[a];
        const PoolEpisode &e = eps[s];
        const PoolParams &p = prm[a];
        const uint32_t v = t - act->vert_prefix[a];
        float x, y, vx, vy;
        swimmer_vertex(e.rest[2 * v], e.rest[2 * v + 1], e.amp[v], e.sin_kx[v], e.cos_kx[v], e.segment[v], p.actions,
                       p.sb[substep], p.cb[substep], e.wave_omega, x, y, vx, vy);
        e.V[2 * v] = x;
        e.V[2 * v + 1] = y;
        e.U[2 * v] = vx;
        e.U[2 * v + 1] = vy;
    }
}

// ---------------------------------------------------------------- detect
// One warp per element of any episode (the single-grid body,
// detect_element2_warp); the warp finds the element's episode once.  (Giving
// each warp a contiguous run of elements, so that the episode search runs
// once per run, measured no faster: the time goes to the link insertions'
// dependent atomics, not to the search.)
template <typename T>
__global__ void __launch_bounds__(256) pool_detect_kernel(const PoolEpisode *eps, const PoolActive *act, LinkTable lt,
                                                          uint32_t *owner, int parity)
{
    __shared__ uint32_t queue[8][64]; // per warp: (cell, direction) pairs for the exact test
    const int n = (int)act->n;
    if (n == 0) return;
    const uint32_t total = act->elem_prefix[n];
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t ge = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ge < total; ge += nwarps) {
        const int a = owner_of(act->elem_prefix, n, ge);
        const uint32_t s = act->slot[a];
        const PoolEpisode &e = eps[s];
        const GridArgs<T> g = episode_args<T>(e, parity);
        const SurfaceArgs sa = episode_surface(e);
        const StepScalars sc{e.cl, e.ct, e.cf};
        detect_element2_warp<T>(g, reinterpret_cast<uint32_t *>(e.flags), lt, sa, sc,
                                (long long)(ge - act->elem_prefix[a]), queue[threadIdx.x >> 5], e.cell_base, owner, s);
    }
}

// ----------------------------------------------------------------- dense
// Persistent CTAs stride over the tiles of all episodes in order, so a CTA's
// episode index only grows: it is advanced from the previous tile's instead of
// searched.
template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY) pool_dense_kernel(const PoolEpisode *eps, const PoolActive *act, int parity)
{
    __shared__ float sp[9][TY + 2][TX + 2];
    const int n = (int)act->n;
    if (n == 0) return;
    const uint32_t total = act->tile_prefix[n];
    int a = 0;
    for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
        while (act->tile_prefix[a + 1] <= t) ++a;
        const uint32_t local = t - act->tile_prefix[a];
        const uint32_t tw = act->tiles_x[a];
        const GridArgs<T> g = episode_args<T>(eps[act->slot[a]], parity);
        dense2d_tile<T, false, TX, TY>(g, (int)(local % tw) * TX, (int)(local / tw) * TY, sp);
        __syncthreads(); // the next tile reuses sp
    }
}

// ---------------------------------------------------------- dense (strips)
// Row-marching variant of the dense pass.  A work unit is a strip of TX-2
// columns and CH rows of one episode; a CTA of TX threads walks up its rows:
//   * the stored moments of each row's TX halo cells (columns x0-1 ..
//     x0+TX-2) are staged in shared memory by 16-byte cp.async copies DEPTH
//     rows ahead of use, from a window that starts on a 16-byte bound, so the
//     loads in flight hold no registers (rows whose width is not a multiple
//     of a copy's cells are copied cell by cell instead);
//   * each row is reconstructed once into a ring of four population rows,
//     one halo cell per thread, so every thread does the same work and a
//     unit reconstructs CH+2 rows for CH;
//   * threads 1..TX-2 update row o from ring rows o-1, o, o+1 in the
//     iteration after row o+1 was reconstructed, which leaves one barrier per
//     row.
// The per-cell arithmetic is dense2d_recon / dense2d_update_cell, the same
// code as the tile kernel, so both give the same bits.  Episodes hold fewer
// than 2^22 cells, so every moment index fits in 32 bits.
template <typename T, int TX, int CH, int DEPTH>
__global__ void __launch_bounds__(TX, 1024 / TX) pool_strip_kernel(const PoolEpisode *eps, const PoolActive *act, int parity)
{
    using L = Lattice<2>;
    constexpr int kOut = TX - 2;              // columns a strip updates
    constexpr int kDepth = DEPTH;             // rows staged ahead of use
    constexpr int kStage = kDepth + 1;        // staging slots
    constexpr int kRing = 4;                  // population rows
    constexpr int kPer = 16 / (int)sizeof(T); // cells per 16-byte copy
    constexpr int kSW = TX + kPer;            // staged cells per row, from xs (see below)
    constexpr int kCopies = kSW / kPer;       // 16-byte copies per staged moment row
    static_assert(TX % kPer == 0, "whole copies per staged row");
    __shared__ __align__(16) T stage[kStage][6][kSW];
    __shared__ float ring[kRing][9][TX];

    const int n = (int)act->n;
    if (n == 0) return;
    const int tid = threadIdx.x;
    const uint32_t total = act->tile_prefix[n];
    int a = 0;
    for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
        while (act->tile_prefix[a + 1] <= t) ++a;
        const uint32_t local = t - act->tile_prefix[a];
        const uint32_t tw = act->tiles_x[a];
        const GridArgs<T> g = episode_args<T>(eps[act->slot[a]], parity);
        const int x0 = (int)(local % tw) * kOut;
        const int yb = (int)(local / tw) * CH, ye = min(yb + CH, g.ny);
        const bool wx = g.periodic & 1, wy = g.periodic & 2;
        // staged window: cells xs .. xs+kSW-1, xs the copy bound at or below
        // x0-1 (0 for the first strip), which covers the halo row x0-1 .. x0+TX-2
        const int xs = (max(x0 - 1, 0) / kPer) * kPer;
        // whole copies start on 16-byte bounds when a row holds a multiple of
        // kPer cells (then so does every moment plane; the buffers themselves
        // are 256-byte aligned)
        const bool vec = g.nx % kPer == 0;
        // staging slot of row r (r >= -1): (r + 1) mod kStage, kept as a
        // counter in the row loop below instead of a division per row
        auto slot_of = [](int r) { return (uint32_t)(r + 1) % (uint32_t)kStage; };
        // stage row r (yb-1 <= r <= ye) into slot sl: the cells that lie inside the grid
        auto issue = [&](int r, uint32_t sl) {
            if (r <= ye) {
                T (*st)[kSW] = stage[sl];
                const uint32_t row = (uint32_t)halo_index(r, g.ny, wy) * (uint32_t)g.nx;
                if (vec) {
                    for (int e = tid; e < 6 * kCopies; e += TX) {
                        const int k = e / kCopies, w = e - k * kCopies;
                        const int x = xs + w * kPer;
                        if (x + kPer <= g.nx)
                            cp_async16(&st[k][w * kPer], g.src + ((uint32_t)k * g.ncell + row + (uint32_t)x));
                    }
                } else {
                    for (int e = tid; e < 6 * kSW; e += TX) {
                        const int k = e / kSW, j = e - k * kSW;
                        if (xs + j < g.nx) st[k][j] = g.src[(uint32_t)k * g.ncell + row + (uint32_t)(xs + j)];
                    }
                }
            }
            cp_async_commit();
        };
        // reconstruct this thread's halo cell x0-1+tid of row r into the
        // ring; the clamped or wrapped source column is read from the staged
        // row when it lies there, else (a wrapped edge) from memory
        auto recon = [&](int r, uint32_t sl) {
            const int gx = halo_index(x0 - 1 + tid, g.nx, wx);
            const int j = gx - xs;
            T raw[6];
            if (j >= 0 && j < kSW) {
                const T (*st)[kSW] = stage[sl];
#pragma unroll
                for (int k = 0; k < 6; ++k) raw[k] = st[k][j];
            } else {
                const size_t cell = (size_t)halo_index(r, g.ny, wy) * g.nx + gx;
#pragma unroll
                for (int k = 0; k < 6; ++k) raw[k] = g.src[(size_t)k * g.ncell + cell];
            }
            float f[9];
            dense2d_recon<T, false>(g, raw, f);
            float (*rg)[TX] = ring[(uint32_t)(r + kRing) % kRing];
#pragma unroll
            for (int i = 0; i < 9; ++i) rg[i][tid] = f[i];
        };

#pragma unroll
        for (int r = 0; r < kDepth; ++r) issue(yb - 1 + r, slot_of(yb - 1 + r));
        const int x = x0 - 1 + tid;
        const bool owner = tid >= 1 && tid <= kOut && x < g.nx; // this thread updates column x
        // flag bytes of this thread's cell: at the top of iteration r, f8 is
        // that of row r-2 (updated this iteration) and f8n that of row r-1;
        // row r's is loaded at the end of iteration r, two iterations ahead
        auto flag_at = [&](int y) -> uint32_t {
            return (owner && y >= yb && y < ye) ? (uint32_t)g.flags[(uint32_t)y * (uint32_t)g.nx + (uint32_t)x] : 0u;
        };
        uint32_t f8 = 0, f8n = 0;
        uint32_t sl = slot_of(yb - 1);                  // slot of row r
        uint32_t sl_prev = sl == 0 ? kStage - 1 : sl - 1; // slot of row r-1 = slot of row r + kDepth
        for (int r = yb - 1; r <= ye + 1; ++r) {
            cp_async_wait<kDepth - 1>(); // this thread's copies of row r have landed
            __syncthreads();             // everyone's copies of row r, and ring row r-1, are visible
            issue(r + kDepth, sl_prev);  // into the slot of row r-1, reconstructed last iteration
            if (r <= ye) recon(r, sl);
            sl_prev = sl;
            sl = sl + 1 == kStage ? 0u : sl + 1;
            // output row o: its ring rows o-1, o, o+1 were written before the barrier
            const int o = r - 2;
            if (o >= yb && owner && is_updated(f8 & kTypeMask) && !(f8 & kBitLink)) {
                const uint32_t idx = (uint32_t)(o * g.nx + x);
                dense2d_update_cell<T, true>(
                    g, idx, f8, [&](int i) { return ring[(uint32_t)(o - L::cy(i) + kRing) % kRing][i][tid - L::cx(i)]; },
                    [&](int i) { return ring[(uint32_t)(o + kRing) % kRing][i][tid]; });
            }
            f8 = f8n;
            f8n = flag_at(o + 2);
        }
    }
}

// ------------------------------------------------------------ link cells
template <typename T>
__global__ void __launch_bounds__(256, 4) pool_link_cells_kernel(const PoolEpisode *eps, LinkTable lt,
                                                                 const uint32_t *owner, int parity)
{
    constexpr int Q = 9, G = kLinkGroup<2>, kPerWarp = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const uint32_t group = (threadIdx.x & 31) / G;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = *lt.count;
    for (uint32_t w = (((blockIdx.x * blockDim.x) + threadIdx.x) >> 5) * kPerWarp; w < n; w += nwarps * kPerWarp) {
        // two cells per warp, possibly of different episodes; a group past the
        // end of the list rides along on the first group's cell
        const bool valid = w + group < n;
        const uint32_t slot = lt.list[valid ? w + group : w];
        const PoolEpisode &e = eps[owner[slot]];
        const uint32_t cell = lt.keys[slot] - 1 - e.cell_base;
        const GridArgs<T> g = episode_args<T>(e, parity);
        const SurfaceArgs sa = episode_surface(e);
        const StepScalars sc{e.cl, e.ct, e.cf};
        link_cell_update<2, T, false>(g, lt.links, slot, cell, e.acc, sa, sc, valid);
        if (valid && lane < Q) lt.links[(size_t)slot * Q + lane] = ~0ull;
        __syncwarp();
        if (valid && lane == 0) {
            lt.keys[slot] = 0;
            set_link_bit(reinterpret_cast<uint32_t *>(e.flags), cell, false);
        }
    }
}

// -------------------------------------------------------------- finalize
// One CTA per active episode: scales the fixed-point sums to forces, clears
// them, and reduces total force, torque and power in a fixed order (so the
// sums do not depend on the mix or on launch order).
__global__ void __launch_bounds__(256) pool_finalize_kernel(const PoolEpisode *eps, const PoolActive *act,
                                                            LinkTable lt)
{
    __shared__ double red[4][8];
    const int n = (int)act->n;
    if (blockIdx.x == 0 && threadIdx.x == 0) *lt.count = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        const PoolEpisode &e = eps[act->slot[a]];
        double fx = 0.0, fy = 0.0, tq = 0.0, pw = 0.0;
        for (int v = threadIdx.x; v < e.nv; v += blockDim.x) {
            // the single-grid finalize's expression (finalize_forces_kernel)
            const double f0 = (double)e.acc[2 * v] * (1.0 / kForceScale) * e.cf;
            const double f1 = (double)e.acc[2 * v + 1] * (1.0 / kForceScale) * e.cf;
            e.acc[2 * v] = 0;
            e.acc[2 * v + 1] = 0;
            e.force[2 * v] = f0;
            e.force[2 * v + 1] = f1;
            const double rx = (double)e.V[2 * v] - (double)e.cx0, ry = (double)e.V[2 * v + 1] - (double)e.cy0;
            fx += f0;
            fy += f1;
            tq += rx * f1 - ry * f0;
            pw -= f0 * (double)e.U[2 * v] + f1 * (double)e.U[2 * v + 1];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            tq += __shfl_xor_sync(0xffffffffu, tq, o);
            pw += __shfl_xor_sync(0xffffffffu, pw, o);
        }
        if (lane == 0) {
            red[0][warp] = fx;
            red[1][warp] = fy;
            red[2][warp] = tq;
            red[3][warp] = pw;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double s[4] = {0.0, 0.0, 0.0, 0.0};
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                for (int k = 0; k < 4; ++k) s[k] += red[k][w];
            // rl/env.py:172-175: energy += power * dt when the power is positive
            if (s[3] > 0.0) e.sums[0] += s[3] * (double)e.ct;
            e.sums[1] += s[0];
            e.sums[2] += s[1];
            e.sums[3] += s[2];
        }
        __syncthreads();
    }
}

// One thread per active episode: publish the control step's sums and the
// latched status, then clear them for the next control step.
__global__ void pool_outputs_kernel(const PoolEpisode *eps, const PoolActive *act, PoolOutput *out, int substeps)
{
    const int n = (int)act->n;
    const double inv = 1.0 / (double)substeps;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        const uint32_t s = act->slot[a];
        const PoolEpisode &e = eps[s];
        PoolOutput o;
        o.energy = e.sums[0];
        o.force[0] = e.sums[1] * inv;
        o.force[1] = e.sums[2] * inv;
        o.torque = e.sums[3] * inv;
        o.status = *e.status;
        o.pad = 0;
        out[s] = o;
        for (int k = 0; k < 4; ++k) e.sums[k] = 0.0;
        *e.status = 0;
    }
}

// -------------------------------------------------------------- launchers
cudaError_t launch_pool_kinematics(const PoolEpisode *eps, const PoolParams *prm, const PoolActive *act, int substep,
                                   int grid, cudaStream_t st)
{
    pool_kinematics_kernel<<<grid, 256, 0, st>>>(eps, prm, act, substep);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_pool_detect(const PoolEpisode *eps, const PoolActive *act, const LinkTable &lt, uint32_t *owner,
                               int parity, int grid, cudaStream_t st)
{
    pool_detect_kernel<T><<<grid, 256, 0, st>>>(eps, act, lt, owner, parity);
    return cudaGetLastError();
}

template <typename T, int TX, int TY> static const void *dense_fn()
{
    return reinterpret_cast<const void *>(&pool_dense_kernel<T, TX, TY>);
}

template <typename T>
cudaError_t launch_pool_dense(const PoolEpisode *eps, const PoolActive *act, int parity, int shape, int grid,
                              cudaStream_t st)
{
    switch (shape) {
    case 0: pool_dense_kernel<T, 32, 4><<<grid, 32 * 4, 0, st>>>(eps, act, parity); break;
    case 1: pool_dense_kernel<T, 32, 8><<<grid, 32 * 8, 0, st>>>(eps, act, parity); break;
    case 2: pool_dense_kernel<T, 64, 4><<<grid, 64 * 4, 0, st>>>(eps, act, parity); break;
    case 3: pool_dense_kernel<T, 32, 16><<<grid, 32 * 16, 0, st>>>(eps, act, parity); break;
    case 4: pool_dense_kernel<T, 64, 8><<<grid, 64 * 8, 0, st>>>(eps, act, parity); break;
    case 5: pool_strip_kernel<T, 64, 32, 4><<<grid, 64, 0, st>>>(eps, act, parity); break;
    case 6: pool_strip_kernel<T, 128, 32, 4><<<grid, 128, 0, st>>>(eps, act, parity); break;
    default: pool_strip_kernel<T, 128, 64, 4><<<grid, 128, 0, st>>>(eps, act, parity); break;
    }
    return cudaGetLastError();
}

template <typename T> int pool_dense_blocks_per_sm(int shape)
{
    const void *fn;
    int threads;
    switch (shape) {
    case 0: fn = dense_fn<T, 32, 4>(); threads = 128; break;
    case 1: fn = dense_fn<T, 32, 8>(); threads = 256; break;
    case 2: fn = dense_fn<T, 64, 4>(); threads = 256; break;
    case 3: fn = dense_fn<T, 32, 16>(); threads = 512; break;
    case 4: fn = dense_fn<T, 64, 8>(); threads = 512; break;
    case 5: fn = reinterpret_cast<const void *>(&pool_strip_kernel<T, 64, 32, 4>); threads = 64; break;
    case 6: fn = reinterpret_cast<const void *>(&pool_strip_kernel<T, 128, 32, 4>); threads = 128; break;
    default: fn = reinterpret_cast<const void *>(&pool_strip_kernel<T, 128, 64, 4>); threads = 128; break;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, 0) != cudaSuccess || blocks < 1) blocks = 1;
    return blocks;
}

template <typename T> int pool_link_cells_blocks_per_sm()
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, pool_link_cells_kernel<T>, 256, 0) != cudaSuccess ||
        blocks < 1)
        blocks = 1;
    return blocks;
}

template <typename T>
cudaError_t launch_pool_link_cells(const PoolEpisode *eps, const LinkTable &lt, const uint32_t *owner, int parity,
                                   int grid, cudaStream_t st)
{
    pool_link_cells_kernel<T><<<grid, 256, 0, st>>>(eps, lt, owner, parity);
    return cudaGetLastError();
}

cudaError_t launch_pool_finalize(const PoolEpisode *eps, const PoolActive *act, const LinkTable &lt, int grid,
                                 cudaStream_t st)
{
    pool_finalize_kernel<<<grid, 256, 0, st>>>(eps, act, lt);
    return cudaGetLastError();
}

cudaError_t launch_pool_outputs(const PoolEpisode *eps, const PoolActive *act, PoolOutput *out, int substeps,
                                cudaStream_t st)
{
    pool_outputs_kernel<<<(kPoolMaxSlots + 127) / 128, 128, 0, st>>>(eps, act, out, substeps);
    return cudaGetLastError();
}

#define FFS_INST_POOL(T)                                                                                               \
    template cudaError_t launch_pool_detect<T>(const PoolEpisode *, const PoolActive *, const LinkTable &, uint32_t *, \
                                               int, int, cudaStream_t);                                                \
    template cudaError_t launch_pool_dense<T>(const PoolEpisode *, const PoolActive *, int, int, int, cudaStream_t);   \
    template int pool_dense_blocks_per_sm<T>(int);                                                                     \
    template int pool_link_cells_blocks_per_sm<T>();                                                                   \
    template cudaError_t launch_pool_link_cells<T>(const PoolEpisode *, const LinkTable &, const uint32_t *, int, int, \
                                                   cudaStream_t);
FFS_INST_POOL(float)
FFS_INST_POOL(__half)
FFS_INST_POOL(__nv_bfloat16)

} // namespace fflbm
