// Moving-boundary (interpolated moving-wall) bounce-back and surface forces.
//
// Reference: the occupancy kernels mrSolver2DComputeOccupancyFlagKernel_v3 /
// mrSolver3DComputeOccupancyFlagKernel_v3 (FsiCoupling2D.cu:31-80,
// FsiCoupling3D.cu:31-81) fill a dense hitIndex of Q u32 per cell, memset to
// 0xFF every step, and the fused kernels consume it (FsiCoupling2D.cu:183-216,
// FsiCoupling3D.cu:224-275) with FP32 atomicAdd force scatter
// (SolidGeometryProxy_Device.cuh:184-194, :401-421).
//
// Here the link set is sparse and O(surface):
//   detect      one warp per element tests the (cell, direction) pairs of the
//               element's bounding box grown by one cell and inserts hits into
//               an open-addressing table keyed by cell; per (cell, direction)
//               atomicMin keeps the nearest (depth, element) key.  The owning
//               cell gets a LINK bit in its flag byte, so the dense kernels
//               skip it.  Nothing proportional to the grid is touched.
//   link cells  one warp per D3Q27 link-owning cell (half a warp per D2Q9
//               cell), lane i = direction i: wall
//               bounce-back, moving-wall reconstruction with the momentum
//               exchange force, or the ordinary pull (reconstructing the
//               neighbour's population from its moments).  The warp reduces
//               the raw moments with shuffles and lane 0 collides and stores.
//   forces      each link's DIM vertex shares are summed as 64-bit fixed point
//               (2^-32 lattice units), first within the warp (lanes hitting the
//               same vertex, found with __match_any_sync, are combined by
//               shuffles) and then with integer atomics: integer addition is
//               associative, so the per-vertex sums are bit-reproducible
//               whatever the launch order, and exact up to the 2^-32
//               quantisation of each share.  A final pass scales by Cf and adds
//               to the caller's force array (+ optional FP64 copy).
#include <algorithm>

#include "ffs_links_dev.cuh"

namespace fflbm {

// ------------------------------------------------------------------ detect
static int sm_count() { return device_sms(); }

// CTAs of `threads` threads of KERNEL that are resident on the device at
// once (no dynamic shared memory); the occupancy is queried once per kernel.
template <auto KERNEL> static int resident_grid(int threads)
{
    static int per_sm = 0;
    if (!per_sm && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, KERNEL, threads, 0) != cudaSuccess ||
                    per_sm < 1))
        per_sm = 1;
    return sm_count() * per_sm;
}

// D3Q27: one warp per triangle, one lane per link direction (lanes 0..25 for
// l = 1..26).  The triangle's own geometry is evaluated once (tri_pre), and so
// is each lane's projected link length a = cl n.c_l and its reciprocal; the
// warp then walks the bounding-box cells (x fastest, nested loops, no index
// arithmetic), and the cell's signed distance to the plane,
// s1 = n.(p - v0), costs one multiply-add per cell (its y/z part is formed
// once per row).  A conservative prefilter discards the (cell, direction)
// pairs whose link segment clearly misses: the plane is not reached (t = s1 / a
// outside [0, 1] by more than a margin of 2e-3 cells, tested as s1 sign(a)
// against [-margin, |a| + margin]) or the plane point lies outside the
// triangle by more than 1% in barycentric terms.  The barycentric test is
// used only where its own rounding is far below that margin: the plane
// point carries an absolute error of a few float ulps of the coordinates
// (about 2.4e-7 x the largest grid extent in cells x cl), and a barycentric
// coordinate divides it by (shortest edge x sin^2 of the angle between the
// edges), so triangles with a tiny edge or angle (slivers, nearly
// coincident vertices) skip it and the exact test decides.  Every remaining pair gets
// the exact, explicitly rounded test, so the link set does not depend on
// this enumeration (the table keeps the minimum key per cell and direction).
// Only a few lanes of a cell pass the prefilter, so the surviving pairs are
// queued in shared memory (64 entries per warp) and the exact test runs on 32
// of them at a time; boxes larger than 1024 x 1024 x 128 cells skip the queue.
template <typename T>
__global__ void __launch_bounds__(256) detect_links3_kernel(GridArgs<T> g, uint32_t *flag_words, LinkTable lt,
                                                            SurfaceArgs s, StepScalars sc)
{
    constexpr int Q = 27;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const float cl = sc.cl;
    const float margin = 2e-3f * cl;
    const bool act = lane < Q - 1;
    const int l = act ? lane + 1 : 1;
    int cx, cy, cz;
    dir_vec<3>(l, cx, cy, cz);
    const float ccx = (float)cx * cl, ccy = (float)cy * cl, ccz = (float)cz * cl;
    __shared__ uint32_t queue[8][64]; // per warp: (cell, direction) pairs for the exact test
    uint32_t *wq = queue[threadIdx.x >> 5];
    const unsigned full = 0xffffffffu, below = (1u << lane) - 1u;
    for (long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < s.ne; e += nwarps) {
        const uint32_t ia = s.E[3 * e], ib = s.E[3 * e + 1], ic = s.E[3 * e + 2];
        if (ia >= (uint32_t)s.nv || ib >= (uint32_t)s.nv || ic >= (uint32_t)s.nv) {
            if (lane == 0) atomicOr(g.status, kStatusBadElement);
            continue;
        }
        const geom::TriPre tr = geom::tri_pre(s.V, ia, ib, ic);
        const float inv_den = __fdividef(1.0f, tr.den);
        const float coord_err = 2.4e-7f * (float)max(g.nx, max(g.ny, g.nz)) * cl;
        const bool bary_ok =
            sqrtf(fminf(tr.d00, tr.d11)) * (tr.den / (tr.d00 * tr.d11)) > 400.0f * coord_err; // error < 0.0025
        float bmin[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
        float bmax[3] = {1.175494351e-38f, 1.175494351e-38f, 1.175494351e-38f};
        const uint32_t vid[3] = {ia, ib, ic};
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float c = s.V[(size_t)vid[j] * 3 + k];
                if (c < bmin[k]) bmin[k] = c;
                if (bmax[k] < c) bmax[k] = c;
            }
        const int n3[3] = {g.nx, g.ny, g.nz};
        int lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = max(__float2int_rz(geom::dvd(bmin[k], cl)) - 1, 0);
            hi[k] = min(__float2int_rz(geom::dvd(bmax[k], cl)) + 1, n3[k] - 1);
        }
        // this lane's direction against the triangle's plane
        const float a = cl * (tr.n[0] * cx + tr.n[1] * cy + tr.n[2] * cz);
        const float fa = fabsf(a);
        const bool reach = fa > margin;              // else: the link runs (nearly) parallel to the plane
        const float sg = a > 0.0f ? 1.0f : -1.0f;
        const float inv_a = reach ? __fdividef(1.0f, a) : 0.0f;
        // the largest plane distance |s1| that any lane's test below accepts
        // (fa + margin, or 2 margin for a lane parallel to the plane): a cell
        // farther from the plane has no candidate, and the whole warp skips
        // it (s1 is the same for every lane)
        float reach_max = act ? (reach ? fa + margin : 2.0f * margin) : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) reach_max = fmaxf(reach_max, __shfl_xor_sync(full, reach_max, o));
        // the exact test of cell (i, j, k3), direction ll, and the insertion on a hit
        auto exact = [&](int i, int j, int k3, int ll) {
            int dx, dy, dz;
            dir_vec<3>(ll, dx, dy, dz);
            float p1[3] = {geom::mul((float)i, cl), geom::mul((float)j, cl), geom::mul((float)k3, cl)};
            float p2[3] = {geom::mul(geom::sub((float)i, (float)dx), cl), geom::mul(geom::sub((float)j, (float)dy), cl),
                           geom::mul(geom::sub((float)k3, (float)dz), cl)};
            const geom::Hit h = geom::isect3_pre(tr, p1, p2);
            if (!h.hit) return;
            const uint32_t cell = (uint32_t)(((long long)k3 * g.ny + j) * g.nx + i);
            insert_link<Q>(lt, flag_words, cell, ll, geom::link_key(h.depth, (uint32_t)e), g.status);
        };
        const bool queued = hi[0] - lo[0] < 1024 && hi[1] - lo[1] < 1024 && hi[2] - lo[2] < 128;
        int qn = 0;
        auto drain = [&](int upto) { // run the exact test on the first `upto` queued pairs
            __syncwarp();
            const uint32_t code = wq[lane];
            __syncwarp();
            if (lane < qn - upto) wq[lane] = wq[upto + lane];
            __syncwarp();
            if (lane < upto)
                exact(lo[0] + (int)(code & 1023u), lo[1] + (int)((code >> 10) & 1023u), lo[2] + (int)((code >> 20) & 127u),
                      (int)(code >> 27) + 1);
            qn -= upto;
        };
        for (int k3 = lo[2]; k3 <= hi[2]; ++k3) {
            const float pz = (float)k3 * cl - tr.v0[2];
            for (int j = lo[1]; j <= hi[1]; ++j) {
                const float py = (float)j * cl - tr.v0[1];
                const float s_yz = tr.n[1] * py + tr.n[2] * pz;
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    const float px = (float)i * cl - tr.v0[0];
                    const float s1 = fmaf(tr.n[0], px, s_yz);
                    if (fabsf(s1) > reach_max) continue;
                    bool cand;
                    if (reach) {
                        const float sa = sg * s1;
                        cand = !(sa < -margin || sa > fa + margin);
                        if (cand && bary_ok) {
                            // plane point relative to v0: p1 - t c cl - v0
                            const float t = s1 * inv_a;
                            const float wx = px - t * ccx, wy = py - t * ccy, wz = pz - t * ccz;
                            const float d20 = wx * tr.e1[0] + wy * tr.e1[1] + wz * tr.e1[2];
                            const float d21 = wx * tr.e2[0] + wy * tr.e2[1] + wz * tr.e2[2];
                            const float u = (tr.d11 * d20 - tr.d01 * d21) * inv_den;
                            const float v = (tr.d00 * d21 - tr.d01 * d20) * inv_den;
                            cand = !(u < -0.01f || v < -0.01f || u + v > 1.01f);
                        }
                    } else {
                        cand = !(fabsf(s1) > 2.0f * margin);
                    }
                    cand = act && cand;
                    if (!queued) {
                        if (cand) exact(i, j, k3, l);
                        continue;
                    }
                    const unsigned m = __ballot_sync(full, cand);
                    if (cand)
                        wq[qn + __popc(m & below)] = (uint32_t)(i - lo[0]) | ((uint32_t)(j - lo[1]) << 10) |
                                                     ((uint32_t)(k3 - lo[2]) << 20) | ((uint32_t)(l - 1) << 27);
                    qn += __popc(m);
                    if (qn >= 32) drain(32);
                }
            }
        }
        if (queued && qn > 0) drain(qn);
        __syncwarp();
    }
}

// D2Q9: one warp per segment (detect_element2_warp).
template <typename T>
__global__ void __launch_bounds__(256) detect_links2_kernel(GridArgs<T> g, uint32_t *flag_words, LinkTable lt,
                                                            SurfaceArgs s, StepScalars sc)
{
    __shared__ uint32_t queue[8][64]; // per warp: (cell, direction) pairs for the exact test
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < s.ne; e += nwarps)
        detect_element2_warp<T>(g, flag_words, lt, s, sc, e, queue[threadIdx.x >> 5]);
}

// -------------------------------------------------------------- link cells
// One fixed-point force sum -> physical force: added to the surface's force
// arrays, or, in the coupled step, written to the mapped volume vertex (whose
// force the gather zeroed), as scatterSurfaceForcesToVolume assigns it
// (src/fsi/FsiCouplingKernels.cu:59-90).
template <int DIM>
__device__ __forceinline__ void finalize_force(const SurfaceArgs &s, long long t, long long a, double cf)
{
    double f = (double)a * (1.0 / kForceScale) * cf;
    if (s.vforces) {
        const long long i = t / DIM;
        const uint32_t m = s.map[i];
        if (m < (uint32_t)s.nvol) s.vforces[(size_t)m * DIM + (t - i * DIM)] = (float)f;
    } else {
        if (s.forces) s.forces[t] += (float)f;
        if (s.forces64) s.forces64[t] += f;
    }
}

template <int DIM, typename T, bool HALF, bool FOLD>
__global__ void __launch_bounds__(256, 5) link_cells_kernel(GridArgs<T> g, uint32_t *flag_words, LinkTable lt, SurfaceArgs s,
                                                         StepScalars sc)
{
    constexpr int Q = Lattice<DIM>::Q, G = kLinkGroup<DIM>, kPerWarp = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const uint32_t group = (threadIdx.x & 31) / G;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = *lt.count;
    for (uint32_t w = (((blockIdx.x * blockDim.x) + threadIdx.x) >> 5) * kPerWarp; w < n; w += nwarps * kPerWarp) {
        // a group past the end of the list rides along on the first group's cell
        const bool valid = w + group < n;
        const uint32_t slot = lt.list[valid ? w + group : w];
        const uint32_t cell = lt.keys[slot] - 1;
        link_cell_update<DIM, T, HALF>(g, lt.links, slot, cell, lt.acc, s, sc, valid);
        // return the slot to the empty state and drop the cell's LINK bit
        if (valid && lane < Q) lt.links[(size_t)slot * Q + lane] = ~0ull;
        __syncwarp();
        if (valid && lane == 0) {
            lt.keys[slot] = 0;
            set_link_bit(flag_words, cell, false);
        }
    }
    if constexpr (!FOLD) return;
    // The CTA that finishes last converts the force sums: every other CTA's
    // atomics are complete and fenced before its count.  No CTA waits for
    // another.  The counters are reset for the next step.
    __shared__ bool last_cta;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last_cta = atomicAdd(lt.done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last_cta) return;
    __threadfence();
    const long long nf = (long long)s.nv * DIM;
    for (long long t = threadIdx.x; t < nf; t += blockDim.x) {
        const long long a = __ldcg(lt.acc + t);
        if (a != 0) {
            finalize_force<DIM>(s, t, a, sc.cf);
            lt.acc[t] = 0;
        }
    }
    if (threadIdx.x == 0) {
        *lt.count = 0;
        *lt.done = 0;
    }
}

// Fixed-point sums -> physical forces: added to the surface's force arrays,
// or, in the coupled step, written to the mapped volume vertices (whose
// forces the gather zeroed), as scatterSurfaceForcesToVolume assigns them
// (src/fsi/FsiCouplingKernels.cu:59-90).
template <int DIM>
__global__ void finalize_forces_kernel(LinkTable lt, SurfaceArgs s, double cf)
{
    const long long n = (long long)s.nv * DIM;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        long long a = lt.acc[t];
        if (a != 0) {
            finalize_force<DIM>(s, t, a, cf);
            lt.acc[t] = 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *lt.count = 0;
}

// First stage of the coupled step (updateSurfaceStatesFromVolume,
// src/fsi/FsiCouplingKernels.cu:14-57, plus the volume-force zeroing of the
// solid solver's applyForces, src/fem/VBDSolver.cpp:105,289).  Map entries
// out of range latch the element-index status bit and gather zeros.
template <int DIM>
__global__ void gather_surface_kernel(const float *vpos, const float *vvel, const uint32_t *map, int nv, int nvol,
                                      float *spos, float *svel, float *vforces, uint32_t *status)
{
    const long long ns = (long long)nv * DIM, nz = (long long)nvol * DIM;
    const long long n = ns > nz ? ns : nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        if (t < nz) vforces[t] = 0.0f;
        if (t < ns) {
            const long long i = t / DIM;
            const uint32_t m = map[i];
            float p = 0.0f, u = 0.0f;
            if (m < (uint32_t)nvol) {
                p = vpos[(size_t)m * DIM + (t - i * DIM)];
                u = vvel[(size_t)m * DIM + (t - i * DIM)];
            } else {
                atomicOr(status, kStatusBadElement);
            }
            spos[t] = p;
            svel[t] = u;
        }
    }
}

template <int DIM>
__global__ void reset_links_kernel(LinkTable lt, uint32_t *flag_words)
{
    constexpr int Q = Lattice<DIM>::Q;
    const uint32_t n = *lt.count;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
        uint32_t slot = lt.list[w];
        uint32_t cell = lt.keys[slot] - 1;
        for (int l = 0; l < Q; ++l) lt.links[(size_t)slot * Q + l] = ~0ull;
        lt.keys[slot] = 0;
        set_link_bit(flag_words, cell, false);
    }
}

__global__ void zero_count_kernel(uint32_t *count) { *count = 0; }

// ---------------------------------------------------------------- launchers
template <int DIM, typename T>
cudaError_t launch_detect_links(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt, const SurfaceArgs &s,
                                const StepScalars &sc, cudaStream_t st)
{
    constexpr int Q = Lattice<DIM>::Q;
    if (s.ne <= 0) return cudaSuccess;
    if (DIM == 3) {
        long long warps = s.ne;
        int grid = (int)std::min<long long>((warps + 7) / 8, (long long)sm_count() * 16);
        detect_links3_kernel<T><<<grid, 256, 0, st>>>(g, flag_words, lt, s, sc);
        return cudaGetLastError();
    }
    const int grid = (int)std::min<long long>((s.ne + 7) / 8, (long long)sm_count() * 16);
    detect_links2_kernel<T><<<grid, 256, 0, st>>>(g, flag_words, lt, s, sc);
    return cudaGetLastError();
}

template <int DIM, typename T, bool HALF, bool FOLD>
static void launch_link_cells_as(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt, const SurfaceArgs &s,
                                 const StepScalars &sc, cudaStream_t st)
{
    link_cells_kernel<DIM, T, HALF, FOLD>
        <<<resident_grid<link_cells_kernel<DIM, T, HALF, FOLD>>(256), 256, 0, st>>>(g, flag_words, lt, s, sc);
}

template <int DIM, typename T>
cudaError_t launch_link_cells(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt, const SurfaceArgs &s,
                              const StepScalars &sc, cudaStream_t st, bool fold_forces)
{
    // persistent warps over the device-side count, one wave: as many CTAs of
    // 8 warps as are resident together (a CTA beyond that would run its fixed
    // share of the cells after the others finish)
    if (g.half_pops) {
        if (fold_forces) launch_link_cells_as<DIM, T, true, true>(g, flag_words, lt, s, sc, st);
        else launch_link_cells_as<DIM, T, true, false>(g, flag_words, lt, s, sc, st);
    } else {
        if (fold_forces) launch_link_cells_as<DIM, T, false, true>(g, flag_words, lt, s, sc, st);
        else launch_link_cells_as<DIM, T, false, false>(g, flag_words, lt, s, sc, st);
    }
    return cudaGetLastError();
}

template <int DIM>
cudaError_t launch_finalize_forces(const LinkTable &lt, const SurfaceArgs &s, double cf, cudaStream_t st)
{
    long long n = (long long)s.nv * DIM;
    int grid = (int)std::min<long long>((n + 255) / 256, (long long)sm_count() * 8);
    if (grid < 1) grid = 1;
    finalize_forces_kernel<DIM><<<grid, 256, 0, st>>>(lt, s, cf);
    return cudaGetLastError();
}

cudaError_t launch_gather_surface(int dim, const float *vpos, const float *vvel, const uint32_t *map, int nv, int nvol,
                                  float *spos, float *svel, float *vforces, uint32_t *status, cudaStream_t st)
{
    const long long n = (long long)std::max(nv, nvol) * dim;
    if (n == 0) return cudaSuccess;
    const int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)sm_count() * 8));
    if (dim == 2) gather_surface_kernel<2><<<grid, 256, 0, st>>>(vpos, vvel, map, nv, nvol, spos, svel, vforces, status);
    else gather_surface_kernel<3><<<grid, 256, 0, st>>>(vpos, vvel, map, nv, nvol, spos, svel, vforces, status);
    return cudaGetLastError();
}

template <int DIM>
cudaError_t launch_reset_links(const LinkTable &lt, uint32_t *flag_words, cudaStream_t st)
{
    reset_links_kernel<DIM><<<sm_count(), 256, 0, st>>>(lt, flag_words);
    zero_count_kernel<<<1, 1, 0, st>>>(lt.count);
    return cudaGetLastError();
}

#define FFS_INST_LINKS(DIM, T)                                                                                         \
    template cudaError_t launch_detect_links<DIM, T>(const GridArgs<T> &, uint32_t *, const LinkTable &,              \
                                                     const SurfaceArgs &, const StepScalars &, cudaStream_t);          \
    template cudaError_t launch_link_cells<DIM, T>(const GridArgs<T> &, uint32_t *, const LinkTable &,                \
                                                   const SurfaceArgs &, const StepScalars &, cudaStream_t, bool);
FFS_INST_LINKS(2, float)
FFS_INST_LINKS(2, __half)
FFS_INST_LINKS(2, __nv_bfloat16)
FFS_INST_LINKS(3, float)
FFS_INST_LINKS(3, __half)
FFS_INST_LINKS(3, __nv_bfloat16)
template cudaError_t launch_finalize_forces<2>(const LinkTable &, const SurfaceArgs &, double, cudaStream_t);
template cudaError_t launch_finalize_forces<3>(const LinkTable &, const SurfaceArgs &, double, cudaStream_t);
template cudaError_t launch_reset_links<2>(const LinkTable &, uint32_t *, cudaStream_t);
template cudaError_t launch_reset_links<3>(const LinkTable &, uint32_t *, cudaStream_t);

} // namespace fflbm
