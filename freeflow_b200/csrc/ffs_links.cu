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
//   detect      one thread per (element, direction) tests the cells of the
//               element's bounding box grown by one cell and inserts hits into
//               an open-addressing table keyed by cell; per (cell, direction)
//               atomicMin keeps the nearest (depth, element) key.  The owning
//               cell gets a LINK bit in its flag byte, so the dense kernels
//               skip it.  Nothing proportional to the grid is touched.
//   link cells  one warp per link-owning cell, lane i = direction i: wall
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

#include "ffs_geom.cuh"
#include "ffs_links.cuh"
#include "ffs_math.cuh"
#include "ffs_outlet.cuh"
#include "ffs_dense2d.cuh"

namespace fflbm {

__device__ __forceinline__ uint32_t hash_cell(uint32_t c)
{
    c ^= c >> 16; c *= 0x7feb352dU; c ^= c >> 15; c *= 0x846ca68bU; c ^= c >> 16;
    return c;
}

__device__ __forceinline__ void set_link_bit(uint32_t *flag_words, uint32_t cell, bool on)
{
    uint32_t bit = (uint32_t)kBitLink << (8 * (cell & 3));
    if (on) atomicOr(flag_words + (cell >> 2), bit);
    else atomicAnd(flag_words + (cell >> 2), ~bit);
}

// ------------------------------------------------------------------ detect
static int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Finds or claims the cell's slot and keeps the smallest key of direction l.
template <int Q>
__device__ __forceinline__ void insert_link(const LinkTable &lt, uint32_t *flag_words, uint32_t cell, int l,
                                            unsigned long long key, uint32_t *status)
{
    uint32_t slot = hash_cell(cell) & (lt.cap - 1);
    for (uint32_t probe = 0; probe < lt.cap; ++probe) {
        uint32_t cur = lt.keys[slot];
        if (cur == 0) {
            uint32_t old = atomicCAS(lt.keys + slot, 0u, cell + 1);
            if (old == 0) {
                uint32_t pos = atomicAdd(lt.count, 1u);
                lt.list[pos] = slot;
                set_link_bit(flag_words, cell, true);
                cur = cell + 1;
            } else {
                cur = old;
            }
        }
        if (cur == cell + 1) {
            atomicMin(lt.links + (size_t)slot * Q + l, key);
            return;
        }
        slot = (slot + 1) & (lt.cap - 1);
    }
    atomicOr(status, kStatusLinkOverflow);
}

// D3Q27: one warp per triangle.  The triangle's own geometry is evaluated
// once (tri_pre); lanes stride over (bounding-box cell, direction) pairs.  A
// conservative plane-distance test discards the pairs whose link segment
// clearly does not reach the triangle's plane (|signed distance of the cell|
// > |projection of the link| + a margin of 2e-3 cells, far above the float
// rounding of either quantity); every remaining pair gets the exact test.
template <typename T>
__global__ void __launch_bounds__(256) detect_links3_kernel(GridArgs<T> g, uint32_t *flag_words, LinkTable lt,
                                                            SurfaceArgs s, StepScalars sc)
{
    constexpr int Q = 27;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const float cl = sc.cl;
    const float margin = 2e-3f * cl;
    for (long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < s.ne; e += nwarps) {
        const uint32_t ia = s.E[3 * e], ib = s.E[3 * e + 1], ic = s.E[3 * e + 2];
        if (ia >= (uint32_t)s.nv || ib >= (uint32_t)s.nv || ic >= (uint32_t)s.nv) {
            if (lane == 0) atomicOr(g.status, kStatusBadElement);
            continue;
        }
        const geom::TriPre tr = geom::tri_pre(s.V, ia, ib, ic);
        const float inv_den = __fdividef(1.0f, tr.den);
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
        int lo[3], ext[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = max(__float2int_rz(geom::dvd(bmin[k], cl)) - 1, 0);
            int hi = min(__float2int_rz(geom::dvd(bmax[k], cl)) + 1, n3[k] - 1);
            ext[k] = max(hi - lo[k] + 1, 0);
        }
        const int ncells = ext[0] * ext[1] * ext[2];
        const int items = ncells * (Q - 1);
        for (int it = lane; it < items; it += 32) {
            const int l = it % (Q - 1) + 1;
            const int c = it / (Q - 1);
            const int i = lo[0] + c % ext[0];
            const int j = lo[1] + (c / ext[0]) % ext[1];
            const int k3 = lo[2] + c / (ext[0] * ext[1]);
            int cx, cy, cz;
            dir_vec<3>(l, cx, cy, cz);
            // prefilter in ordinary (fast) float math; it only rejects clear
            // misses: the plane is not reached (t outside [0, 1] by more than a
            // margin of 2e-3 cells) or the plane point lies outside the
            // triangle by more than 1% in barycentric terms
            const float px = (float)i * cl - tr.v0[0], py = (float)j * cl - tr.v0[1], pz = (float)k3 * cl - tr.v0[2];
            const float s1 = tr.n[0] * px + tr.n[1] * py + tr.n[2] * pz;
            const float a = cl * (tr.n[0] * cx + tr.n[1] * cy + tr.n[2] * cz);
            const float fa = fabsf(a);
            if (fa > margin) {
                const float t = __fdividef(s1, a);
                const float tol = __fdividef(margin, fa);
                if (t < -tol || t > 1.0f + tol) continue;
                // plane point relative to v0: p1 - t c cl - v0
                const float tc = t * cl;
                const float wx = px - tc * cx, wy = py - tc * cy, wz = pz - tc * cz;
                const float d20 = wx * tr.e1[0] + wy * tr.e1[1] + wz * tr.e1[2];
                const float d21 = wx * tr.e2[0] + wy * tr.e2[1] + wz * tr.e2[2];
                const float u = (tr.d11 * d20 - tr.d01 * d21) * inv_den;
                const float v = (tr.d00 * d21 - tr.d01 * d20) * inv_den;
                if (u < -0.01f || v < -0.01f || u + v > 1.01f) continue;
            } else if (fabsf(s1) > 2.0f * margin) {
                continue; // link parallel to the plane and away from it
            }
            float p1[3] = {geom::mul((float)i, cl), geom::mul((float)j, cl), geom::mul((float)k3, cl)};
            float p2[3] = {geom::mul(geom::sub((float)i, (float)cx), cl), geom::mul(geom::sub((float)j, (float)cy), cl),
                           geom::mul(geom::sub((float)k3, (float)cz), cl)};
            const geom::Hit h = geom::isect3_pre(tr, p1, p2);
            if (!h.hit) continue;
            const uint32_t cell = (uint32_t)(((long long)k3 * g.ny + j) * g.nx + i);
            insert_link<Q>(lt, flag_words, cell, l, geom::link_key(h.depth, (uint32_t)e), g.status);
        }
    }
}

template <int DIM, typename T>
__global__ void detect_links_kernel(GridArgs<T> g, uint32_t *flag_words, LinkTable lt, SurfaceArgs s, StepScalars sc)
{
    constexpr int Q = Lattice<DIM>::Q;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long e = gid / (Q - 1);
    const int l = (int)(gid % (Q - 1)) + 1;
    if (e >= s.ne) return;
    uint32_t vid[3] = {0, 0, 0};
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
        vid[j] = s.E[DIM * e + j];
        if (vid[j] >= (uint32_t)s.nv) { atomicOr(g.status, kStatusBadElement); return; }
    }
    // getBoundingBox: min from FLT_MAX, max from FLT_MIN (sic), then / dx
    float bmin[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float bmax[3] = {1.175494351e-38f, 1.175494351e-38f, 1.175494351e-38f};
#pragma unroll
    for (int j = 0; j < DIM; ++j)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float c = s.V[(size_t)vid[j] * DIM + k];
            if (c < bmin[k]) bmin[k] = c;
            if (bmax[k] < c) bmax[k] = c;
        }
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        lo[k] = max(__float2int_rz(geom::dvd(bmin[k], sc.cl)) - 1, 0);
        hi[k] = min(__float2int_rz(geom::dvd(bmax[k], sc.cl)) + 1, n[k] - 1);
    }
    int cx, cy, cz;
    dir_vec<DIM>(l, cx, cy, cz);
    const float cl = sc.cl;
    for (int k3 = lo[2]; k3 <= hi[2]; ++k3)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                geom::Hit h;
                if (DIM == 2) {
                    h = geom::isect2(s.V, vid[0], vid[1], geom::mul((float)i, cl), geom::mul((float)j, cl),
                                     geom::mul(geom::sub((float)i, (float)cx), cl),
                                     geom::mul(geom::sub((float)j, (float)cy), cl));
                } else {
                    float p1[3] = {geom::mul((float)i, cl), geom::mul((float)j, cl), geom::mul((float)k3, cl)};
                    float p2[3] = {geom::mul(geom::sub((float)i, (float)cx), cl),
                                   geom::mul(geom::sub((float)j, (float)cy), cl),
                                   geom::mul(geom::sub((float)k3, (float)cz), cl)};
                    h = geom::isect3(s.V, vid[0], vid[1], vid[2], p1, p2);
                }
                if (!h.hit) continue;
                const uint32_t cell = (uint32_t)(((long long)k3 * g.ny + j) * g.nx + i);
                insert_link<Q>(lt, flag_words, cell, l, geom::link_key(h.depth, (uint32_t)e), g.status);
            }
}

// -------------------------------------------------------------- link cells
// Per-vertex force shares of the links of one cell.  Lanes whose links hit
// the same element (found with __match_any_sync) are summed with the warp's
// integer reduction unit (__reduce_add_sync), one value per (vertex slot,
// component), in 2^-24 fixed point; the group leader then adds each sum, in
// 2^-32 fixed point, to the vertex accumulator with one 64-bit integer
// atomic.  Integer sums are associative, so the per-vertex result does not
// depend on warp, lane or launch order.  A share beyond +-127 lattice units
// (outside the 2^-24 range of 27 summed int32 shares) is clamped and flagged.
template <int DIM>
__device__ __forceinline__ void add_forces_warp(long long *acc, bool active, uint32_t elem, const uint32_t *vert,
                                                const float (*share)[3], uint32_t *status)
{
    const unsigned full = 0xffffffffu;
    const unsigned peers = __match_any_sync(full, active ? elem : 0xffffffffu);
    const int lane = threadIdx.x & 31;
    const bool leader = active && lane == __ffs(peers) - 1;
#pragma unroll
    for (int j = 0; j < DIM; ++j)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float v = active ? share[j][k] : 0.0f;
            if (!(fabsf(v) < 127.0f)) {
                if (active) atomicOr(status, kStatusForceRange);
                v = isfinite(v) ? copysignf(127.0f, v) : 0.0f;
            }
            const int q = __float2int_rn(v * 16777216.0f); // 2^24
            const int sum = (int)__reduce_add_sync(peers, (unsigned)q);
            if (leader && sum != 0)
                atomicAdd(reinterpret_cast<unsigned long long *>(acc + (size_t)vert[j] * DIM + k),
                          (unsigned long long)((long long)sum * 256)); // 2^24 -> 2^32
        }
}

template <int DIM, typename T, bool HALF>
__global__ void __launch_bounds__(256, 3) link_cells_kernel(GridArgs<T> g, uint32_t *flag_words, LinkTable lt, SurfaceArgs s,
                                                         StepScalars sc)
{
    constexpr int Q = Lattice<DIM>::Q, NM = Lattice<DIM>::NM;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = *lt.count;
    const long long nxy = (long long)g.nx * g.ny;
    const bool wx = g.periodic & 1, wy = g.periodic & 2, wz = g.periodic & 4;
    for (uint32_t w = ((blockIdx.x * blockDim.x) + threadIdx.x) >> 5; w < n; w += nwarps) {
        const uint32_t slot = lt.list[w];
        const uint32_t cell = lt.keys[slot] - 1;
        const int x = (int)(cell % g.nx);
        const int y = (int)((cell / g.nx) % g.ny);
        const int z = (int)(cell / nxy);
        const uint8_t f8 = g.flags[cell];
        if (is_updated(f8 & kTypeMask)) {
            float mc[NM];
            load_moments<DIM, T>(mc, g.src, g.ncell, cell, g.codec);
            Coef<DIM> own;
            own.make(mc);
            float pop = 0.0f;
            bool has_share = false;
            uint32_t hit_elem = 0xffffffffu;
            uint32_t vshare[3] = {0, 0, 0};
            float share[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}; // [vertex][component]
            if (lane < Q) {
                const int i = lane;
                int cx, cy, cz;
                dir_vec<DIM>(i, cx, cy, cz);
                const int x1 = x - cx, y1 = y - cy, z1 = z - cz;
                const bool notCross = x1 >= 0 && x1 < g.nx && y1 >= 0 && y1 < g.ny && z1 >= 0 && z1 < g.nz;
                const int ax = (x1 + g.nx) % g.nx, ay = (y1 + g.ny) % g.ny, az = (z1 + g.nz) % g.nz;
                const uint32_t ib = (uint32_t)((long long)az * nxy + (long long)ay * g.nx + ax);
                bool done = false;
                if (is_bounce_back<DIM>(g.flags[ib] & kTypeMask)) {
                    float v = own.population(-cx, -cy, -cz);
                    if (HALF) v = round_half(v);
                    pop = fmaxf(v, 0.0f);
                    done = true;
                } else if (notCross) {
                    const unsigned long long key = lt.links[(size_t)slot * Q + i];
                    if (key != ~0ull) {
                        const uint32_t e = (uint32_t)(key & 0xffffffffull);
                        const float cl = sc.cl;
                        geom::Hit h;
                        uint32_t vv[3] = {s.E[DIM * (size_t)e], s.E[DIM * (size_t)e + 1], DIM == 3 ? s.E[DIM * (size_t)e + 2] : 0u};
                        if (DIM == 2) {
                            h = geom::isect2(s.V, vv[0], vv[1], geom::mul((float)x, cl), geom::mul((float)y, cl),
                                             geom::mul((float)x1, cl), geom::mul((float)y1, cl));
                        } else {
                            float p1[3] = {geom::mul((float)x, cl), geom::mul((float)y, cl), geom::mul((float)z, cl)};
                            float p2[3] = {geom::mul((float)x1, cl), geom::mul((float)y1, cl), geom::mul((float)z1, cl)};
                            h = geom::isect3(s.V, vv[0], vv[1], vv[2], p1, p2);
                        }
                        if (h.hit) {
                            // wall velocity at the hit point, in lattice units
                            float uw[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                            for (int k = 0; k < DIM; ++k) {
                                float a = s.U[(size_t)vv[0] * DIM + k] * h.b[0] + s.U[(size_t)vv[1] * DIM + k] * h.b[1];
                                if (DIM == 3) a += s.U[(size_t)vv[2] * DIM + k] * h.b[2];
                                uw[k] = (DIM == 2) ? a * (sc.ct / sc.cl) : (a * sc.ct) / sc.cl;
                            }
                            // moving-wall population: Hermite expansion with the cell's
                            // density, the wall velocity and pi' = pi + uw uw - u u
                            float mw[NM];
                            mw[0] = mc[0];
#pragma unroll
                            for (int k = 0; k < DIM; ++k) mw[1 + k] = uw[k];
#pragma unroll
                            for (int k = DIM + 1; k < NM; ++k) {
                                const int a = MomentLayout<DIM>::pa(k), b = MomentLayout<DIM>::pb(k);
                                mw[k] = mc[k] + uw[a] * uw[b] - mc[1 + a] * mc[1 + b];
                            }
                            Coef<DIM> wc;
                            wc.make(mw);
                            const float fout = wc.population(cx, cy, cz);
                            float fin = own.population(-cx, -cy, -cz);
                            if (HALF) fin = round_half(fin);
                            fin = fmaxf(fin, 0.0f);
                            pop = fout;
                            done = true;
                            // momentum exchange, lattice units: fin (-c - uw) - fout (c - uw)
                            const float c3[3] = {(float)cx, (float)cy, (float)cz};
                            float F[3];
#pragma unroll
                            for (int k = 0; k < DIM; ++k) F[k] = fin * (-c3[k] - uw[k]) - fout * (c3[k] - uw[k]);
                            has_share = true;
                            hit_elem = e;
#pragma unroll
                            for (int j = 0; j < DIM; ++j) {
                                vshare[j] = vv[j];
#pragma unroll
                                for (int k = 0; k < DIM; ++k) share[j][k] = F[k] * h.b[j];
                            }
                        }
                    }
                }
                if (!done) {
                    // ordinary pull from the (clamped or wrapped) upstream cell
                    const int sx = halo_index(x1, g.nx, wx), sy = halo_index(y1, g.ny, wy), sz = halo_index(z1, g.nz, wz);
                    const uint32_t sidx = (uint32_t)((long long)sz * nxy + (long long)sy * g.nx + sx);
                    float mn[NM];
                    load_moments<DIM, T>(mn, g.src, g.ncell, sidx, g.codec);
                    Coef<DIM> nc;
                    nc.make(mn);
                    float v = nc.population(cx, cy, cz);
                    if (HALF) v = round_half(v);
                    pop = fmaxf(v, 0.0f);
                }
            }
            // forces: one share per (link, element vertex), summed per element
            add_forces_warp<DIM>(lt.acc, has_share, hit_elem, vshare, share, g.status);
            // raw moments by warp reduction
            int cx = 0, cy = 0, cz = 0;
            if (lane < Q) dir_vec<DIM>(lane, cx, cy, cz);
            const float fx = (float)cx, fy = (float)cy, fz = (float)cz;
            float R[NM];
            if (DIM == 2) {
                R[0] = pop; R[1] = pop * fx; R[2] = pop * fy;
                R[3] = pop * fx * fx; R[4] = pop * fy * fy; R[5] = pop * fx * fy;
            } else {
                R[0] = pop; R[1] = pop * fx; R[2] = pop * fy; R[3] = pop * fz;
                R[4] = pop * fx * fx; R[5] = pop * fy * fy; R[6] = pop * fz * fz;
                R[7] = pop * fx * fy; R[8] = pop * fy * fz; R[9] = pop * fx * fz;
            }
#pragma unroll
            for (int k = 0; k < NM; ++k)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) R[k] += __shfl_xor_sync(full, R[k], o);
            if (lane == 0) {
                float m[NM];
                if (DIM == 2) collide2(R, g.omega, m);
                else collide3(R, g.omega, m);
                T *planes[NM];
#pragma unroll
                for (int k = 0; k < NM; ++k) planes[k] = g.dst + (size_t)k * g.ncell;
                encode_store<DIM, T>(m, planes, cell, g.codec);
                if (bad_state<DIM>(m)) atomicOr(g.status, kStatusNonFinite);
                if (f8 & kBitOutletSrc) {
                    float ms[NM];
                    stored_values<DIM, T>(m, ms, g.codec);
                    feed_outlets<DIM, T>(g, cell, ms, g.wallmask[cell]);
                }
            }
        }
        // return the slot to the empty state and drop the cell's LINK bit
        if (lane < Q) lt.links[(size_t)slot * Q + lane] = ~0ull;
        __syncwarp();
        if (lane == 0) {
            lt.keys[slot] = 0;
            set_link_bit(flag_words, cell, false);
        }
    }
}

template <int DIM>
__global__ void finalize_forces_kernel(LinkTable lt, SurfaceArgs s, double cf)
{
    const long long n = (long long)s.nv * DIM;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        long long a = lt.acc[t];
        if (a != 0) {
            double f = (double)a * (1.0 / kForceScale) * cf;
            if (s.forces) s.forces[t] += (float)f;
            if (s.forces64) s.forces64[t] += f;
            lt.acc[t] = 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *lt.count = 0;
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
    long long threads = (long long)s.ne * (Q - 1);
    int block = 128;
    long long grid = (threads + block - 1) / block;
    detect_links_kernel<DIM, T><<<(unsigned)grid, block, 0, st>>>(g, flag_words, lt, s, sc);
    return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t launch_link_cells(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt, const SurfaceArgs &s,
                              const StepScalars &sc, cudaStream_t st)
{
    // persistent warps over the device-side count: 8 warps per CTA, 4 CTAs per SM
    int grid = sm_count() * 4;
    if (g.half_pops)
        link_cells_kernel<DIM, T, true><<<grid, 256, 0, st>>>(g, flag_words, lt, s, sc);
    else
        link_cells_kernel<DIM, T, false><<<grid, 256, 0, st>>>(g, flag_words, lt, s, sc);
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
                                                   const SurfaceArgs &, const StepScalars &, cudaStream_t);
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
