// Device bodies of the moving-boundary stages, shared by the single-grid
// kernels (ffs_links.cu) and the batched many-grid kernels (ffs_batch2d.cu).
#pragma once
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

// Finds or claims the cell's slot and keeps the smallest key of direction l.
// The table key is key_base + cell + 1: one table can serve many grids whose
// cells are numbered from distinct bases; the claiming thread tags the slot
// with owner_id in `owner` when that array is given.
template <int Q>
__device__ __forceinline__ void insert_link(const LinkTable &lt, uint32_t *flag_words, uint32_t cell, int l,
                                            unsigned long long key, uint32_t *status, uint32_t key_base = 0,
                                            uint32_t *owner = nullptr, uint32_t owner_id = 0)
{
    const uint32_t tkey = key_base + cell + 1;
    uint32_t slot = hash_cell(tkey - 1) & (lt.cap - 1);
    for (uint32_t probe = 0; probe < lt.cap; ++probe) {
        uint32_t cur = lt.keys[slot];
        if (cur == 0) {
            uint32_t old = atomicCAS(lt.keys + slot, 0u, tkey);
            if (old == 0) {
                uint32_t pos = atomicAdd(lt.count, 1u);
                lt.list[pos] = slot;
                if (owner) owner[slot] = owner_id;
                set_link_bit(flag_words, cell, true);
                cur = tkey;
            } else {
                cur = old;
            }
        }
        if (cur == tkey) {
            atomicMin(lt.links + (size_t)slot * Q + l, key);
            return;
        }
        slot = (slot + 1) & (lt.cap - 1);
    }
    atomicOr(status, kStatusLinkOverflow);
}

// D2Q9 link detection of segment e by one warp: every cell of the segment's
// bounding box grown by one cell (getBoundingBox: min from FLT_MAX, max from
// FLT_MIN (sic), then / dx) and every direction 1 <= l < 9 whose link segment
// x -> x - c_l crosses the element gets a (depth, element) key.  Items are
// numbered cell * 8 + (l - 1) with cells in row-major order; 32 items are four
// cells, so a lane keeps one direction and steps its cell by four, carrying
// the cell's coordinates forward instead of dividing them out.
//
// Most pairs cannot cross: a hit needs the element's line to separate the
// link's two end points (line_intersect's t1 = s2 / (s2 - s1) in (0, 1), with
// s1, s2 their signed distances).  A cheap prefilter drops a pair only when
// both end points lie on the same side by more than a hundredth of a cell
// (times the element's length); then t1 is at least about 7e-3 outside
// (0, 1), far beyond the exact test's rounding, so the link set is the
// exact test's.  The surviving pairs are queued in `wq` (64 entries of this
// warp's shared memory) and the exact, explicitly rounded test runs on 32 of
// them at a time, so that its lanes are not idle.  Boxes wider or taller than
// 16,383 cells skip the queue (the packed item holds 14-bit coordinates).
template <typename T>
__device__ __forceinline__ void detect_element2_warp(const GridArgs<T> &g, uint32_t *flag_words, const LinkTable &lt,
                                                     const SurfaceArgs &s, const StepScalars &sc, long long e,
                                                     uint32_t *wq, uint32_t key_base = 0, uint32_t *owner = nullptr,
                                                     uint32_t owner_id = 0)
{
    constexpr int Q = 9;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const uint32_t va = s.E[2 * e], vb = s.E[2 * e + 1];
    if (va >= (uint32_t)s.nv || vb >= (uint32_t)s.nv) {
        if (lane == 0) atomicOr(g.status, kStatusBadElement);
        return;
    }
    float bmin[2] = {3.402823466e+38f, 3.402823466e+38f};
    float bmax[2] = {1.175494351e-38f, 1.175494351e-38f};
    const uint32_t vid[2] = {va, vb};
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float c = s.V[(size_t)vid[j] * 2 + k];
            if (c < bmin[k]) bmin[k] = c;
            if (bmax[k] < c) bmax[k] = c;
        }
    const float cl = sc.cl;
    const int lo0 = max(__float2int_rz(geom::dvd(bmin[0], cl)) - 1, 0);
    const int hi0 = min(__float2int_rz(geom::dvd(bmax[0], cl)) + 1, g.nx - 1);
    const int lo1 = max(__float2int_rz(geom::dvd(bmin[1], cl)) - 1, 0);
    const int hi1 = min(__float2int_rz(geom::dvd(bmax[1], cl)) + 1, g.ny - 1);
    const int ext0 = hi0 - lo0 + 1, ext1 = hi1 - lo1 + 1;
    if (ext0 <= 0 || ext1 <= 0) return;
    const long long items = (long long)ext0 * ext1 * (Q - 1);
    const int l = (lane & 7) + 1;
    int cx, cy, cz;
    dir_vec<2>(l, cx, cy, cz);
    // the exact test of cell (i, j), direction ll, and the insertion on a hit
    auto exact = [&](int i, int j, int ll) {
        int dx, dy, dz;
        dir_vec<2>(ll, dx, dy, dz);
        const geom::Hit h = geom::isect2(s.V, va, vb, geom::mul((float)i, cl), geom::mul((float)j, cl),
                                         geom::mul(geom::sub((float)i, (float)dx), cl),
                                         geom::mul(geom::sub((float)j, (float)dy), cl));
        if (!h.hit) return;
        const uint32_t cell = (uint32_t)((long long)j * g.nx + i);
        insert_link<Q>(lt, flag_words, cell, ll, geom::link_key(h.depth, (uint32_t)e), g.status, key_base, owner,
                       owner_id);
    };
    int ci = lane >> 3, cj = 0;
    while (ci >= ext0) { ci -= ext0; ++cj; }
    if (ext0 > 16383 || ext1 > 16383) {
        for (long long it = lane; it < items; it += 32) {
            if (it != lane) {
                ci += 4;
                while (ci >= ext0) { ci -= ext0; ++cj; }
            }
            exact(lo0 + ci, lo1 + cj, l);
        }
        return;
    }
    // the element's line: normal (y3 - y4, x4 - x3) through vertex 4; the
    // prefilter's own rounding is far below its margin
    const float x3 = s.V[2 * (size_t)va], y3 = s.V[2 * (size_t)va + 1];
    const float x4 = s.V[2 * (size_t)vb], y4 = s.V[2 * (size_t)vb + 1];
    const float en0 = y3 - y4, en1 = x4 - x3;
    const float margin = 1e-2f * cl * sqrtf(en0 * en0 + en1 * en1);
    const float dstep = cl * (en0 * (float)cx + en1 * (float)cy); // s1 - s2 of this lane's direction
    const unsigned below = (1u << lane) - 1u;
    int qn = 0;
    for (long long base = 0; base < items; base += 32) {
        if (base != 0) {
            ci += 4;
            while (ci >= ext0) { ci -= ext0; ++cj; }
        }
        bool cand = false;
        if (base + lane < items) {
            const float s1 = en0 * ((float)(lo0 + ci) * cl - x4) + en1 * ((float)(lo1 + cj) * cl - y4);
            const float s2 = s1 - dstep;
            cand = !(fabsf(s1) > margin && fabsf(s2) > margin && ((s1 > 0.0f) == (s2 > 0.0f)));
        }
        const unsigned m = __ballot_sync(full, cand);
        if (cand) wq[qn + __popc(m & below)] = ((uint32_t)cj << 17) | ((uint32_t)ci << 3) | (uint32_t)(l - 1);
        qn += __popc(m);
        if (qn >= 32) {
            __syncwarp();
            const uint32_t code = wq[lane];
            __syncwarp();
            if (lane < qn - 32) wq[lane] = wq[32 + lane];
            __syncwarp();
            qn -= 32;
            exact(lo0 + (int)((code >> 3) & 0x3fffu), lo1 + (int)(code >> 17), (int)(code & 7u) + 1);
        }
    }
    __syncwarp();
    if (lane < qn) {
        const uint32_t code = wq[lane];
        exact(lo0 + (int)((code >> 3) & 0x3fffu), lo1 + (int)(code >> 17), (int)(code & 7u) + 1);
    }
    __syncwarp();
}

// Per-vertex force shares of the links of one cell, added to the vertex
// accumulators in 2^-32 fixed point with 64-bit integer atomics, one per
// (link, vertex slot, component).  Integer sums are associative, so the
// per-vertex result does not depend on warp, lane or launch order.  Each
// share is first rounded to 2^-24 (as an int32) and then scaled by 2^8,
// which is exactly what summing the int32 shares of a cell's links to one
// element and scaling the sum would give; a share beyond +-127 lattice units
// is clamped and flagged.  (An earlier form summed the links of one element
// within the warp first, with __match_any_sync and __reduce_add_sync over
// partial masks; the compiler loops such collectives per group, which cost
// about 120 instructions per cell, more than the atomics they saved.)
template <int DIM>
__device__ __forceinline__ void add_forces_warp(long long *acc, bool active, uint32_t elem, const uint32_t *vert,
                                                const float (*share)[3], uint32_t *status, uint32_t group = 0)
{
    (void)elem;
    (void)group;
    if (!active) return;
#pragma unroll
    for (int j = 0; j < DIM; ++j)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float v = share[j][k];
            if (!(fabsf(v) < 127.0f)) {
                atomicOr(status, kStatusForceRange);
                v = isfinite(v) ? copysignf(127.0f, v) : 0.0f;
            }
            const int q = __float2int_rn(v * 16777216.0f); // 2^24
            if (q != 0)
                atomicAdd(reinterpret_cast<unsigned long long *>(acc + (size_t)vert[j] * DIM + k),
                          (unsigned long long)((long long)q * 256)); // 2^24 -> 2^32
        }
}

// Lanes per link cell: a D3Q27 cell takes a whole warp, a D2Q9 cell half of
// one, so a warp updates two D2Q9 cells at once.
template <int DIM> constexpr int kLinkGroup = DIM == 2 ? 16 : 32;

// Update of one link-owning cell by one lane group of kLinkGroup<DIM> lanes
// (lane i of the group = direction i): wall bounce-back, moving-wall
// reconstruction with its momentum-exchange force shares, or the ordinary
// pull; the raw moments are reduced across the group and its lane 0
// collides, stores and feeds outlets.  `links` holds the Q keys of the
// cell's table slot; the force shares go to `acc`.  Every lane of the warp
// calls this together (the force sums and the reduction are warp-wide); a
// group with valid = false has no cell in this iteration and only takes part in
// those, with arguments that still name a real cell.
template <int DIM, typename T, bool HALF>
__device__ __forceinline__ void link_cell_update(const GridArgs<T> &g, const unsigned long long *links,
                                                 uint32_t slot, uint32_t cell, long long *acc,
                                                 const SurfaceArgs &s, const StepScalars &sc, bool valid = true)
{
    constexpr int Q = Lattice<DIM>::Q, NM = Lattice<DIM>::NM, G = kLinkGroup<DIM>;
    static_assert(Q <= G, "one lane per direction");
    const int lane = threadIdx.x & (G - 1);
    const unsigned full = 0xffffffffu;
    // cell indices are 32-bit (the link table keys them so), and so is every
    // index formed from them here
    const uint32_t nx = (uint32_t)g.nx, nxy = nx * (uint32_t)g.ny;
    const bool wx = g.periodic & 1, wy = g.periodic & 2, wz = g.periodic & 4;
    const uint32_t row = cell / nx;
    const int x = (int)(cell - row * nx);
    const uint32_t z32 = row / (uint32_t)g.ny;
    const int y = (int)(row - z32 * (uint32_t)g.ny);
    const int z = (int)z32;
    const uint8_t f8 = g.flags[cell];
    const bool upd = valid && is_updated(f8 & kTypeMask);
    float mc[NM];
    float pop = 0.0f;
    bool has_share = false;
    uint32_t hit_elem = 0xffffffffu;
    uint32_t vshare[3] = {0, 0, 0};
    float share[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}; // [vertex][component]
    // Every load the update may need goes out before any of them is tested:
    // the cell's own moments and, per lane, the node type of the wrapped
    // neighbour, the link key and the moments of the cell an ordinary pull
    // reads (a lane that takes the bounce-back or a moving-wall link discards
    // its pull).  The update then waits for one round of loads where testing
    // the node type and the key first would make it wait for three.
    load_moments<DIM, T>(mc, g.src, g.ncell, cell, g.codec);
    if (upd) {
        Coef<DIM> own;
        own.make(mc);
        if (lane < Q) {
            const int i = lane;
            int cx, cy, cz;
            dir_vec<DIM>(i, cx, cy, cz);
            const int x1 = x - cx, y1 = y - cy, z1 = z - cz;
            const bool notCross = x1 >= 0 && x1 < g.nx && y1 >= 0 && y1 < g.ny && z1 >= 0 && z1 < g.nz;
            // the wrapped neighbour (x1, y1, z1 are within one cell of the grid)
            auto wrap1 = [](int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); };
            const uint32_t ib = (uint32_t)wrap1(z1, g.nz) * nxy + (uint32_t)wrap1(y1, g.ny) * nx + (uint32_t)wrap1(x1, g.nx);
            // the ordinary pull's source: the upstream halo cell (halo_index)
            const int sx = halo_index(x1, g.nx, wx), sy = halo_index(y1, g.ny, wy), sz = halo_index(z1, g.nz, wz);
            const uint32_t sidx = (uint32_t)sz * nxy + (uint32_t)sy * nx + (uint32_t)sx;
            const uint8_t fb = g.flags[ib];
            const unsigned long long key = notCross ? links[(size_t)slot * Q + i] : ~0ull;
            float pulled;
            {
                float mn[NM];
                load_moments<DIM, T>(mn, g.src, g.ncell, sidx, g.codec);
                Coef<DIM> nc;
                nc.make(mn);
                float v = nc.population(cx, cy, cz);
                if (HALF) v = round_half(v);
                pulled = fmaxf(v, 0.0f);
            }
            bool done = false;
            // a wall neighbour: bounce-back, no link (with wall_stream in 2D, the
            // reference's 2D kernel: the ordinary pull, no link either)
            const bool bb = is_bounce_back<DIM>(fb & kTypeMask);
            if (bb && !(DIM == 2 && g.wall_stream)) {
                float v = own.population(-cx, -cy, -cz);
                if (HALF) v = round_half(v);
                pop = fmaxf(v, 0.0f);
                done = true;
            } else if (!bb && notCross) {
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
            if (!done) pop = pulled;
        }
    }
    // forces: one share per (link, element vertex), summed per element
    add_forces_warp<DIM>(acc, has_share, hit_elem, vshare, share, g.status, (threadIdx.x & 31) / G);
    // raw moments by reduction within the group (lanes Q.. add exact zeros,
    // so the sums equal those of a whole-warp reduction)
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
        for (int o = G / 2; o > 0; o >>= 1) R[k] += __shfl_xor_sync(full, R[k], o);
    if (upd) {
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
                stored_values<DIM, T>(m, ms, cell, g.codec);
                feed_outlets<DIM, T>(g, cell, ms, g.wallmask[cell]);
            }
        }
    }
}

} // namespace fflbm
