// Tile body of the fused D2Q9 update, shared by the single-grid kernel
// (ffs_dense2d.cu) and the batched many-grid kernel (ffs_batch2d.cu).
#pragma once
#include "ffs_common.cuh"
#include "ffs_math.cuh"
#include "ffs_outlet.cuh"

namespace fflbm {

struct D2 {
    static constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
    static constexpr int kHX = kTX + 2, kHY = kTY + 2, kHalo = kHX * kHY;
};

// Source index of a halo cell, as the reference's shared-memory fill computes
// it (FsiCoupling2D.cu:104-105, FsiCoupling3D.cu:106-108):
// min(n - 1, max(0, (sm - 1) + blockDim * blockIdx)).  blockDim * blockIdx is
// unsigned, so below the grid the sum wraps to a huge unsigned value and the
// index comes out as n - 1; above it the min clamps to n - 1.  The halo
// therefore wraps at the low face and clamps at the high face of every axis.
// A periodic axis wraps at both.  v >= -1 always; v may exceed n by a tile
// width.
__device__ __forceinline__ int halo_index(int v, int n, bool wrap)
{
    if (!wrap) return (v < 0 || v >= n) ? n - 1 : v;
    if (v < 0) v += n;
    if (v >= n) v -= n;
    if (v >= n) v %= n;
    return v;
}

// Halo cells of a TX x TY tile per thread (at most two for every shape used).
template <int TX, int TY> struct Halo2 {
    static constexpr int kHX = TX + 2, kHalo = (TX + 2) * (TY + 2), kThreads = TX * TY;
    static constexpr int kPer = (kHalo + kThreads - 1) / kThreads;
};

// Stored moments of the thread's halo cells of the tile at (x0, y0), as they
// are in memory (step 1 of dense2d_tile decodes them).  Issued ahead of use,
// these loads overlap the previous tile's work.
template <typename T, int TX, int TY>
__device__ __forceinline__ void dense2d_load(const GridArgs<T> &g, int x0, int y0, T (&raw)[Halo2<TX, TY>::kPer][6])
{
    using H = Halo2<TX, TY>;
    const bool wx = g.periodic & 1, wy = g.periodic & 2;
#pragma unroll
    for (int r = 0; r < H::kPer; ++r) {
        const int c = threadIdx.x + r * H::kThreads;
        if (c < H::kHalo) {
            const int hx = c % H::kHX, hy = c / H::kHX;
            const int gx = halo_index(x0 + hx - 1, g.nx, wx);
            const int gy = halo_index(y0 + hy - 1, g.ny, wy);
            const uint32_t idx = (uint32_t)(gy * g.nx + gx);
#pragma unroll
            for (int k = 0; k < 6; ++k) raw[r][k] = g.src[(size_t)k * g.ncell + idx];
        }
    }
}

// Populations of one cell from its stored moments (reconstruction step of
// the update); HALF rounds them to binary16 like the reference's __half tile.
template <typename T, bool HALF>
__device__ __forceinline__ void dense2d_recon(const GridArgs<T> &g, const T (&raw)[6], float (&f)[9])
{
    float m[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) m[k] = from_storage<2, T>(k, raw[k]);
    decode_moments<2, T>(m, g.codec);
    Coef<2> cf;
    cf.make(m);
    cf.populations(f);
    if (HALF) {
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = round_half(f[i]);
    }
}

// Update of one cell that the dense pass owns (flag f8: Fluid or
// SolidDynamic, no moving-boundary link): pull(i) is the reconstructed
// population i of the upstream cell x - c_i and own(i) that of the cell
// itself.  Bounce-back, clamp, raw moments, collision, store and the outlet
// feed follow FsiCoupling2D.cu:154-252.  IDX32: every moment index
// k * ncell + idx fits in 32 bits (the caller guarantees it), so the stores
// take 32-bit indices instead of six 64-bit plane pointers.
template <typename T, bool IDX32 = false, typename Pull, typename Own>
__device__ __forceinline__ void dense2d_update_cell(const GridArgs<T> &g, uint32_t idx, uint32_t f8, Pull &&pull,
                                                    Own &&own)
{
    using L = Lattice<2>;
    float pop[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) pop[i] = pull(i);
    const uint32_t wm = (f8 & (kBitNearWall | kBitOutletSrc)) ? g.wallmask[idx] : 0u;
    if ((f8 & kBitNearWall) && !g.wall_stream) {
        // bounce-back: f_i(x) = f_inv(i)^rec(x) when x - c_i is a wall (with
        // wall_stream the reference's 2D kernel is followed instead: it
        // overwrites that value with the ordinary pull, FsiCoupling2D.cu:
        // 171-224, since is_blocked is set only on the moving-wall path)
#pragma unroll
        for (int i = 1; i < 9; ++i)
            if (wm & (1u << i)) pop[i] = own(L::inv(i));
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) pop[i] = fmaxf(pop[i], 0.0f);
    float R[6], m[6];
    raw_moments2(pop, R);
    collide2(R, g.omega, m);
    if constexpr (IDX32) {
        encode_store_idx32<2, T>(m, g.dst, idx, g.ncell, g.codec);
    } else {
        T *planes[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) planes[k] = g.dst + (size_t)k * g.ncell;
        encode_store<2, T>(m, planes, idx, g.codec);
    }
    if (bad_state<2>(m)) atomicOr(g.status, kStatusNonFinite);
    if (f8 & kBitOutletSrc) {
        float ms[6];
        stored_values<2, T>(m, ms, idx, g.codec);
        feed_outlets<2, T>(g, idx, ms, wm);
    }
}

// Processes the TX x TY tile with lower-left cell (x0, y0) from the halo
// moments `raw` (dense2d_load).  The caller's CTA has TX * TY threads; sp is
// the CTA's population tile (tile + halo).  after_recon() runs once the halo
// is reconstructed and raw is no longer needed (a persistent caller loads its
// next tile there).
template <typename T, bool HALF, int TX, int TY, typename After>
__device__ __forceinline__ void dense2d_tile_loaded(const GridArgs<T> &g, int x0, int y0, float (*sp)[TY + 2][TX + 2],
                                                    const T (&raw)[Halo2<TX, TY>::kPer][6], After &&after_recon)
{
    using L = Lattice<2>;
    using H = Halo2<TX, TY>;
    const int tid = threadIdx.x;

    // 1. reconstruct the tile + halo (halo indices: halo_index).
#pragma unroll
    for (int r = 0; r < H::kPer; ++r) {
        const int c = tid + r * H::kThreads;
        if (c < H::kHalo) {
            const int hx = c % H::kHX, hy = c / H::kHX;
            float f[9];
            dense2d_recon<T, HALF>(g, raw[r], f);
#pragma unroll
            for (int i = 0; i < 9; ++i) sp[i][hy][hx] = f[i];
        }
    }
    after_recon();
    __syncthreads();

    const int tx = tid % TX, ty = tid / TX;
    const int x = x0 + tx, y = y0 + ty;
    if (x < g.nx && y < g.ny) {
        const uint32_t idx = (uint32_t)(y * g.nx + x);
        const uint8_t f8 = g.flags[idx];
        if (is_updated(f8 & kTypeMask) && !(f8 & kBitLink))
            dense2d_update_cell(
                g, idx, f8, [&](int i) { return sp[i][ty + 1 - L::cy(i)][tx + 1 - L::cx(i)]; },
                [&](int i) { return sp[i][ty + 1][tx + 1]; });
    }
}

// The tile with its own loads (the single-grid kernel).
template <typename T, bool HALF, int TX = D2::kTX, int TY = D2::kTY>
__device__ __forceinline__ void dense2d_tile(const GridArgs<T> &g, int x0, int y0, float (*sp)[TY + 2][TX + 2])
{
    T raw[Halo2<TX, TY>::kPer][6];
    dense2d_load<T, TX, TY>(g, x0, y0, raw);
    dense2d_tile_loaded<T, HALF, TX, TY>(g, x0, y0, sp, raw, [] {});
}

template <typename T> cudaError_t launch_dense2d(const GridArgs<T> &g, cudaStream_t s);

} // namespace fflbm
