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

// Source index of a halo cell: clamped like the reference's min/max
// (FsiCoupling2D.cu:104-105, FsiCoupling3D.cu:106-108) or wrapped for a
// periodic axis.  v >= -1 always; v may exceed n by a tile width.
__device__ __forceinline__ int halo_index(int v, int n, bool wrap)
{
    if (!wrap) return v < 0 ? 0 : (v >= n ? n - 1 : v);
    if (v < 0) v += n;
    if (v >= n) v -= n;
    if (v >= n) v %= n;
    return v;
}

// Processes the TX x TY tile with lower-left cell (x0, y0).  The caller's
// CTA has TX * TY threads; sp is the CTA's population tile (tile + halo).
template <typename T, bool HALF, int TX = D2::kTX, int TY = D2::kTY>
__device__ __forceinline__ void dense2d_tile(const GridArgs<T> &g, int x0, int y0, float (*sp)[TY + 2][TX + 2])
{
    using L = Lattice<2>;
    constexpr int kHX = TX + 2, kHalo = (TX + 2) * (TY + 2), kThreads = TX * TY;
    const int tid = threadIdx.x;
    const bool wx = g.periodic & 1, wy = g.periodic & 2;

    // 1. reconstruct the tile + halo.  The halo index is clamped (the
    //    reference's min/max, FsiCoupling2D.cu:104-105) or wrapped (periodic).
    for (int c = tid; c < kHalo; c += kThreads) {
        int hx = c % kHX, hy = c / kHX;
        int gx = halo_index(x0 + hx - 1, g.nx, wx);
        int gy = halo_index(y0 + hy - 1, g.ny, wy);
        float m[6];
        load_moments<2, T>(m, g.src, g.ncell, (uint32_t)(gy * g.nx + gx), g.codec);
        Coef<2> cf;
        cf.make(m);
        float f[9];
        cf.populations(f);
#pragma unroll
        for (int i = 0; i < 9; ++i) sp[i][hy][hx] = HALF ? round_half(f[i]) : f[i];
    }
    __syncthreads();

    const int tx = tid % TX, ty = tid / TX;
    const int x = x0 + tx, y = y0 + ty;
    if (x < g.nx && y < g.ny) {
        const uint32_t idx = (uint32_t)(y * g.nx + x);
        const uint8_t f8 = g.flags[idx];
        if (is_updated(f8 & kTypeMask) && !(f8 & kBitLink)) {
            float pop[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) pop[i] = sp[i][ty + 1 - L::cy(i)][tx + 1 - L::cx(i)];
            const uint32_t wm = (f8 & (kBitNearWall | kBitOutletSrc)) ? g.wallmask[idx] : 0u;
            if (f8 & kBitNearWall) {
                // bounce-back: f_i(x) = f_inv(i)^rec(x) when x - c_i is a wall
#pragma unroll
                for (int i = 1; i < 9; ++i)
                    if (wm & (1u << i)) pop[i] = sp[L::inv(i)][ty + 1][tx + 1];
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) pop[i] = fmaxf(pop[i], 0.0f);
            float R[6], m[6];
            raw_moments2(pop, R);
            collide2(R, g.omega, m);
            T *planes[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) planes[k] = g.dst + (size_t)k * g.ncell;
            encode_store<2, T>(m, planes, idx, g.codec);
            if (bad_state<2>(m)) atomicOr(g.status, kStatusNonFinite);
            if (f8 & kBitOutletSrc) {
                float ms[6];
                stored_values<2, T>(m, ms, g.codec);
                feed_outlets<2, T>(g, idx, ms, wm);
            }
        }
    }
}

template <typename T> cudaError_t launch_dense2d(const GridArgs<T> &g, cudaStream_t s);

} // namespace fflbm
