#pragma once
#include "ffs_common.cuh"

namespace fflbm {

// Tile geometry of the z-marching D3Q27 kernel (ffs_dense3d.cu).
struct D3 {
    static constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
    static constexpr int kHX = kTX + 2, kHY = kTY + 2, kHalo = kHX * kHY;
    static constexpr int kRing = kHalo - kTX * kTY;           // halo cells outside the tile (84)
    static constexpr int kPlaneFloats = 27 * kHalo;           // all populations of one halo plane
    static constexpr size_t kSmemBytes = 2 * (size_t)kPlaneFloats * sizeof(float); // double buffer
};
static_assert(D3::kRing <= D3::kThreads, "every ring cell needs a partner thread");

// variant: 0 = two CTAs per SM (no spills), 1 = three CTAs per SM, 2 = two
// CTAs per SM with the paired shared-memory layout and packed c_z = -1 / +1
// arithmetic (a three-CTA build of it spills and ran 40 % slower), 3 = the
// same with each halo plane's moments staged in shared memory by TMA copies
// two planes ahead (grids whose rows of moments are not a multiple of 16
// bytes run 2; on 384 x 192 x 192 it ran 5 % slower than 2, so the tuner
// keeps 2 there).  All
// round identically; the first step times them, variant 2 first, and keeps
// another only if it is at least 1 % faster (FFS_DENSE3D_VARIANT pins one).
constexpr int kDense3dVariants = 4;
template <typename T> cudaError_t launch_dense3d(const GridArgs<T> &g, cudaStream_t s, int variant);
template <typename T> int tune_dense3d(const GridArgs<T> &g, cudaStream_t s);

} // namespace fflbm
