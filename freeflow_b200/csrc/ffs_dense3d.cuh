#pragma once
#include "ffs_common.cuh"

namespace fflbm {

// Tile geometry of the z-marching D3Q27 kernel (ffs_dense3d.cu).
struct D3 {
    static constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
    static constexpr int kHX = kTX + 2, kHY = kTY + 2, kHalo = kHX * kHY;
    static constexpr int kSetFloats = 9 * kHalo; // one 9-population c_z slice of one plane
    // one c_z=-1 slice, two c_z=0 slices, three c_z=+1 slices
    static constexpr size_t kSmemBytes = 6 * (size_t)kSetFloats * sizeof(float);
};

template <typename T> cudaError_t launch_dense3d(const GridArgs<T> &g, cudaStream_t s);

} // namespace fflbm
