// Fused D2Q9 step for all cells without moving-boundary links.
//
// Reference: mrDeformableSolver2DKernel_Shrd (src/core/FsiCoupling2D.cu:82-255)
// followed by mrApplyOutlet2DKernel (:257-316).
//
// One CTA = one 32 x 8 tile.  The CTA reconstructs the populations of the
// tile plus a one-cell halo (34 x 10 cells) from their moments into shared
// memory, then every thread pulls its nine incoming populations, applies
// bounce-back for wall neighbours (precomputed per-cell mask), forms the raw
// moments, collides and stores the new moments.  Moments live in HBM as SoA
// planes (coalesced 128 B per warp per moment); populations never leave the
// SM.  Outlet writes are issued by the outlet's feeding cell (ffs_outlet.cuh),
// so the step is one launch.  D2Q9 grids of the sizes FreeFlow runs (<= 1200
// x 400) are L2-resident on B200, so this kernel is bound by issue rate and
// launch latency rather than HBM; the batched variant (ffs_batch2d.cu)
// amortises launches over many grids.
#include "ffs_dense2d.cuh"

namespace fflbm {

template <typename T, bool HALF>
__global__ void __launch_bounds__(D2::kThreads) dense2d_kernel(GridArgs<T> g)
{
    __shared__ float sp[9][D2::kHY][D2::kHX];
    dense2d_tile<T, HALF>(g, blockIdx.x * D2::kTX, blockIdx.y * D2::kTY, sp);
}

template <typename T>
cudaError_t launch_dense2d(const GridArgs<T> &g, cudaStream_t s)
{
    dim3 grid((g.nx + D2::kTX - 1) / D2::kTX, (g.ny + D2::kTY - 1) / D2::kTY);
    if (g.half_pops)
        dense2d_kernel<T, true><<<grid, D2::kThreads, 0, s>>>(g);
    else
        dense2d_kernel<T, false><<<grid, D2::kThreads, 0, s>>>(g);
    return cudaGetLastError();
}

template cudaError_t launch_dense2d<float>(const GridArgs<float> &, cudaStream_t);
template cudaError_t launch_dense2d<__half>(const GridArgs<__half> &, cudaStream_t);
template cudaError_t launch_dense2d<__nv_bfloat16>(const GridArgs<__nv_bfloat16> &, cudaStream_t);

} // namespace fflbm
