// Fused D3Q27 step for all cells without moving-boundary links.
//
// Reference: mrDeformableSolver3DKernel_ShrdM (src/core/FsiCoupling3D.cu:83-334)
// followed by mrApplyOutlet3DKernel (:336-420).
//
// B200 design.  The reference gives each 8x4x4 block a 10x6x6 halo and
// reconstructs all 27 populations of every halo cell (2.8x the interior),
// and reads AoS moments with a 40 B stride.  Here a CTA owns a 32 x 8
// column of cells and marches up z through a chunk of planes:
//
//   * each plane is reconstructed once, for its 34 x 10 xy halo (1.33x);
//   * the 27 populations of a plane split into three 9-population slices by
//     c_z: the c_z = -1 slice is consumed by the plane below at once, the
//     c_z = 0 slice by the plane itself one iteration later, the c_z = +1
//     slice by the plane above two iterations later.  Shared memory holds
//     one c_z=-1, two c_z=0 and three c_z=+1 slices (72 KB), so two CTAs fit
//     per SM;
//   * moments are SoA planes in HBM: every warp load/store is 128 B
//     coalesced; the next plane's moments are prefetched into registers
//     while the current plane is processed;
//   * wall neighbours are a per-cell bit mask read only for near-wall cells,
//     outlets are fed by their inner neighbour in the same pass, and cells
//     with moving-boundary links are skipped here and finished by the sparse
//     link kernel (ffs_links.cu).
#include "ffs_dense2d.cuh"
#include "ffs_dense3d.cuh"

namespace fflbm {

namespace {
constexpr int kTX = D3::kTX, kTY = D3::kTY, kHX = D3::kHX, kHalo = D3::kHalo, kSet = D3::kSetFloats;

__device__ __forceinline__ int mod3(int z) { return ((z % 3) + 3) % 3; }
} // namespace

template <typename T>
__global__ void __launch_bounds__(D3::kThreads, 2) dense3d_kernel(GridArgs<T> g, int zchunk)
{
    extern __shared__ float smem[];
    float *sMinus = smem;
    float *sZero0 = smem + kSet, *sZero1 = smem + 2 * kSet;
    float *sPlus0 = smem + 3 * kSet;

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, g.nz);
    const long long nxy = (long long)g.nx * g.ny;
    const bool wx = g.periodic & 1, wy = g.periodic & 2, wz = g.periodic & 4;

    // the (up to) two halo cells this thread reconstructs
    const int c0 = tid, c1 = tid + D3::kThreads;
    const bool has1 = c1 < kHalo;
    auto planar = [&](int c) {
        int hx = c % kHX, hy = c / kHX;
        int gx = halo_index(x0 + hx - 1, g.nx, wx);
        int gy = halo_index(y0 + hy - 1, g.ny, wy);
        return (uint32_t)(gy * g.nx + gx);
    };
    const uint32_t off0 = planar(c0), off1 = has1 ? planar(c1) : 0u;
    auto zsrc = [&](int z) { return halo_index(z, g.nz, wz); };

    float mA[10], mB[10];
    auto load_plane = [&](int z) {
        const size_t pb = (size_t)zsrc(z) * nxy;
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            const T *pl = g.src + (size_t)k * g.ncell + pb;
            mA[k] = StorageTraits<T>::from(pl[off0]);
            if (has1) mB[k] = StorageTraits<T>::from(pl[off1]);
        }
    };
    auto recon_cell = [&](float *m, int c, float *minus, float *zero, float *plus) {
        decode_moments<3, T>(m, g.codec);
        Coef<3> cf;
        cf.make(m);
        float o[3][3][3];
        cf.populations_xyz(o);
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            if (minus) minus[j * kHalo + c] = o[0][j / 3][j % 3];
            if (zero) zero[j * kHalo + c] = o[1][j / 3][j % 3];
            if (plus) plus[j * kHalo + c] = o[2][j / 3][j % 3];
        }
    };
    auto recon_plane = [&](float *minus, float *zero, float *plus) {
        recon_cell(mA, c0, minus, zero, plus);
        if (has1) recon_cell(mB, c1, minus, zero, plus);
    };
    auto plus_slot = [&](int z) { return sPlus0 + mod3(z) * kSet; };
    auto zero_slot = [&](int z) { return (z & 1) ? sZero1 : sZero0; };

    // prologue: c_z=+1 slice of plane zb-1, c_z=0 and c_z=+1 slices of plane zb
    load_plane(zb - 1);
    recon_plane(nullptr, nullptr, plus_slot(zb - 1));
    load_plane(zb);
    recon_plane(nullptr, zero_slot(zb), plus_slot(zb));
    load_plane(zb + 1);

    const int tx = tid % kTX, ty = tid / kTX;
    const int x = x0 + tx, y = y0 + ty;
    const bool inside = x < g.nx && y < g.ny;

    for (int z = zb; z < ze; ++z) {
        recon_plane(sMinus, zero_slot(z + 1), plus_slot(z + 1));
        if (z + 1 < ze) load_plane(z + 2);
        __syncthreads();

        if (inside) {
            const uint32_t idx = (uint32_t)(z * nxy + (long long)y * g.nx + x);
            const uint8_t f8 = g.flags[idx];
            if (is_updated(f8 & kTypeMask) && !(f8 & kBitLink)) {
                const float *sP = plus_slot(z - 1), *sZ = zero_slot(z);
                float F[3][3][3]; // F[kz][ky][kx], k = c + 1
#pragma unroll
                for (int kz = 0; kz < 3; ++kz)
#pragma unroll
                    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
                        for (int kx = 0; kx < 3; ++kx) {
                            const float *set = kz == 2 ? sP : (kz == 1 ? sZ : sMinus);
                            const int c = (ty + 2 - ky) * kHX + (tx + 2 - kx);
                            F[kz][ky][kx] = set[(ky * 3 + kx) * kHalo + c];
                        }
                if (f8 & kBitNearWall) {
                    // bounce-back: f_i(x) = f_inv(i)^rec(x) for wall neighbours x - c_i
                    const uint32_t wm = g.wallmask[idx];
                    float m[10];
                    load_moments<3, T>(m, g.src, g.ncell, idx, g.codec);
                    Coef<3> own;
                    own.make(m);
#pragma unroll
                    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
                        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
                            for (int kx = 0; kx < 3; ++kx)
                                if (wm & (1u << dir_index<3>(kx, ky, kz)))
                                    F[kz][ky][kx] = own.population(1 - kx, 1 - ky, 1 - kz);
                }
#pragma unroll
                for (int kz = 0; kz < 3; ++kz)
#pragma unroll
                    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
                        for (int kx = 0; kx < 3; ++kx) F[kz][ky][kx] = fmaxf(F[kz][ky][kx], 0.0f);
                float R[10], m[10];
                raw_moments3(F, R);
                collide3(R, g.omega, m);
                T *planes[10];
#pragma unroll
                for (int k = 0; k < 10; ++k) planes[k] = g.dst + (size_t)k * g.ncell;
                encode_store<3, T>(m, planes, idx, g.codec);
                if (!isfinite(m[0])) atomicOr(g.status, kStatusNonFinite);
                if (f8 & kBitOutletSrc) feed_outlets<3, T>(g, idx);
            }
        }
        __syncthreads();
    }
}

// Number of z chunks that best fills the GPU: whole waves of CTAs, with the
// two prologue planes per chunk counted as overhead.
static int choose_zchunks(int tiles, int nz, int slots)
{
    int best = 1;
    double best_eff = 0.0;
    for (int n = 1; n <= 16 && n <= nz; ++n) {
        int chunk = (nz + n - 1) / n;
        long long ctas = (long long)tiles * ((nz + chunk - 1) / chunk);
        long long waves = (ctas + slots - 1) / slots;
        double eff = (double)ctas / (double)(waves * slots) * (double)chunk / (double)(chunk + 2);
        if (eff > best_eff + 1e-9) { best_eff = eff; best = n; }
    }
    return best;
}

template <typename T>
cudaError_t launch_dense3d(const GridArgs<T> &g, cudaStream_t s)
{
    static bool configured = false;
    static int slots = 0;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(dense3d_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D3::kSmemBytes);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dense3d_kernel<T>, D3::kThreads, D3::kSmemBytes);
        slots = sms * (per_sm > 0 ? per_sm : 1);
        configured = true;
    }
    int tx = (g.nx + kTX - 1) / kTX, ty = (g.ny + kTY - 1) / kTY;
    int nchunk = choose_zchunks(tx * ty, g.nz, slots);
    int zchunk = (g.nz + nchunk - 1) / nchunk;
    dim3 grid(tx, ty, (g.nz + zchunk - 1) / zchunk);
    dense3d_kernel<T><<<grid, D3::kThreads, D3::kSmemBytes, s>>>(g, zchunk);
    return cudaGetLastError();
}

template cudaError_t launch_dense3d<float>(const GridArgs<float> &, cudaStream_t);
template cudaError_t launch_dense3d<__half>(const GridArgs<__half> &, cudaStream_t);
template cudaError_t launch_dense3d<__nv_bfloat16>(const GridArgs<__nv_bfloat16> &, cudaStream_t);

} // namespace fflbm
