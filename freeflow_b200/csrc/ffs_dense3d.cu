// Fused D3Q27 step for all cells without moving-boundary links.
//
// Reference: mrDeformableSolver3DKernel_ShrdM (src/core/FsiCoupling3D.cu:83-334)
// followed by mrApplyOutlet3DKernel (:336-420).
//
// B200 design.  The reference gives each 8x4x4 block a 10x6x6 halo and
// reconstructs all 27 populations of every halo cell (2.8x the interior),
// then pulls them back out of shared memory.  Here a CTA owns a 32 x 8 column
// of cells and marches up z through a chunk of planes:
//
//   * each plane is reconstructed once, for its 34 x 10 xy halo (1.33x the
//     interior), by 170 threads that handle two halo cells each with packed
//     FP32-pair arithmetic (add/fma.rn.f32x2), into one of two shared-memory
//     buffers (2 x 27 x 340 floats = 72 KB, three CTAs per SM);
//   * every population of plane p is consumed as soon as the plane exists:
//     the c_z = -1 slice completes the raw moments of the cell below (plane
//     p-1), the c_z = 0 slice feeds plane p, the c_z = +1 slice starts plane
//     p+1.  Each thread keeps the partial raw moments of its column's next two
//     cells in registers, so a plane is read once, one barrier per plane;
//   * moments are SoA planes in HBM (128 B coalesced per warp and moment);
//     the next plane's moments and flag bytes are prefetched into registers
//     while the current plane is processed;
//   * wall neighbours are a per-cell bit mask, applied only to cells flagged
//     near-wall (an exact correction of the pulled population by the
//     bounce-back one), outlets are fed by their inner neighbour in the same
//     pass, and cells with moving-boundary links are left to the sparse link
//     kernel (ffs_links.cu).
#include "ffs_dense2d.cuh"
#include "ffs_dense3d.cuh"

namespace fflbm {

namespace {
constexpr int kTX = D3::kTX, kTY = D3::kTY, kHX = D3::kHX, kHalo = D3::kHalo, kHalf = D3::kHalf;
constexpr int kPlane = D3::kPlaneFloats;

// raw-moment slot of M_pqr: {rho, jx, jy, jz, Pxx, Pyy, Pzz, Pxy, Pyz, Pxz}
// 9 populations of one c_z slice (f[ky][kx], clamped) -> the six x/y moments
// Y = {Y00, Y01, Y02, Y10, Y11, Y20}
__device__ __forceinline__ void slice_sums(const float *buf, int kz, int tx, int ty, float *Y)
{
    float X0[3], X1[3], X2[3];
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
        const float *row = buf + ((kz * 3 + ky) * 3) * kHalo + (ty + 2 - ky) * kHX + tx;
        float fm = fmaxf(row[0 * kHalo + 2], 0.0f); // kx = 0 (c_x = -1): source x + 1
        float f0 = fmaxf(row[1 * kHalo + 1], 0.0f); // kx = 1
        float fp = fmaxf(row[2 * kHalo + 0], 0.0f); // kx = 2 (c_x = +1): source x - 1
        float s = fp + fm;
        X1[ky] = fp - fm;
        X0[ky] = f0 + s;
        X2[ky] = s;
    }
    float s0 = X0[2] + X0[0];
    Y[0] = X0[1] + s0;
    Y[1] = X0[2] - X0[0];
    Y[2] = s0;
    Y[3] = X1[1] + (X1[2] + X1[0]);
    Y[4] = X1[2] - X1[0];
    Y[5] = X2[1] + (X2[2] + X2[0]);
}

// add a slice with velocity component c_z to the raw moments R
template <int CZ> __device__ __forceinline__ void slice_add(float *R, const float *Y)
{
    R[0] += Y[0]; R[2] += Y[1]; R[5] += Y[2]; R[1] += Y[3]; R[7] += Y[4]; R[4] += Y[5];
    if (CZ != 0) {
        R[3] += CZ * Y[0]; R[6] += Y[0]; R[8] += CZ * Y[1]; R[9] += CZ * Y[3];
    }
}
// start R from a c_z = +1 slice
__device__ __forceinline__ void slice_init_plus(float *R, const float *Y)
{
    R[0] = Y[0]; R[2] = Y[1]; R[5] = Y[2]; R[1] = Y[3]; R[7] = Y[4]; R[4] = Y[5];
    R[3] = Y[0]; R[6] = Y[0]; R[8] = Y[1]; R[9] = Y[3];
}
} // namespace

// Replace, in the raw moments R of near-wall cell (x, y, z), every population
// pulled from a bounce-back neighbour by the reflected population of the cell
// itself (FsiCoupling3D.cu:209-222): R += basis(c_i) (max(0, f_inv(i)^rec(x)) -
// max(0, f_i^rec(x - c_i))), the second term being what the slice pass added.
template <typename T>
__device__ __noinline__ void wall_correct(const GridArgs<T> &g, float *R, int x, int y, int z, uint32_t idx)
{
    const uint32_t wm = g.wallmask[idx];
    const long long nxy = (long long)g.nx * g.ny;
    const bool wx = g.periodic & 1, wy = g.periodic & 2, wz = g.periodic & 4;
    float m[10];
    load_moments<3, T>(m, g.src, g.ncell, idx, g.codec);
    Coef<3> own;
    own.make(m);
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                if (!(wm & (1u << dir_index<3>(kx, ky, kz)))) continue;
                const int cx = kx - 1, cy = ky - 1, cz = kz - 1;
                const int sx = halo_index(x - cx, g.nx, wx), sy = halo_index(y - cy, g.ny, wy);
                const int sz = halo_index(z - cz, g.nz, wz);
                float mn[10];
                load_moments<3, T>(mn, g.src, g.ncell, (uint32_t)(sz * nxy + (long long)sy * g.nx + sx), g.codec);
                Coef<3> nb;
                nb.make(mn);
                const float d = fmaxf(own.population(-cx, -cy, -cz), 0.0f) - fmaxf(nb.population(cx, cy, cz), 0.0f);
                R[0] += d;
                R[1] += cx * d; R[2] += cy * d; R[3] += cz * d;
                R[4] += cx * cx * d; R[5] += cy * cy * d; R[6] += cz * cz * d;
                R[7] += cx * cy * d; R[8] += cy * cz * d; R[9] += cx * cz * d;
            }
}

// MINB = CTAs per SM the register budget is cut for: 3 (80 registers, a few
// spills) or 2 (no spills); launch_dense3d times both on the grid and keeps
// the faster (tune_dense3d).
template <typename T, int MINB>
__global__ void __launch_bounds__(D3::kThreads, MINB) dense3d_kernel(GridArgs<T> g, int zchunk)
{
    extern __shared__ float smem[];
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, g.nz);
    const long long nxy = (long long)g.nx * g.ny;
    const bool wx = g.periodic & 1, wy = g.periodic & 2, wz = g.periodic & 4;

    // reconstruction role: threads 0..169 own halo cells tid and tid + 170
    const bool rec = tid < kHalf;
    auto planar = [&](int c) {
        int hx = c % kHX, hy = c / kHX;
        return (uint32_t)(halo_index(y0 + hy - 1, g.ny, wy) * g.nx + halo_index(x0 + hx - 1, g.nx, wx));
    };
    const uint32_t off0 = rec ? planar(tid) : 0u, off1 = rec ? planar(tid + kHalf) : 0u;
    float mA[10], mB[10];
    auto load_plane = [&](int z) {
        if (!rec) return;
        const T *base = g.src + (size_t)halo_index(z, g.nz, wz) * nxy;
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            mA[k] = StorageTraits<T>::from(base[(size_t)k * g.ncell + off0]);
            mB[k] = StorageTraits<T>::from(base[(size_t)k * g.ncell + off1]);
        }
    };
    auto recon_plane = [&](float *buf) {
        if (!rec) return;
        decode_moments<3, T>(mA, g.codec);
        decode_moments<3, T>(mB, g.codec);
        f2 m[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) m[k] = f2make(mA[k], mB[k]);
        Coef3V<f2> cf;
        cf.make(m);
        cf.populations_each([&](int kz, int ky, int kx, f2 v) {
            float a, b;
            f2split(v, a, b);
            float *set = buf + ((kz * 3 + ky) * 3 + kx) * kHalo;
            set[tid] = a;
            set[tid + kHalf] = b;
        });
    };

    const int tx = tid % kTX, ty = tid / kTX;
    const int x = x0 + tx, y = y0 + ty;
    const bool inside = x < g.nx && y < g.ny;
    const uint32_t col = inside ? (uint32_t)(y * g.nx + x) : 0u;

    float Ap[10], Ac[10];  // partial raw moments of the cells at z = p-1 and z = p
    uint8_t fp = 0, fc = 0; // their flag bytes
#pragma unroll
    for (int k = 0; k < 10; ++k) Ap[k] = Ac[k] = 0.0f;

    load_plane(zb - 1);
    for (int p = zb - 1; p <= ze; ++p) {
        float *buf = smem + (p & 1) * kPlane;
        recon_plane(buf);
        if (p < ze) load_plane(p + 1);
        uint8_t fn = 0;
        if (inside && p + 1 < ze) fn = g.flags[(size_t)(p + 1) * nxy + col];
        __syncthreads();
        if (inside) {
            float Y[6];
            // c_z = -1 slice completes the cell at z = p - 1
            slice_sums(buf, 0, tx, ty, Y);
            slice_add<-1>(Ap, Y);
            const int d = p - 1;
            if (d >= zb && is_updated(fp & kTypeMask) && !(fp & kBitLink)) {
                const uint32_t idx = (uint32_t)(d * nxy + col);
                if (fp & kBitNearWall) wall_correct<T>(g, Ap, x, y, d, idx);
                float m[10];
                collide3(Ap, g.omega, m);
                encode_store_strided<3, T>(m, g.dst + idx, g.ncell, g.codec);
                if (bad_state<3>(m)) atomicOr(g.status, kStatusNonFinite);
                if (fp & kBitOutletSrc) feed_outlets<3, T>(g, idx);
            }
            // c_z = 0 slice feeds z = p; c_z = +1 slice starts z = p + 1
            slice_sums(buf, 1, tx, ty, Y);
            slice_add<0>(Ac, Y);
#pragma unroll
            for (int k = 0; k < 10; ++k) Ap[k] = Ac[k];
            slice_sums(buf, 2, tx, ty, Y);
            slice_init_plus(Ac, Y);
            fp = fc;
            fc = fn;
        }
    }
}

// Number of z chunks that best fills the GPU: whole waves of CTAs, with the
// two extra planes each chunk reconstructs counted as overhead.
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

template <typename T, int MINB> struct Dense3dLaunch {
    static cudaError_t run(const GridArgs<T> &g, cudaStream_t s)
    {
        static bool configured = false;
        static int slots = 0;
        if (!configured) {
            cudaError_t e = cudaFuncSetAttribute(dense3d_kernel<T, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)D3::kSmemBytes);
            if (e != cudaSuccess) return e;
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dense3d_kernel<T, MINB>, D3::kThreads, D3::kSmemBytes);
            slots = sms * (per_sm > 0 ? per_sm : 1);
            configured = true;
        }
        int tx = (g.nx + kTX - 1) / kTX, ty = (g.ny + kTY - 1) / kTY;
        int nchunk = choose_zchunks(tx * ty, g.nz, slots);
        int zchunk = (g.nz + nchunk - 1) / nchunk;
        dim3 grid(tx, ty, (g.nz + zchunk - 1) / zchunk);
        dense3d_kernel<T, MINB><<<grid, D3::kThreads, D3::kSmemBytes, s>>>(g, zchunk);
        return cudaGetLastError();
    }
};

template <typename T>
cudaError_t launch_dense3d(const GridArgs<T> &g, cudaStream_t s, int variant)
{
    return variant == 1 ? Dense3dLaunch<T, 3>::run(g, s) : Dense3dLaunch<T, 2>::run(g, s);
}

// Times each variant on this grid (the pass only reads src and writes dst, so
// repeating it is harmless) and returns the faster one.
template <typename T>
int tune_dense3d(const GridArgs<T> &g, cudaStream_t s)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    int best_v = 0;
    for (int v = 0; v < 2; ++v) {
        if (launch_dense3d<T>(g, s, v) != cudaSuccess) continue;  // warm-up
        cudaEventRecord(a, s);
        for (int r = 0; r < 3; ++r) launch_dense3d<T>(g, s, v);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) { best = ms; best_v = v; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best_v;
}

template cudaError_t launch_dense3d<float>(const GridArgs<float> &, cudaStream_t, int);
template cudaError_t launch_dense3d<__half>(const GridArgs<__half> &, cudaStream_t, int);
template cudaError_t launch_dense3d<__nv_bfloat16>(const GridArgs<__nv_bfloat16> &, cudaStream_t, int);
template int tune_dense3d<float>(const GridArgs<float> &, cudaStream_t);
template int tune_dense3d<__half>(const GridArgs<__half> &, cudaStream_t);
template int tune_dense3d<__nv_bfloat16>(const GridArgs<__nv_bfloat16> &, cudaStream_t);

} // namespace fflbm
