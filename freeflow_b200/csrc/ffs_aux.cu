// Grid set-up kernels: derived flag bits, initial state, solid fill and the
// moment layout / precision conversions used by the C ABI.
#include <algorithm>

#include "ffs_common.cuh"
#include "ffs_geom.cuh"
#include "ffs_links.cuh"
#include "ffs_outlet.cuh"

namespace fflbm {

namespace {
__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

template <int DIM> __device__ __forceinline__ void dir3(int i, int &cx, int &cy, int &cz)
{
    cx = Lattice<DIM>::cx(i); cy = Lattice<DIM>::cy(i); cz = Lattice<DIM>::cz(i);
}
} // namespace

// Per cell: the bounce-back mask (bit i set when the wrapped neighbour
// x - c_i is a wall type, as the reference tests every step at
// FsiCoupling2D.cu:159-176 / FsiCoupling3D.cu:199-216), NEAR_WALL when the
// mask is non-zero, and OUTLET_SRC when the cell is the Fluid feeder of an
// outlet node.  Node types are static between flag uploads, so this runs
// once per upload instead of every step.
template <int DIM>
__global__ void prepare_flags_kernel(uint8_t *flags, uint32_t *wallmask, int nx, int ny, int nz)
{
    constexpr int Q = Lattice<DIM>::Q;
    const long long nxy = (long long)nx * ny, n = nxy * nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / nxy);
        const uint32_t t = flags[c] & kTypeMask;
        uint32_t mask = 0;
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            int cx, cy, cz;
            dir3<DIM>(i, cx, cy, cz);
            long long ib = ((long long)wrapi(z - cz, nz) * ny + wrapi(y - cy, ny)) * nx + wrapi(x - cx, nx);
            if (is_bounce_back<DIM>(flags[ib] & kTypeMask)) mask |= 1u << i;
        }
        uint8_t bits = (uint8_t)t;
        if (mask) bits |= kBitNearWall;
        if (t == kFluid) {
            for (int r = 0; r < kNumOutletRules<DIM>; ++r) {
                long long q = c + outlet_offset<DIM>(r, nx, nxy);
                if (q >= 0 && q < n && (flags[q] & kTypeMask) == outlet_rule<DIM>(r).type) {
                    bits |= kBitOutletSrc;
                    mask |= outlet_bit<DIM>(r);
                }
            }
        }
        wallmask[c] = mask;
        flags[c] = bits; // neighbours only read the type bits, which do not change
    }
}

template <int DIM>
cudaError_t launch_prepare_flags(uint8_t *flags, uint32_t *wallmask, int nx, int ny, int nz, cudaStream_t st)
{
    long long n = (long long)nx * ny * nz;
    int grid = (int)std::min<long long>((n + 255) / 256, (long long)device_sms() * 16);
    prepare_flags_kernel<DIM><<<grid, 256, 0, st>>>(flags, wallmask, nx, ny, nz);
    return cudaGetLastError();
}
template cudaError_t launch_prepare_flags<2>(uint8_t *, uint32_t *, int, int, int, cudaStream_t);
template cudaError_t launch_prepare_flags<3>(uint8_t *, uint32_t *, int, int, int, cudaStream_t);

// initialize_state_kernel_2d/3d (LbmInitializer2D.cu:32-95,
// LbmInitializer3D.cu:33-113): rho = 1, u set on inlet nodes from the
// boundary velocities, equilibrium stress pi_ab = u_a u_b (the second moments
// of the reference's second-order feq, evaluated exactly), both buffers.
template <int DIM, typename T>
__global__ void initialize_kernel(GridArgs<T> g, T *other, Vel6 bc)
{
    constexpr int NM = Lattice<DIM>::NM;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell; c += (long long)gridDim.x * blockDim.x) {
        const uint32_t t = g.flags[c] & kTypeMask;
        float u[3] = {0.0f, 0.0f, 0.0f};
        if (DIM == 2) {
            if (t == kInletLeft) u[0] = bc.v[0];
            else if (t == kInletDown) u[1] = bc.v[1];
            else if (t == kInletRight) u[0] = -bc.v[2];
            else if (t == kInletUp) u[1] = -bc.v[3];
        } else {
            if (t == kInletLeft) u[0] = bc.v[0];
            else if (t == kInletDown) u[2] = bc.v[1];
            else if (t == kInletRight) u[0] = -bc.v[2];
            else if (t == kInletUp) u[2] = -bc.v[3];
            else if (t == kInletFront) u[1] = bc.v[4];
            else if (t == kInletBack) u[1] = -bc.v[5];
        }
        float m[NM];
        m[0] = 1.0f;
        for (int a = 0; a < DIM; ++a) m[1 + a] = u[a];
        for (int k = DIM + 1; k < NM; ++k) m[k] = u[MomentLayout<DIM>::pa(k)] * u[MomentLayout<DIM>::pb(k)];
        T *pa[NM], *pb[NM];
        for (int k = 0; k < NM; ++k) { pa[k] = g.dst + (size_t)k * g.ncell; pb[k] = other + (size_t)k * g.ncell; }
        encode_store<DIM, T>(m, pa, (uint32_t)c, g.codec);
        encode_store<DIM, T>(m, pb, (uint32_t)c, g.codec);
    }
}

template <int DIM, typename T>
cudaError_t launch_initialize(const GridArgs<T> &g, T *other, const float *bcvel, cudaStream_t st)
{
    Vel6 bc;
    for (int i = 0; i < 6; ++i) bc.v[i] = bcvel[i];
    int grid = (int)std::min<long long>(((long long)g.ncell + 255) / 256, (long long)device_sms() * 16);
    initialize_kernel<DIM, T><<<grid, 256, 0, st>>>(g, other, bc);
    return cudaGetLastError();
}

// fillSolidFlags2D (FsiCoupling2D.cu:318-354, 434-464): a Fluid or
// SolidDynamic cell becomes SolidDynamic when its centre is inside the closed
// polygon, Fluid otherwise.  The reference tests every cell against every edge
// (crossing-number parity, SolidGeometryProxy_Device.cuh:126-144).  Here one
// warp takes one row: the crossing abscissae of the row's scanline with the
// edges are computed once per row, with the same explicitly rounded
// operations as the reference's per-cell expression, and each cell's parity
// is the number of crossings to its right.  Every operation is explicitly
// rounded, so the mask is bit-identical to the per-cell test (and to the CPU
// oracle); a row with more crossings than fit in shared memory falls back to
// the per-cell test.
constexpr int kFillCrossings = 256;

__global__ void __launch_bounds__(256) fill_solid2_kernel(uint8_t *flags, int nx, int ny, float cl, SurfaceArgs s)
{
    using namespace geom;
    __shared__ float xs_all[8][kFillCrossings];
    float *xs = xs_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int y = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); y < ny; y += nwarps) {
        const float py = mul(add((float)y, 0.5f), cl);
        int count = 0;
        for (int i0 = 0; i0 < s.ne; i0 += 32) {
            const int i = i0 + lane;
            bool cross = false;
            float xc = 0.0f;
            if (i < s.ne && s.E[2 * i] < (uint32_t)s.nv && s.E[2 * i + 1] < (uint32_t)s.nv) {
                const uint32_t a = s.E[2 * i], b = s.E[2 * i + 1];
                const float sx = s.V[2 * a], sy = s.V[2 * a + 1], tx = s.V[2 * b], ty = s.V[2 * b + 1];
                if ((sy < py && ty >= py) || (sy >= py && ty < py)) {
                    cross = true;
                    xc = add(sx, dvd(mul(sub(py, sy), sub(tx, sx)), sub(ty, sy)));
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, cross);
            const int pos = count + __popc(m & below);
            if (cross && pos < kFillCrossings) xs[pos] = xc;
            count += __popc(m);
        }
        __syncwarp();
        for (int x = lane; x < nx; x += 32) {
            const size_t c = (size_t)y * nx + x;
            const uint32_t t = flags[c] & kTypeMask;
            if (t != kFluid && t != kSolidDynamic) continue;
            const float px = mul(add((float)x, 0.5f), cl);
            bool in = false;
            if (count <= kFillCrossings) {
                for (int k = 0; k < count; ++k) in ^= (xs[k] > px);
            } else {
                for (int i = 0; i < s.ne; ++i) {
                    const uint32_t a = s.E[2 * i], b = s.E[2 * i + 1];
                    if (a >= (uint32_t)s.nv || b >= (uint32_t)s.nv) continue;
                    const float sx = s.V[2 * a], sy = s.V[2 * a + 1], tx = s.V[2 * b], ty = s.V[2 * b + 1];
                    if ((sy < py && ty >= py) || (sy >= py && ty < py))
                        in ^= (add(sx, dvd(mul(sub(py, sy), sub(tx, sx)), sub(ty, sy))) > px);
                }
            }
            flags[c] = in ? kSolidDynamic : kFluid;
        }
        __syncwarp();
    }
}

cudaError_t launch_fill_solid2(uint8_t *flags, int nx, int ny, float cl, const SurfaceArgs &s, cudaStream_t st)
{
    const int grid = std::max(1, std::min((ny + 7) / 8, device_sms() * 8));
    fill_solid2_kernel<<<grid, 256, 0, st>>>(flags, nx, ny, cl, s);
    return cudaGetLastError();
}

// ------------------------------------------------------------- 3D fill
// Counterpart of fillSolidFlags2D for D3Q27 grids.  The reference has the 3D
// inside test (SolidGeometryProxy_Device<3>::isInside,
// SolidGeometryProxy_Device.cuh:231-289: the parity of the triangles that the
// segment from a point to the origin crosses) but no 3D fill; testing every
// cell against every triangle that way is O(cells x triangles).  Here the
// rays run along +x through the (y, z) rows of cell centres:
//   cross   one warp per triangle, lanes over the rows of its (y, z) bounding
//           box: the row crosses the triangle when its point lies in the
//           triangle's (y, z) projection, by edge functions evaluated in
//           vertex-index order (two triangles sharing an edge see exactly
//           opposite values) with ties given to edges that point up in y
//           (then z), so a row through a shared edge or vertex counts once per
//           sheet of the surface.  The crossing's x, from the edge functions
//           as barycentric weights, toggles (atomicXor) one bit of the row's
//           mask: the last cell whose centre lies left of it;
//   apply   one warp per row: a suffix XOR over the mask gives each cell's
//           crossing parity to its right; Fluid and SolidDynamic cells become
//           SolidDynamic where it is odd and Fluid elsewhere (as
//           resetSolidFlagKernel + updateSolidFlagKernel do in 2D,
//           FsiCoupling2D.cu:318-354); the mask is cleared for the next call.
// Every operation is explicitly rounded, in the order of the CPU oracle's
// restatement, so the two give the same flags.
namespace {
__device__ __forceinline__ float fs3_edge(const float *V, uint32_t ip, uint32_t is, float qy, float qz)
{
    using namespace geom;
    const float py = V[3 * (size_t)ip + 1], pz = V[3 * (size_t)ip + 2];
    const float sy = V[3 * (size_t)is + 1], sz = V[3 * (size_t)is + 2];
    return sub(mul(sub(sy, py), sub(qz, pz)), mul(sub(sz, pz), sub(qy, py)));
}
__device__ __forceinline__ float fs3_dir(const float *V, uint32_t iu, uint32_t iv, float qy, float qz, bool &tie)
{
    const float uy = V[3 * (size_t)iu + 1], uz = V[3 * (size_t)iu + 2];
    const float vy = V[3 * (size_t)iv + 1], vz = V[3 * (size_t)iv + 2];
    tie = (vy > uy) || (vy == uy && vz > uz);
    return iu < iv ? fs3_edge(V, iu, iv, qy, qz) : -fs3_edge(V, iv, iu, qy, qz);
}
__device__ __forceinline__ bool fs3_incl(float e, bool tie) { return e > 0.0f || (e == 0.0f && tie); }

// cells x in [0, nx) whose centre (x + 0.5) cl lies left of xc
__device__ __forceinline__ int fs3_count_left(float xc, float cl, int nx)
{
    using namespace geom;
    if (xc != xc) return 0;
    const float t = sub(dvd(xc, cl), 0.5f);
    int k = !(t > 0.0f) ? 0 : (t >= (float)nx ? nx : (int)ceilf(t));
    while (k > 0 && mul(add((float)(k - 1), 0.5f), cl) >= xc) --k;
    while (k < nx && mul(add((float)k, 0.5f), cl) < xc) ++k;
    return k;
}

// rows whose centre can lie in [lo, hi], padded by one, clamped to [0, n)
__device__ __forceinline__ void fs3_rows(float lo, float hi, float cl, int n, int &r0, int &r1)
{
    using namespace geom;
    float a = floorf(sub(dvd(lo, cl), 0.5f)) - 1.0f, b = ceilf(sub(dvd(hi, cl), 0.5f)) + 1.0f;
    a = fminf(fmaxf(a, 0.0f), (float)n);
    b = fminf(fmaxf(b, -1.0f), (float)(n - 1));
    r0 = (int)a;
    r1 = (int)b;
}
} // namespace

__global__ void __launch_bounds__(256) fill_solid3_cross_kernel(uint32_t *bits, int nx, int ny, int nz, int words,
                                                                float cl, SurfaceArgs s)
{
    using namespace geom;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < s.ne; e += nwarps) {
        const uint32_t ia = s.E[3 * e], ib = s.E[3 * e + 1], ic = s.E[3 * e + 2];
        if (ia >= (uint32_t)s.nv || ib >= (uint32_t)s.nv || ic >= (uint32_t)s.nv) continue;
        const float *a = s.V + 3 * (size_t)ia, *b = s.V + 3 * (size_t)ib, *c = s.V + 3 * (size_t)ic;
        bool finite = true;
#pragma unroll
        for (int k = 0; k < 3; ++k) finite &= isfinite(a[k]) && isfinite(b[k]) && isfinite(c[k]);
        if (!finite) continue;
        int y0, y1, z0, z1;
        fs3_rows(fminf(fminf(a[1], b[1]), c[1]), fmaxf(fmaxf(a[1], b[1]), c[1]), cl, ny, y0, y1);
        fs3_rows(fminf(fminf(a[2], b[2]), c[2]), fmaxf(fmaxf(a[2], b[2]), c[2]), cl, nz, z0, z1);
        if (y0 > y1 || z0 > z1) continue;
        const int ey = y1 - y0 + 1, items = ey * (z1 - z0 + 1);
        for (int it = lane; it < items; it += 32) {
            const int y = y0 + it % ey, z = z0 + it / ey;
            const float qy = mul(add((float)y, 0.5f), cl), qz = mul(add((float)z, 0.5f), cl);
            bool t0, t1, t2;
            const float e0 = fs3_dir(s.V, ib, ic, qy, qz, t0);
            const float e1 = fs3_dir(s.V, ic, ia, qy, qz, t1);
            const float e2 = fs3_dir(s.V, ia, ib, qy, qz, t2);
            if (e0 == 0.0f && e1 == 0.0f && e2 == 0.0f) continue;
            const bool pos = fs3_incl(e0, t0) && fs3_incl(e1, t1) && fs3_incl(e2, t2);
            const bool neg = fs3_incl(-e0, !t0) && fs3_incl(-e1, !t1) && fs3_incl(-e2, !t2);
            if (!pos && !neg) continue;
            const float xc = dvd(add(add(mul(e0, a[0]), mul(e1, b[0])), mul(e2, c[0])), add(add(e0, e1), e2));
            const int k = fs3_count_left(xc, cl, nx);
            if (k < 1) continue;
            atomicXor(bits + ((size_t)z * ny + y) * words + ((k - 1) >> 5), 1u << ((k - 1) & 31));
        }
    }
}

__global__ void __launch_bounds__(256) fill_solid3_apply_kernel(uint8_t *flags, uint32_t *bits, int nx, long long rows,
                                                                int words)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += nwarps) {
        uint32_t *rb = bits + (size_t)row * words;
        // word w becomes: bit i = parity of the mask bits at positions >= 32 w + i
        uint32_t carry = 0; // parity of the words above the current chunk of 32
        for (int base = ((words - 1) >> 5) << 5; base >= 0; base -= 32) {
            const int w = base + lane;
            uint32_t m = w < words ? rb[w] : 0u;
            const unsigned par = __ballot_sync(full, __popc(m) & 1);
            const uint32_t above = ((uint32_t)__popc((par >> lane) >> 1) & 1u) ^ carry;
            m ^= m >> 1; m ^= m >> 2; m ^= m >> 4; m ^= m >> 8; m ^= m >> 16;
            if (above) m = ~m;
            if (w < words) rb[w] = m;
            carry ^= (uint32_t)__popc(par) & 1u;
        }
        __syncwarp();
        for (int x = lane; x < nx; x += 32) {
            uint8_t *f = flags + (size_t)row * nx + x;
            const uint32_t t = *f & kTypeMask;
            if (t == kFluid || t == kSolidDynamic) *f = ((rb[x >> 5] >> (x & 31)) & 1u) ? kSolidDynamic : kFluid;
        }
        __syncwarp();
        for (int w = lane; w < words; w += 32) rb[w] = 0u; // clear for the next fill
    }
}

cudaError_t launch_fill_solid3(uint8_t *flags, uint32_t *bits, int nx, int ny, int nz, float cl, const SurfaceArgs &s,
                               cudaStream_t st)
{
    const int sms = device_sms();
    const int words = (nx + 31) / 32;
    if (s.ne > 0) {
        const int grid = (int)std::max<long long>(1, std::min<long long>((s.ne + 7) / 8, (long long)sms * 16));
        fill_solid3_cross_kernel<<<grid, 256, 0, st>>>(bits, nx, ny, nz, words, cl, s);
    }
    const long long rows = (long long)ny * nz;
    const int grid = (int)std::max<long long>(1, std::min<long long>((rows + 7) / 8, (long long)sms * 8));
    fill_solid3_apply_kernel<<<grid, 256, 0, st>>>(flags, bits, nx, rows, words);
    return cudaGetLastError();
}

// FP32 AoS/SoA <-> device storage (SoA planes, possibly encoded)
template <int DIM, typename T>
__global__ void convert_in_kernel(const float *in, bool aos, T *out, uint32_t ncell, Codec cdc)
{
    constexpr int NM = Lattice<DIM>::NM;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        float m[NM];
        for (int k = 0; k < NM; ++k) m[k] = aos ? in[c * NM + k] : in[(size_t)k * ncell + c];
        T *pl[NM];
        for (int k = 0; k < NM; ++k) pl[k] = out + (size_t)k * ncell;
        encode_store<DIM, T>(m, pl, (uint32_t)c, cdc);
    }
}

template <int DIM, typename T>
__global__ void convert_out_kernel(const T *in, float *out, bool aos, uint32_t ncell, Codec cdc)
{
    constexpr int NM = Lattice<DIM>::NM;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        float m[NM];
        load_moments<DIM, T>(m, in, ncell, (uint32_t)c, cdc);
        for (int k = 0; k < NM; ++k) {
            if (aos) out[c * NM + k] = m[k];
            else out[(size_t)k * ncell + c] = m[k];
        }
    }
}

template <int DIM, typename T>
cudaError_t launch_convert_in(const float *in, bool aos, T *out, uint32_t ncell, Codec c, cudaStream_t st)
{
    int grid = (int)std::min<long long>(((long long)ncell + 255) / 256, (long long)device_sms() * 16);
    convert_in_kernel<DIM, T><<<grid, 256, 0, st>>>(in, aos, out, ncell, c);
    return cudaGetLastError();
}
template <int DIM, typename T>
cudaError_t launch_convert_out(const T *in, float *out, bool aos, uint32_t ncell, Codec c, cudaStream_t st)
{
    int grid = (int)std::min<long long>(((long long)ncell + 255) / 256, (long long)device_sms() * 16);
    convert_out_kernel<DIM, T><<<grid, 256, 0, st>>>(in, out, aos, ncell, c);
    return cudaGetLastError();
}

#define FFS_INST_AUX(DIM, T)                                                                                           \
    template cudaError_t launch_initialize<DIM, T>(const GridArgs<T> &, T *, const float *, cudaStream_t);            \
    template cudaError_t launch_convert_in<DIM, T>(const float *, bool, T *, uint32_t, Codec, cudaStream_t);          \
    template cudaError_t launch_convert_out<DIM, T>(const T *, float *, bool, uint32_t, Codec, cudaStream_t);
FFS_INST_AUX(2, float)
FFS_INST_AUX(2, __half)
FFS_INST_AUX(2, __nv_bfloat16)
FFS_INST_AUX(3, float)
FFS_INST_AUX(3, __half)
FFS_INST_AUX(3, __nv_bfloat16)

} // namespace fflbm
