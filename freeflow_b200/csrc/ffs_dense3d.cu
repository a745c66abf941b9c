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
//   * each plane is reconstructed once for its 34 x 10 xy halo: every thread
//     reconstructs its own cell, and the first 84 threads one cell of the
//     ring around the tile as well (only the 9 populations it feeds into the
//     tile, one kind of ring cell per warp);
//   * the populations of plane p go to one of two shared-memory buffers
//     (2 x 27 x 340 floats) and are consumed as soon as they exist: the
//     c_z = -1 slice completes the raw moments of the cell below (plane p-1),
//     the c_z = 0 slice feeds plane p, the c_z = +1 slice starts plane p+1.
//     Each thread keeps the partial raw moments of its column's next two
//     cells in registers, so there is one barrier per plane;
//   * bounce-back: a halo cell of a bounce-back type (wall, solid) gets zeros
//     in its 27 population slots instead of a reconstruction, so whatever a
//     fluid neighbour pulls from it adds nothing; each fluid cell next to a
//     wall then adds its own reflected populations max(0, f_inv(i)^rec(x))
//     once, while its own plane is in shared memory.  The result is the
//     reference's f_i(x) = max(0, f_inv(i)^rec(x)) for wall neighbours x - c_i
//     (FsiCoupling3D.cu:209-222), whose wall test looks at the wrapped index.
//     The halo index is the reference's too (halo_index: it wraps at the low
//     face and clamps at the high face of a non-periodic axis), so the halo
//     cell and the tested cell coincide everywhere except across a high face:
//     halo cells beyond a high face are always reconstructed, walls included
//     (the reference pulls them when the wrapped test says fluid), and a cell
//     whose wrapped neighbour across the face is a wall removes that pulled
//     value explicitly (wall_fix_part);
//   * moments are SoA planes in HBM (128 B coalesced per warp and moment);
//     moments, flag bytes and wall masks are prefetched a plane ahead;
//     outlets are fed by their inner neighbour in the same pass, and cells with
//     moving-boundary links are left to the sparse link kernel (ffs_links.cu).
#include "ffs_dense2d.cuh"
#include "ffs_dense3d.cuh"

#include <cstdlib>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

namespace fflbm {

namespace {
constexpr int kTX = D3::kTX, kTY = D3::kTY, kHX = D3::kHX, kHalo = D3::kHalo, kRing = D3::kRing;
constexpr int kPlane = D3::kPlaneFloats;

__device__ __forceinline__ int set_of(int kx, int ky, int kz) { return (kz * 3 + ky) * 3 + kx; }

// halo index (hx, hy) of ring cell r, grouped so that each warp holds one
// kind of ring cell: r < 32 the row y0-1 (hx 1..32), r < 64 the row y0+8
// (hx 1..32), r < 74 the column x0-1 (hy 0..9, corners included), r < 84
// the column x0+32
__device__ __forceinline__ int ring_cell(int r)
{
    if (r < 32) return r + 1;
    if (r < 64) return (kHalo - kHX) + (r - 31);
    if (r < 74) return (r - 64) * kHX;
    return (r - 74) * kHX + kHX - 1;
}

// raw-moment slot: {rho, jx, jy, jz, Pxx, Pyy, Pzz, Pxy, Pyz, Pxz}
//
// Unweighted populations.  The single-plane kernel stores each population
// as its Hermite sum F_i without the lattice weight and applies the weights
// on the way into the raw moments.  The D3Q27 weights are one constant times
// powers of four, w_i = W0 4^-n(i) with W0 = wgt3(1,1,1) = 8/27 and n(i) the
// number of non-zero components of c_i (8/27, 2/27, 1/54, 1/216 exactly, as
// float constants too), and max(0, w F) = w max(0, F), so every weighted sum
// follows from the unweighted one by exact power-of-two scalings.  The kernel
// accumulates R''_k = R_k / (W0 s_k) with
//   s = {1/4, 1/16, 1/16, 1/4, 1/16, 1/16, 1/4, 1/64, 1/16, 1/16},
// chosen so that the c_z = +-1 slices add their sums as they are and the
// c_z = 0 slice adds 4 Y; a completed cell's sums are multiplied by W0 s_k.
// This replaces the 27 weight multiplications of every reconstruction (own
// cell and ring) by 10 per updated cell.  (W0 s_k are exact products.)
constexpr float kW0 = wgt3(1, 1, 1);
__device__ __forceinline__ void raw_from_scaled(const float *Rs, float *R)
{
    constexpr float s[10] = {0.25f, 0.0625f, 0.0625f, 0.25f, 0.0625f, 0.0625f, 0.25f, 0.015625f, 0.0625f, 0.0625f};
#pragma unroll
    for (int k = 0; k < 10; ++k) R[k] = Rs[k] * (kW0 * s[k]);
}

// 9 unweighted populations of one c_z slice (clamped) -> x/y sums
// Y = {Y00, Y01, Y02, Y10, Y11, Y20}; the weighted sums are
// W0 4^-|c_z| c_k Y_k with c = {1, 1/4, 1/4, 1/4, 1/16, 1/4}
__device__ __forceinline__ void slice_sums(const float *buf, int kz, int c_own, float *Y)
{
    float X0[3], X1[3], X2[3];
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
        // population (kx, ky, kz) of the cell at c_own - (kx-1) - (ky-1)*kHX
        const int crow = c_own - (ky - 1) * kHX;
        float fm = fmaxf(buf[set_of(0, ky, kz) * kHalo + crow + 1], 0.0f);
        float f0 = fmaxf(buf[set_of(1, ky, kz) * kHalo + crow], 0.0f);
        float fp = fmaxf(buf[set_of(2, ky, kz) * kHalo + crow - 1], 0.0f);
        float s = fp + fm;
        X1[ky] = fp - fm;
        X0[ky] = fmaf(0.25f, s, f0);
        X2[ky] = s;
    }
    float s0 = X0[2] + X0[0];
    Y[0] = fmaf(0.25f, s0, X0[1]);
    Y[1] = X0[2] - X0[0];
    Y[2] = s0;
    Y[3] = fmaf(0.25f, X1[2] + X1[0], X1[1]);
    Y[4] = X1[2] - X1[0];
    Y[5] = fmaf(0.25f, X2[2] + X2[0], X2[1]);
}

// add the slice with c_z = CZ to the scaled sums R''
template <int CZ> __device__ __forceinline__ void slice_add(float *R, const float *Y)
{
    if (CZ == 0) {
        R[0] = fmaf(4.0f, Y[0], R[0]); R[2] = fmaf(4.0f, Y[1], R[2]); R[5] = fmaf(4.0f, Y[2], R[5]);
        R[1] = fmaf(4.0f, Y[3], R[1]); R[7] = fmaf(4.0f, Y[4], R[7]); R[4] = fmaf(4.0f, Y[5], R[4]);
    } else {
        R[0] += Y[0]; R[2] += Y[1]; R[5] += Y[2]; R[1] += Y[3]; R[7] += Y[4]; R[4] += Y[5];
        R[3] += CZ * Y[0]; R[6] += Y[0]; R[8] += CZ * Y[1]; R[9] += CZ * Y[3];
    }
}
__device__ __forceinline__ void slice_init_plus(float *R, const float *Y)
{
    R[0] = Y[0]; R[2] = Y[1]; R[5] = Y[2]; R[1] = Y[3]; R[7] = Y[4]; R[4] = Y[5];
    R[3] = Y[0]; R[6] = Y[0]; R[8] = Y[1]; R[9] = Y[3];
}

// R'' += (basis(c) w F) / (W0 s) for one unweighted population F of
// direction c: the weight and the scales are powers of two
__device__ __forceinline__ void add_basis_scaled(float *R, int cx, int cy, int cz, float F)
{
    const int n = (cx != 0) + (cy != 0) + (cz != 0);
    const float t = F * (n == 0 ? 1.0f : n == 1 ? 0.25f : n == 2 ? 0.0625f : 0.015625f);
    const float fx = (float)cx, fy = (float)cy, fz = (float)cz;
    R[0] = fmaf(4.0f, t, R[0]);
    R[1] = fmaf(16.0f * fx, t, R[1]); R[2] = fmaf(16.0f * fy, t, R[2]); R[3] = fmaf(4.0f * fz, t, R[3]);
    R[4] = fmaf(16.0f * fx * fx, t, R[4]); R[5] = fmaf(16.0f * fy * fy, t, R[5]); R[6] = fmaf(4.0f * fz * fz, t, R[6]);
    R[7] = fmaf(64.0f * fx * fy, t, R[7]); R[8] = fmaf(16.0f * fy * fz, t, R[8]); R[9] = fmaf(16.0f * fx * fz, t, R[9]);
}

// R += s * basis(c) for the velocity (cx, cy, cz)
__device__ __forceinline__ void add_basis(float *R, int cx, int cy, int cz, float s)
{
    R[0] += s;
    R[1] += cx * s; R[2] += cy * s; R[3] += cz * s;
    R[4] += cx * cx * s; R[5] += cy * cy * s; R[6] += cz * cz * s;
    R[7] += cx * cy * s; R[8] += cy * cz * s; R[9] += cx * cz * s;
}

// Bounce-back corrections that the current plane (buf, plane p) allows:
//   cell p-1 (Rp, mask wp): remove the pulled c_z = -1 populations of wall
//                           directions (they came from plane p);
//   cell p   (Rc, mask wc): remove the pulled c_z = 0 ones, add the cell's own
//                           reflected populations f_inv(i)(x) (its plane is p);
//   cell p+1 (Rn, mask wn): remove the pulled c_z = +1 ones.
// Reference rule: FsiCoupling3D.cu:209-222, f_i(x) = max(0, f_inv(i)^rec(x)).
// Only the set bits are visited (a wall face sets nine of them).
__device__ __forceinline__ void add_basis_rt(float *R, int cx, int cy, int cz, float s)
{
    const float fx = (float)cx, fy = (float)cy, fz = (float)cz;
    R[0] += s;
    R[1] = fmaf(fx, s, R[1]); R[2] = fmaf(fy, s, R[2]); R[3] = fmaf(fz, s, R[3]);
    R[4] = fmaf(fx * fx, s, R[4]); R[5] = fmaf(fy * fy, s, R[5]); R[6] = fmaf(fz * fz, s, R[6]);
    R[7] = fmaf(fx * fy, s, R[7]); R[8] = fmaf(fy * fz, s, R[8]); R[9] = fmaf(fx * fz, s, R[9]);
}

// R'' += basis(c_i) w_i max(0, F_inv(i)(x)) (scaled as above) for every wall
// direction i in w, with the cell's own unweighted populations read from the
// current plane.
__device__ __forceinline__ void add_reflected(const float *buf, int c_own, uint32_t w, float (&R)[10])
{
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const int i = dir_index<3>(kx, ky, kz);
                if (i == 0) continue;
                float f = fmaxf(buf[set_of(2 - kx, 2 - ky, 2 - kz) * kHalo + c_own], 0.0f);
                f = (w & (1u << i)) ? f : 0.0f;
                add_basis_scaled(R, kx - 1, ky - 1, kz - 1, f);
            }
}

// Removes from R'' the pulled populations of the wall directions in w whose
// c_z slice is kz_sel (their source is the current plane): across a high
// face the halo cell holds real populations, but the wrapped test found a
// wall, so the step takes the cell's reflected population instead
// (add_reflected).
__device__ __forceinline__ void wall_fix_part(const float *buf, int c_own, uint32_t w, int kz_sel, float (&R)[10])
{
    while (w) {
        const int i = __ffs(w) - 1;
        w &= w - 1;
        int cx, cy, cz;
        dir_vec<3>(i, cx, cy, cz);
        if (cz + 1 == kz_sel) {
            const float pulled = fmaxf(buf[set_of(cx + 1, cy + 1, cz + 1) * kHalo + c_own - cx - cy * kHX], 0.0f);
            add_basis_scaled(R, cx, cy, cz, -pulled);
        }
    }
}
} // namespace

// MINB = CTAs per SM the register budget is cut for; launch_dense3d times the
// variants on the grid and keeps the faster (tune_dense3d).
// IDX32: every moment, flag and mask index (k * ncell + cell) fits in 32
// bits, as it does for grids of up to 429 M cells; each access then takes one
// 32-bit index and one widening multiply-add instead of 64-bit arithmetic,
// which saves registers (112 against 122) and about 5 % of the pass.
template <typename T, int MINB, bool IDX32>
__global__ void __launch_bounds__(D3::kThreads, MINB) dense3d_kernel(GridArgs<T> g, int zchunk)
{
    extern __shared__ float smem[];
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, g.nz);
    const long long nxy = (long long)g.nx * g.ny;
    const bool wx = g.periodic & 1, wy = g.periodic & 2, wz = g.periodic & 4;

    const int tx = tid % kTX, ty = tid / kTX;
    const int x = x0 + tx, y = y0 + ty;
    const bool inside = x < g.nx && y < g.ny;
    const int c_own = (ty + 1) * kHX + (tx + 1);
    // partner cell of the reconstruction pair
    const bool has_ring = tid < kRing;
    const int c_ring = has_ring ? ring_cell(tid) : c_own;
    auto planar = [&](int c) {
        int hx = c % kHX, hy = c / kHX;
        return (uint32_t)(halo_index(y0 + hy - 1, g.ny, wy) * g.nx + halo_index(x0 + hx - 1, g.nx, wx));
    };
    const uint32_t off_own = planar(c_own), off_ring = planar(c_ring);
    const uint32_t col = inside ? (uint32_t)(y * g.nx + x) : 0u;
    // directions whose pull crosses the high x or y face of a non-periodic
    // axis (only there can the halo cell and the wrapped test differ)
    uint32_t oor_xy = 0;
    if (inside && ((!wx && x == g.nx - 1) || (!wy && y == g.ny - 1))) {
#pragma unroll
        for (int i = 1; i < 27; ++i) {
            int cx, cy, cz;
            dir_vec<3>(i, cx, cy, cz);
            if ((!wx && x - cx >= g.nx) || (!wy && y - cy >= g.ny)) oor_xy |= 1u << i;
        }
    }
    uint32_t oor_zhi = 0; // directions pulling across z = nz-1 from above
    if (!wz) {
#pragma unroll
        for (int i = 1; i < 27; ++i) {
            int cx, cy, cz;
            dir_vec<3>(i, cx, cy, cz);
            if (cz == -1) oor_zhi |= 1u << i;
        }
    }
    // halo cells beyond a high face keep their real populations even when
    // they are walls (x and y per thread, z per plane)
    auto beyond_hi = [&](int c) {
        const int hx = x0 + c % kHX - 1, hy = y0 + c / kHX - 1;
        return (!wx && hx >= g.nx) || (!wy && hy >= g.ny);
    };
    const bool own_hi = beyond_hi(c_own), ring_hi = beyond_hi(c_ring);

    // stored moments of the two halo cells, converted when they are
    // reconstructed (so that only the ring warps convert the ring cell's;
    // the loads themselves stay predicated in every warp, which overlaps them
    // with the own-cell loads: a warp-uniform branch around the ring loads
    // measured 9 % slower on 384 x 192 x 192)
    T mA[10], mB[10];
    uint32_t hA = 0, hB = 0; // node types of the two halo cells (bounce-back cells get zero slots)
    auto load_plane = [&](int z) {
        if constexpr (IDX32) {
            const uint32_t zo = (uint32_t)halo_index(z, g.nz, wz) * (uint32_t)nxy;
            const uint32_t io = zo + off_own, ir = zo + off_ring;
#pragma unroll
            for (int k = 0; k < 10; ++k) {
                mA[k] = g.src[io + (uint32_t)k * g.ncell];
                if (has_ring) mB[k] = g.src[ir + (uint32_t)k * g.ncell];
            }
            hA = g.flags[io] & kTypeMask;
            if (has_ring) hB = g.flags[ir] & kTypeMask;
        } else {
            const size_t zo = (size_t)halo_index(z, g.nz, wz) * nxy;
            const T *base = g.src + zo;
#pragma unroll
            for (int k = 0; k < 10; ++k) {
                mA[k] = base[(size_t)k * g.ncell + off_own];
                if (has_ring) mB[k] = base[(size_t)k * g.ncell + off_ring];
            }
            hA = g.flags[zo + off_own] & kTypeMask;
            if (has_ring) hB = g.flags[zo + off_ring] & kTypeMask;
        }
    };
    // index of the column's cell in plane z (32 or 64-bit, as above)
    auto cell_at = [&](int z) {
        if constexpr (IDX32) return (size_t)((uint32_t)z * (uint32_t)nxy + col);
        else return (size_t)z * nxy + col;
    };
    auto recon_cell = [&](float *buf, const T *raw, bool zero, int c) {
        if (zero) {
#pragma unroll
            for (int j = 0; j < 27; ++j) buf[j * kHalo + c] = 0.0f;
            return;
        }
        float m[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) m[k] = from_storage<3, T>(k, raw[k]);
        decode_moments<3, T>(m, g.codec);
        Coef3V<float> cf;
        cf.make(m);
        cf.populations_each<false>([&](int kz, int ky, int kx, float v) { buf[set_of(kx, ky, kz) * kHalo + c] = v; });
    };
    // A ring cell feeds the tile only the 9 populations that point into it:
    // c_y = +1 from the row below (warp 0), c_y = -1 from the row above
    // (warp 1), c_x = +-1 from the columns (warp 2).  Each warp runs one
    // uniform path that evaluates just those; no other slot of a ring cell is
    // ever read.
    const int ring_kind = tid < 32 ? 0 : tid < 64 ? 1 : 2;
    const float ring_sx = tid < 74 ? 1.0f : -1.0f;                 // columns: c_x of the fed populations
    const int ring_kxo = (tid < 74 ? 2 : 0) * kHalo;               // their kx plane offset
    auto recon_ring = [&](float *buf, bool zero) {
        const int c = c_ring;
        if (zero) {
#pragma unroll
            for (int kz = 0; kz < 3; ++kz)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (ring_kind == 0) buf[set_of(k, 2, kz) * kHalo + c] = 0.0f;
                    else if (ring_kind == 1) buf[set_of(k, 0, kz) * kHalo + c] = 0.0f;
                    else buf[set_of(0, k, kz) * kHalo + ring_kxo + c] = 0.0f;
                }
            return;
        }
        float m[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) m[k] = from_storage<3, T>(k, mB[k]);
        decode_moments<3, T>(m, g.codec);
        Coef3V<float> cf;
        cf.make(m);
        if (ring_kind == 0)
            cf.populations_row<2>([&](int kz, int kx, float v) { buf[set_of(kx, 2, kz) * kHalo + c] = v; });
        else if (ring_kind == 1)
            cf.populations_row<0>([&](int kz, int kx, float v) { buf[set_of(kx, 0, kz) * kHalo + c] = v; });
        else
            cf.populations_col(ring_sx, [&](int kz, int ky, float v) { buf[set_of(0, ky, kz) * kHalo + ring_kxo + c] = v; });
    };
    // plane p's halo cells; bounce-back cells get zero slots unless they lie
    // beyond a high face
    auto recon_plane = [&](float *buf, int p) {
        const bool zhi = !wz && p >= g.nz;
        recon_cell(buf, mA, is_bounce_back<3>(hA) && !(own_hi || zhi), c_own);
        if (has_ring) recon_ring(buf, is_bounce_back<3>(hB) && !(ring_hi || zhi));
    };
    auto flag_at = [&](int z) -> uint32_t {
        return (inside && z >= zb && z < ze) ? (uint32_t)g.flags[cell_at(z)] : 0u;
    };

    // Two register sets hold the partial raw moments of the column's cells at
    // z = p-1 and z = p; their roles swap every plane (loop unrolled by two).
    float X[10], Y[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) X[k] = Y[k] = 0.0f;
    // flag bytes of z = p-1, p, p+1 and wall masks of z = p-1, p
    uint32_t fp = 0, fc = 0, fn = flag_at(zb);
    uint32_t wp = 0, wc = 0;

    // one plane: Rp = sums of z = p-1 (completed here), Rc = sums of z = p,
    // Rn receives the new c_z = +1 slice (the cell at z = p+1)
    auto plane = [&](int p, float (&Rp)[10], float (&Rc)[10]) {
        float *buf = smem + (p & 1) * kPlane;
        recon_plane(buf, p);
        if (p < ze) load_plane(p + 1);
        const uint32_t fnn = flag_at(p + 2);
        // mask word (wall and outlet bits) of the cell at z = p+1; only cells
        // this pass updates use it (walls, inlets and outlets carry mask bits
        // of their own neighbours that must not trigger any work)
        const bool upd_n = is_updated(fn & kTypeMask) && !(fn & kBitLink);
        const uint32_t wn = (upd_n && (fn & (kBitNearWall | kBitOutletSrc))) ? g.wallmask[cell_at(p + 1)] : 0u;
        __syncthreads();
        if (inside) {
            float S[6];
            slice_sums(buf, 0, c_own, S);
            slice_add<-1>(Rp, S);
            slice_sums(buf, 1, c_own, S);
            slice_add<0>(Rc, S);
            constexpr uint32_t kWall = wall_bits_mask<3>();
            if (wc & kWall) add_reflected(buf, c_own, wc & kWall, Rc);
            // wall directions across a high face (their halo cell held real
            // populations): remove the pulled value, per destination cell
            // z = p-1 (c_z = -1 slice) and z = p (c_z = 0)
            const uint32_t oor_p = oor_xy | ((p - 1 == g.nz - 1) ? oor_zhi : 0u);
            if (wp & kWall & oor_p) wall_fix_part(buf, c_own, wp & kWall & oor_p, 0, Rp);
            if (wc & kWall & oor_xy) wall_fix_part(buf, c_own, wc & kWall & oor_xy, 1, Rc);
            // the cell at z = p - 1 is complete
            const int d = p - 1;
            if (d >= zb && is_updated(fp & kTypeMask) && !(fp & kBitLink)) {
                const uint32_t idx = (uint32_t)(d * nxy + col);
                float R[10], m[10];
                raw_from_scaled(Rp, R);
                collide3(R, g.omega, m);
                if constexpr (IDX32) encode_store_idx32<3, T>(m, g.dst, idx, g.ncell, g.codec);
                else encode_store_strided<3, T>(m, g.dst, (size_t)idx, g.ncell, g.codec);
                if (bad_state<3>(m)) atomicOr(g.status, kStatusNonFinite);
                if (fp & kBitOutletSrc) {
                    float ms[10];
                    stored_values<3, T>(m, ms, idx, g.codec);
                    feed_outlets<3, T>(g, idx, ms, wp);
                }
            }
            // Rp is free: it becomes the cell at z = p + 1
            slice_sums(buf, 2, c_own, S);
            slice_init_plus(Rp, S);
            if (wn & kWall & oor_xy) wall_fix_part(buf, c_own, wn & kWall & oor_xy, 2, Rp);
        }
        fp = fc; fc = fn; fn = fnn;
        wp = wc; wc = wn;
    };

    load_plane(zb - 1);
    int p = zb - 1;
    for (; p + 1 <= ze; p += 2) {
        plane(p, X, Y);     // completes X (z = p-1); X := z = p+1
        plane(p + 1, Y, X); // completes Y (z = p);   Y := z = p+2
    }
    if (p <= ze) plane(p, X, Y);
}

// CTAs of `kernel` resident on the current device at once (SMs x occupancy),
// with the kernel's dynamic shared-memory limit raised to `smem` first.
// Cached per (kernel, device ordinal): a process may step grids on several
// GPUs, and the first launch on each device configures the kernel there.
static cudaError_t resident_slots(const void *kernel, int threads, size_t smem, int &slots)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> cache;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({kernel, dev});
    if (it != cache.end()) {
        slots = it->second;
        return cudaSuccess;
    }
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    slots = device_sms() * (per_sm > 0 ? per_sm : 1);
    cache[{kernel, dev}] = slots;
    return cudaSuccess;
}

// Number of z chunks that best fills the GPU: whole waves of CTAs, with the
// two extra planes each chunk reconstructs counted as overhead.
static int choose_zchunks(int tiles, int nz, int slots)
{
    // CTAs next to walls and outlets carry extra work; several waves of CTAs
    // let the scheduler even that out, so aim for three waves or more while
    // chunks keep at least 16 planes
    int nmin = 1;
    while ((long long)tiles * nmin < 3LL * slots && nz / (nmin + 1) >= 16) ++nmin;
    int best = nmin;
    double best_eff = 0.0;
    for (int n = nmin; n <= nmin + 8 && n <= nz; ++n) {
        int chunk = (nz + n - 1) / n;
        long long ctas = (long long)tiles * ((nz + chunk - 1) / chunk);
        long long waves = (ctas + slots - 1) / slots;
        double eff = (double)ctas / (double)(waves * slots) * (double)chunk / (double)(chunk + 2);
        if (eff > best_eff + 1e-9) { best_eff = eff; best = n; }
    }
    return best;
}

template <typename T, int MINB, bool IDX32> struct Dense3dLaunchAs {
    static cudaError_t run(const GridArgs<T> &g, cudaStream_t s)
    {
        int slots = 0;
        cudaError_t e = resident_slots(reinterpret_cast<const void *>(dense3d_kernel<T, MINB, IDX32>), D3::kThreads,
                                       D3::kSmemBytes, slots);
        if (e != cudaSuccess) return e;
        int tx = (g.nx + kTX - 1) / kTX, ty = (g.ny + kTY - 1) / kTY;
        int nchunk = choose_zchunks(tx * ty, g.nz, slots);
        int zchunk = (g.nz + nchunk - 1) / nchunk;
        dim3 grid(tx, ty, (g.nz + zchunk - 1) / zchunk);
        dense3d_kernel<T, MINB, IDX32><<<grid, D3::kThreads, D3::kSmemBytes, s>>>(g, zchunk);
        return cudaGetLastError();
    }
};

// 32-bit indices whenever every moment index of the grid fits (FFS_DENSE3D_INDEX64
// forces 64-bit indices, so that tests reach that path on small grids)
template <typename T, int MINB> struct Dense3dLaunch {
    static cudaError_t run(const GridArgs<T> &g, cudaStream_t s)
    {
        const char *force64 = std::getenv("FFS_DENSE3D_INDEX64");
        if (10ull * g.ncell <= 0xFFFFFFFFull && !(force64 && force64[0] == '1'))
            return Dense3dLaunchAs<T, MINB, true>::run(g, s);
        return Dense3dLaunchAs<T, MINB, false>::run(g, s);
    }
};


template <typename T> bool dense3d_has_variant(int v) { return v >= 0 && v < kDense3dVariants; }

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
    // FFS_DENSE3D_VARIANT pins the variant (tests run every variant this way)
    if (const char *pin = std::getenv("FFS_DENSE3D_VARIANT")) {
        const int v = std::atoi(pin);
        if (dense3d_has_variant<T>(v)) return v;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    int best_v = 0;
    // the single-plane kernel for two and three CTAs per SM, which round
    // identically
    for (int v = 0; v < kDense3dVariants; ++v) {
        if (!dense3d_has_variant<T>(v)) continue;
        if (launch_dense3d<T>(g, s, v) != cudaSuccess) continue; // warm-up
        cudaEventRecord(a, s);
        for (int r = 0; r < 3; ++r) launch_dense3d<T>(g, s, v);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        // a later variant must win clearly (both give the same bits; this
        // only keeps the choice stable)
        if (ms < (v == 0 ? 1.0f : 0.97f) * best) { best = ms; best_v = v; }
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
