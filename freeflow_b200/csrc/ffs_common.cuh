// Common device definitions for the B200 moment-encoded LBM fluid step.
//
// Lattices (same direction numbering as the reference, so link indices,
// inverse directions and the AoS layout exchanged through the C ABI agree):
//   D2Q9  include/FSI_Simulator/lbm/LbmConstants.hpp:48-54
//   D3Q27 include/FSI_Simulator/lbm/LbmConstants.hpp:24-35
// Node flags: include/FSI_Simulator/lbm/LbmDataTypes.cuh:17-56.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

namespace fflbm {

// ---------------------------------------------------------------- lattices
template <int DIM> struct Lattice;

template <> struct Lattice<2> {
    static constexpr int Q = 9, NM = 6;
    static __host__ __device__ constexpr int cx(int i) { return i == 1 || i == 5 || i == 8 ? 1 : (i == 3 || i == 6 || i == 7 ? -1 : 0); }
    static __host__ __device__ constexpr int cy(int i) { return i == 2 || i == 5 || i == 6 ? 1 : (i == 4 || i == 7 || i == 8 ? -1 : 0); }
    static __host__ __device__ constexpr int cz(int) { return 0; }
    static __host__ __device__ constexpr int inv(int i) { return i == 0 ? 0 : (i <= 4 ? ((i + 1) % 4) + 1 : ((i - 3) % 4) + 5); }
};

template <> struct Lattice<3> {
    static constexpr int Q = 27, NM = 10;
    static __host__ __device__ constexpr int cx(int i)
    {
        constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
        return t[i];
    }
    static __host__ __device__ constexpr int cy(int i)
    {
        constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
        return t[i];
    }
    static __host__ __device__ constexpr int cz(int i)
    {
        constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
        return t[i];
    }
    // reference numbering pairs i with i+1 (odd i) after the rest population
    static __host__ __device__ constexpr int inv(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
};

// direction index of the velocity (cx, cy, cz); -1 if none
template <int DIM> __host__ __device__ constexpr int dir_of(int x, int y, int z)
{
    for (int i = 0; i < Lattice<DIM>::Q; ++i)
        if (Lattice<DIM>::cx(i) == x && Lattice<DIM>::cy(i) == y && Lattice<DIM>::cz(i) == z) return i;
    return -1;
}

// Direction index by velocity, [kz][ky][kx] with k = c + 1, filled at compile
// time so that unrolled loops over (kx, ky, kz) index it with constants.
template <int DIM> struct DirTable {
    int v[3][3][3];
    __host__ __device__ constexpr DirTable() : v{}
    {
        for (int kz = 0; kz < 3; ++kz)
            for (int ky = 0; ky < 3; ++ky)
                for (int kx = 0; kx < 3; ++kx) v[kz][ky][kx] = dir_of<DIM>(kx - 1, ky - 1, kz - 1);
    }
};
template <int DIM> __host__ __device__ constexpr int dir_index(int kx, int ky, int kz)
{
    constexpr DirTable<DIM> t{};
    return t.v[kz][ky][kx];
}

// (c_x, c_y, c_z) of a direction index known only at run time (e.g. lane
// = direction), decoded from 64-bit immediates: 6 bits per direction holding
// c + 1 in base 4.  Unlike a __constant__ table this costs no memory access,
// and lanes asking for different directions do not serialise.
namespace dirpack {
template <int DIM> struct Packed;
template <> struct Packed<2> {
    static constexpr unsigned long long word(int w)
    {
        unsigned long long r = 0;
        for (int i = 0; i < 9; ++i)
            r |= (unsigned long long)((Lattice<2>::cx(i) + 1) | ((Lattice<2>::cy(i) + 1) << 2) | (1 << 4)) << (6 * i);
        return w == 0 ? r : 0ull;
    }
};
template <> struct Packed<3> {
    static constexpr unsigned long long word(int w)
    {
        unsigned long long r = 0;
        for (int i = 10 * w; i < 10 * w + 10 && i < 27; ++i)
            r |= (unsigned long long)((Lattice<3>::cx(i) + 1) | ((Lattice<3>::cy(i) + 1) << 2) | ((Lattice<3>::cz(i) + 1) << 4))
                 << (6 * (i - 10 * w));
        return r;
    }
};
} // namespace dirpack

template <int DIM> __host__ __device__ __forceinline__ void dir_vec(int i, int &cx, int &cy, int &cz)
{
    constexpr unsigned long long w0 = dirpack::Packed<DIM>::word(0);
    constexpr unsigned long long w1 = dirpack::Packed<DIM>::word(1);
    constexpr unsigned long long w2 = dirpack::Packed<DIM>::word(2);
    unsigned long long w;
    int sh;
    if (DIM == 2) { w = w0; sh = 6 * i; }
    else {
        w = i < 10 ? w0 : (i < 20 ? w1 : w2);
        sh = 6 * (i < 10 ? i : (i < 20 ? i - 10 : i - 20));
    }
    const unsigned v = (unsigned)(w >> sh) & 63u;
    cx = (int)(v & 3u) - 1;
    cy = (int)((v >> 2) & 3u) - 1;
    cz = (int)(v >> 4) - 1;
}

// ------------------------------------------------------------------- flags
enum Flag : uint8_t {
    kInvalid = 0, kFluid = 1, kFluidRest = 2, kSolid = 3, kSolidDynamic = 4, kWall = 5,
    kWallLeft = 6, kWallRight = 7, kWallFront = 8, kWallBack = 9, kWallDown = 10, kWallUp = 11,
    kWallCorner = 12, kInletLeft = 13, kInletRight = 14, kInletUp = 15, kInletDown = 16,
    kInletFront = 17, kInletBack = 18, kOutletLeft = 19, kOutletRight = 20, kOutletUp = 21,
    kOutletDown = 22, kOutletFront = 23, kOutletBack = 24, kReceptor = 25, kDeactivated = 26, kSmoke = 27,
};

// The device flag byte keeps the node type in its low 5 bits and three
// derived bits the kernels use to stay on the fast path:
constexpr uint8_t kTypeMask = 0x1F;
constexpr uint8_t kBitOutletSrc = 0x20; // fluid cell that feeds a neighbouring outlet node
constexpr uint8_t kBitNearWall = 0x40;  // some neighbour x - c_i is a bounce-back node
constexpr uint8_t kBitLink = 0x80;      // cell has moving-boundary links this step

// bounce-back node types: FsiCoupling2D.cu:171-176, FsiCoupling3D.cu:209-216
template <int DIM> __host__ __device__ inline bool is_bounce_back(uint32_t t)
{
    uint32_t m = (1u << kSolid) | (1u << kWall) | (1u << kWallLeft) | (1u << kWallRight) | (1u << kWallUp) | (1u << kWallDown);
    if (DIM == 3) m |= (1u << kWallFront) | (1u << kWallBack);
    return t < 32 && ((m >> t) & 1u);
}

__host__ __device__ inline bool is_updated(uint32_t t) { return t == kFluid || t == kSolidDynamic; }

// ------------------------------------------------------------ status bits
enum StatusBits : uint32_t {
    kStatusNonFinite = 1u << 0,     // a fluid update produced a non-finite density
    kStatusLinkOverflow = 1u << 1,  // link hash table full; some links were dropped
    kStatusForceRange = 1u << 2,    // a force contribution exceeded the fixed-point range
    kStatusBadElement = 1u << 3,    // element index out of range in the surface
    kStatusStageTimeout = 1u << 4,  // a staged plane of moments did not arrive within the wait limit
};

// A post-collision state the step cannot continue from: density not
// positive, or a non-finite density or velocity.  (Populations are clamped
// with max(0, f) before the moments are formed, which turns a NaN population
// into 0, so a poisoned neighbour shows up as a vanishing or infinite
// density rather than as a NaN.)
template <int DIM> __device__ __forceinline__ bool bad_state(const float *m)
{
    float s = m[0] + m[1] + m[2];
    if (DIM == 3) s += m[3];
    return !(m[0] > 0.0f) || !isfinite(s);
}

// ---------------------------------------------------------------- storage
enum Storage : int { kF32 = 0, kF16 = 1, kBF16 = 2 };

// Reduced-precision storage keeps scaled deviations from equilibrium:
//   rho - 1,  u * su,  (pi_ab - u_a u_b) * sp
// su and sp are powers of two, so scaling is exact; decode(encode(x)) loses
// only the 11-bit (fp16) or 8-bit (bf16) rounding of the deviation (the
// velocity of bf16 storage is kept in binary16: StorageTraits below).
struct Codec {
    float su, inv_su, sp, inv_sp;
};

template <typename T> struct StorageTraits;
// to/from: one stored value of the storage type.  to_vel/from_vel: a stored
// velocity (u * su).  FP32 and FP16 storage keep the velocity like every
// other moment; bfloat16 storage keeps it as a binary16 bit pattern in its
// 16-bit slot, because an 8-bit significand rounds the per-step velocity
// changes of slow flows away (a Taylor-Green vortex at u = 0.04 changes u by
// about 1e-5 per step, below half an ulp of u * 16 in bfloat16), while rho - 1
// and the stress deviations keep bfloat16's range.
template <> struct StorageTraits<float> {
    static constexpr bool kEncoded = false;
    __device__ static float to(float v) { return v; }
    __device__ static float from(float v) { return v; }
    __device__ static float to_vel(float v) { return v; }
    __device__ static float from_vel(float v) { return v; }
};
template <> struct StorageTraits<__half> {
    static constexpr bool kEncoded = true;
    __device__ static __half to(float v) { return __float2half_rn(v); }
    __device__ static float from(__half v) { return __half2float(v); }
    __device__ static __half to_vel(float v) { return __float2half_rn(v); }
    __device__ static float from_vel(__half v) { return __half2float(v); }
};
template <> struct StorageTraits<__nv_bfloat16> {
    static constexpr bool kEncoded = true;
    __device__ static __nv_bfloat16 to(float v) { return __float2bfloat16_rn(v); }
    __device__ static float from(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static __nv_bfloat16 to_vel(float v)
    {
        return __ushort_as_bfloat16(__half_as_ushort(__float2half_rn(v)));
    }
    __device__ static float from_vel(__nv_bfloat16 v) { return __half2float(__ushort_as_half(__bfloat16_as_ushort(v))); }
};

// Conversion of moment k of a stored vector ([rho, u_1..u_DIM, pi...]): the
// velocity moments through to_vel/from_vel, the others through to/from.
template <int DIM, typename T> __device__ __forceinline__ float from_storage(int k, T v)
{
    return (k >= 1 && k <= DIM) ? StorageTraits<T>::from_vel(v) : StorageTraits<T>::from(v);
}
template <int DIM, typename T> __device__ __forceinline__ T to_storage(int k, float v)
{
    return (k >= 1 && k <= DIM) ? StorageTraits<T>::to_vel(v) : StorageTraits<T>::to(v);
}

// Index of pi_ab in the moment vector and the (a, b) pair of each stored
// second moment, for the encoding above.
template <int DIM> struct MomentLayout;
template <> struct MomentLayout<2> {
    // [rho, ux, uy, pixx, piyy, pixy]
    static __host__ __device__ constexpr int pa(int k) { return k == 3 ? 0 : (k == 4 ? 1 : 0); }
    static __host__ __device__ constexpr int pb(int k) { return k == 3 ? 0 : (k == 4 ? 1 : 1); }
};
template <> struct MomentLayout<3> {
    // [rho, ux, uy, uz, pixx, piyy, pizz, pixy, piyz, pixz]
    static __host__ __device__ constexpr int pa(int k) { return k == 4 ? 0 : k == 5 ? 1 : k == 6 ? 2 : k == 7 ? 0 : k == 8 ? 1 : 0; }
    static __host__ __device__ constexpr int pb(int k) { return k == 4 ? 0 : k == 5 ? 1 : k == 6 ? 2 : k == 7 ? 1 : k == 8 ? 2 : 2; }
};

// Decode a stored moment vector (already loaded as floats) in place.
template <int DIM, typename T>
__device__ __forceinline__ void decode_moments(float *m, const Codec &c)
{
    if constexpr (StorageTraits<T>::kEncoded) {
        constexpr int NM = Lattice<DIM>::NM;
        m[0] = 1.0f + m[0];
#pragma unroll
        for (int a = 0; a < DIM; ++a) m[1 + a] *= c.inv_su;
#pragma unroll
        for (int k = DIM + 1; k < NM; ++k)
            m[k] = fmaf(m[k], c.inv_sp, m[1 + MomentLayout<DIM>::pa(k)] * m[1 + MomentLayout<DIM>::pb(k)]);
    }
}

// Stochastic rounding of the stored velocity.  With round-to-nearest, a
// velocity whose per-step change is below half an ulp of its 11-bit
// significand never changes in storage: a Taylor-Green vortex on 128^3 cells
// (u ~ 0.04, relative decay 4e-5 per step) stalls that way.  Rounding up with
// the probability given by the position between the two neighbouring binary16
// values keeps the stored velocity unbiased, so slow changes accumulate.
// The dither is a hash of the cell index and of the bits of the cell's new
// density, so a cell's encoding depends only on what it stores (every kernel
// that writes a cell gives the same bits) and changes from step to step.
// lowbias32 (C. Wellons, "Prospecting for Hash Functions", 2018): an integer
// mixing function with good avalanche.
__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t vel_dither(size_t idx, float rho)
{
    return mix32((uint32_t)idx * 0x9e3779b9u ^ (uint32_t)((uint64_t)idx >> 32) ^ __float_as_uint(rho));
}
// v rounded to binary16 stochastically with 10 random bits r: adding r << 3
// to the magnitude bits of the float and truncating the 13 bits binary16
// does not keep rounds up with probability (dropped bits) / 2^13, to within
// 2^-10 of an ulp; values below binary16's normal range (2^-14) or at its
// top round to nearest.  `back` receives the value the result represents:
// in range, the truncated float itself (it has binary16's 11 significant
// bits, so the conversion is exact), which saves converting back.  The add
// goes to the whole float: below the top of the range the magnitude cannot
// carry into the sign bit.
__device__ __forceinline__ __half half_sr(float v, uint32_t r, float &back)
{
    const uint32_t b = __float_as_uint(v), mag = b & 0x7fffffffu;
    if (mag < 0x38800000u || mag >= 0x47000000u) {
        const __half h = __float2half_rn(v);
        back = __half2float(h);
        return h;
    }
    back = __uint_as_float((b + (r << 3)) & ~0x1fffu);
    return __float2half_rn(back);
}
template <typename T> __device__ __forceinline__ T to_vel_sr(float v, uint32_t r, float &back);
template <> __device__ __forceinline__ float to_vel_sr<float>(float v, uint32_t, float &back)
{
    back = v;
    return v;
}
template <> __device__ __forceinline__ __half to_vel_sr<__half>(float v, uint32_t r, float &back)
{
    return half_sr(v, r, back);
}
template <> __device__ __forceinline__ __nv_bfloat16 to_vel_sr<__nv_bfloat16>(float v, uint32_t r, float &back)
{
    return __ushort_as_bfloat16(__half_as_ushort(half_sr(v, r, back)));
}

// The stored form of moment vector m of cell idx: FP32 as is; reduced
// storage as rho - 1, u * su (stochastically rounded) and the stress
// deviations from the rounded u, so that decoding reproduces pi up to the
// deviation's rounding.
template <int DIM, typename T>
__device__ __forceinline__ void encode_values(const float *m, size_t idx, const Codec &c, T *enc)
{
    constexpr int NM = Lattice<DIM>::NM;
    if constexpr (!StorageTraits<T>::kEncoded) {
#pragma unroll
        for (int k = 0; k < NM; ++k) enc[k] = m[k];
    } else {
        float ud[DIM];
        enc[0] = StorageTraits<T>::to(m[0] - 1.0f);
        const uint32_t h = vel_dither(idx, m[0]);
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            float back;
            enc[1 + a] = to_vel_sr<T>(m[1 + a] * c.su, (h >> (10 * a)) & 0x3ffu, back);
            ud[a] = back * c.inv_su;
        }
#pragma unroll
        for (int k = DIM + 1; k < NM; ++k)
            enc[k] = StorageTraits<T>::to(fmaf(-ud[MomentLayout<DIM>::pa(k)], ud[MomentLayout<DIM>::pb(k)], m[k]) * c.sp);
    }
}

// Encode m (floats) to storage at cell idx of the planes.
template <int DIM, typename T>
__device__ __forceinline__ void encode_store(const float *m, T *const *planes, uint32_t idx, const Codec &c)
{
    T enc[Lattice<DIM>::NM];
    encode_values<DIM, T>(m, idx, c, enc);
#pragma unroll
    for (int k = 0; k < Lattice<DIM>::NM; ++k) planes[k][idx] = enc[k];
}

// Same as encode_store with planes[k] = base + k * stride.
template <int DIM, typename T>
__device__ __forceinline__ void encode_store_strided(const float *m, T *base, size_t idx, size_t stride, const Codec &c)
{
    T enc[Lattice<DIM>::NM];
    encode_values<DIM, T>(m, idx, c, enc);
#pragma unroll
    for (int k = 0; k < Lattice<DIM>::NM; ++k) base[idx + k * stride] = enc[k];
}

// Same as encode_store with planes[k] = base + k * stride and a 32-bit index
// idx + k * stride (the caller guarantees it fits).
template <int DIM, typename T>
__device__ __forceinline__ void encode_store_idx32(const float *m, T *base, uint32_t idx, uint32_t stride,
                                                   const Codec &c)
{
    T enc[Lattice<DIM>::NM];
    encode_values<DIM, T>(m, idx, c, enc);
#pragma unroll
    for (int k = 0; k < Lattice<DIM>::NM; ++k) base[idx + (uint32_t)k * stride] = enc[k];
}

// The values encode_store writes for cell idx, as they read back: m itself
// for FP32, the decoded rounded deviations otherwise.
template <int DIM, typename T>
__device__ __forceinline__ void stored_values(const float *m, float *out, size_t idx, const Codec &c)
{
    constexpr int NM = Lattice<DIM>::NM;
    if constexpr (!StorageTraits<T>::kEncoded) {
#pragma unroll
        for (int k = 0; k < NM; ++k) out[k] = m[k];
    } else {
        T enc[NM];
        encode_values<DIM, T>(m, idx, c, enc);
        out[0] = 1.0f + StorageTraits<T>::from(enc[0]);
#pragma unroll
        for (int a = 0; a < DIM; ++a) out[1 + a] = StorageTraits<T>::from_vel(enc[1 + a]) * c.inv_su;
#pragma unroll
        for (int k = DIM + 1; k < NM; ++k) {
            const float ua = out[1 + MomentLayout<DIM>::pa(k)], ub = out[1 + MomentLayout<DIM>::pb(k)];
            out[k] = fmaf(StorageTraits<T>::from(enc[k]), c.inv_sp, ua * ub);
        }
    }
}

template <int DIM, typename T>
__device__ __forceinline__ void load_moments(float *m, const T *base, uint32_t ncell, uint32_t idx, const Codec &c)
{
    constexpr int NM = Lattice<DIM>::NM;
#pragma unroll
    for (int k = 0; k < NM; ++k) m[k] = from_storage<DIM, T>(k, base[(size_t)k * ncell + idx]);
    decode_moments<DIM, T>(m, c);
}

struct Vel6 {
    float v[6];
};

// --------------------------------------------------------- grid descriptor
// Everything one fluid grid's kernels need, passed by value.
// SMs of the current device: grid-stride launches are capped at a multiple of it.
inline int device_sms()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 1;
    return n;
}

// cp.async (LDGSTS): 4-byte global -> shared copies that hold no registers
// while in flight.  Both addresses must be 4-byte aligned.
__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
// 16-byte copy (L2 only); both addresses must be 16-byte aligned.
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// waits until at most N of this thread's committed groups are still in flight
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T> struct GridArgs {
    int nx, ny, nz;
    uint32_t ncell;
    int periodic;            // bit0 x, bit1 y, bit2 z wrap the pull halo (reference: clamp)
    int half_pops;           // D2Q9: round reconstructed populations to binary16 (reference tile)
    int wall_stream;         // D2Q9: walls stream their stored moments instead of bouncing back
                             // (the reference's 2D kernel, ffs_lbm_desc::ref_2d_wall_stream)
    float omega;
    Codec codec;
    const T *src;            // SoA: moment k of cell c at src[k * ncell + c]
    T *dst;
    const uint8_t *flags;
    const uint32_t *wallmask; // per-cell bounce-back direction mask (read only for near-wall cells)
    uint32_t *status;
};

} // namespace fflbm
