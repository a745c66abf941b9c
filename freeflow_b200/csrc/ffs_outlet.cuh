// Zero-gradient outlets, fused into the fluid update.
//
// The reference runs a separate full-grid kernel after the buffer swap
// (mrApplyOutlet2DKernel, FsiCoupling2D.cu:257-316; mrApplyOutlet3DKernel,
// FsiCoupling3D.cu:336-420): an outlet node q copies the normal velocity of its
// inner neighbour p = q - n (a Fluid node) when that velocity points outward,
// and sets pi_nn = u_n(p)^2, in place on the freshly written buffer.  Each
// outlet has exactly one feeder p, and p's new moments are final once p is
// updated, so the same writes are issued here by the thread that updates p,
// straight into the buffer being written.  No other node reads q's entries
// of that buffer during the step, so the result is the reference's.
#pragma once
#include "ffs_common.cuh"

namespace fflbm {

struct OutletRule {
    uint8_t type;   // outlet flag of the node q fed by this cell
    int comp;       // normal velocity component in the moment vector
    int pcomp;      // pi_nn index
    int sign;       // +1: copy when u_n > 0, -1: copy when u_n < 0
};

// q = p + offset(rule) for the six / four outlet types
template <int DIM> __device__ __forceinline__ long long outlet_offset(int r, int nx, long long nxy)
{
    if (DIM == 2) {
        switch (r) {
        case 0: return nx;   // OutletUp   : p = q - nx
        case 1: return -nx;  // OutletDown : p = q + nx
        case 2: return -1;   // OutletLeft : p = q + 1
        default: return 1;   // OutletRight: p = q - 1
        }
    } else {
        switch (r) {
        case 0: return nxy;  // OutletUp   (z)
        case 1: return -nxy; // OutletDown
        case 2: return -1;   // OutletLeft
        case 3: return 1;    // OutletRight
        case 4: return -nx;  // OutletFront: p = q + nx
        default: return nx;  // OutletBack : p = q - nx
        }
    }
}

template <int DIM> __device__ __forceinline__ OutletRule outlet_rule(int r)
{
    if (DIM == 2) {
        switch (r) {
        case 0: return {kOutletUp, 2, 4, 1};
        case 1: return {kOutletDown, 2, 4, -1};
        case 2: return {kOutletLeft, 1, 3, -1};
        default: return {kOutletRight, 1, 3, 1};
        }
    } else {
        switch (r) {
        case 0: return {kOutletUp, 3, 6, 1};
        case 1: return {kOutletDown, 3, 6, -1};
        case 2: return {kOutletLeft, 1, 4, -1};
        case 3: return {kOutletRight, 1, 4, 1};
        case 4: return {kOutletFront, 2, 5, -1};
        default: return {kOutletBack, 2, 5, 1};
        }
    }
}

template <int DIM> constexpr int kNumOutletRules = DIM == 2 ? 4 : 6;

// Outlet rules a cell feeds, kept in the spare bits of its wall-mask word
// (bit i < Q of that word is the bounce-back mask of direction i; bit 0 is
// never a wall because direction 0 does not move):
//   D2Q9 : rules 0..3 at bits 16..19;  D3Q27: rules 0..4 at bits 27..31, rule 5 at bit 0.
template <int DIM> __host__ __device__ constexpr uint32_t outlet_bit(int r)
{
    return DIM == 2 ? (1u << (16 + r)) : (r < 5 ? (1u << (27 + r)) : 1u);
}
template <int DIM> __host__ __device__ constexpr uint32_t outlet_bits_mask()
{
    return DIM == 2 ? 0xF0000u : 0xF8000001u;
}
template <int DIM> __host__ __device__ constexpr uint32_t wall_bits_mask()
{
    return DIM == 2 ? 0x1FEu : 0x07FFFFFEu;
}

// Called by the thread that has just stored cell p's new moments into g.dst.
// `ms` are the stored values as they read back (after storage rounding) and
// `word` the cell's mask word, whose outlet bits name the outlet neighbours
// q = p + offset(rule) to update.  No flag or moment of p is re-read.
template <int DIM, typename T>
__device__ __forceinline__ void feed_outlets(const GridArgs<T> &g, uint32_t p, const float *ms, uint32_t word)
{
    constexpr int NM = Lattice<DIM>::NM;
    const long long nxy = (long long)g.nx * g.ny;
#pragma unroll
    for (int r = 0; r < kNumOutletRules<DIM>; ++r) {
        if (!(word & outlet_bit<DIM>(r))) continue;
        const uint32_t q = (uint32_t)((long long)p + outlet_offset<DIM>(r, g.nx, nxy));
        const OutletRule rule = outlet_rule<DIM>(r);
        float up = 0.0f;
#pragma unroll
        for (int k = 0; k < NM; ++k)
            if (k == rule.comp) up = ms[k];
        const bool outward = (rule.sign > 0 && up > 0.0f) || (rule.sign < 0 && up < 0.0f);
        if constexpr (!StorageTraits<T>::kEncoded) {
            if (outward) g.dst[(size_t)rule.comp * g.ncell + q] = up;
            g.dst[(size_t)rule.pcomp * g.ncell + q] = up * up;
        } else {
            float mq[NM];
            load_moments<DIM, T>(mq, g.dst, g.ncell, q, g.codec);
#pragma unroll
            for (int k = 0; k < NM; ++k) {
                if (k == rule.comp && outward) mq[k] = up;
                if (k == rule.pcomp) mq[k] = up * up;
            }
            encode_store_strided<DIM, T>(mq, g.dst, q, g.ncell, g.codec);
        }
    }
}

} // namespace fflbm
