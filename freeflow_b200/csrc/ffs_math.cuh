// Moment-space math of the fluid step: third-order Hermite reconstruction of
// populations from moments, raw moments of populations, and the moment-space
// collision with re-encoding.
//
// Reference semantics (FreeFlow):
//   reconstruction  src/lbm/LbmUtilsFunc.cu:212-335 (D3Q27), :476-510 (D2Q9)
//   collision       src/lbm/LbmUtilsFunc.cu:337-414 (D3Q27), :512-543 (D2Q9)
//   re-encode       src/core/FsiCoupling2D.cu:243-252, src/core/FsiCoupling3D.cu:310-320
//
// The reference writes every population as its own explicit sum.  Here the
// expansion is evaluated as what it is, a tensor product of the 1D basis
// {1, c, g(c)} with g(+-1) = 1, g(0) = -1/2 and weights w(0) = 2/3,
// w(+-1) = 1/6: the coefficient A_pqr multiplies phi_p(cx) phi_q(cy) phi_r(cz),
// so the 27 (9) populations come out of three (two) small 1D passes, and the
// raw moments go back through the matching forward passes.  The results equal
// the reference's up to FP32 rounding order.
#pragma once
#include "ffs_common.cuh"
#include "ffs_f2.cuh"

namespace fflbm {

// v[0..2] = a0 + a1*c + a2*g(c) at c = -1, 0, +1
__device__ __forceinline__ void herm3(float a0, float a1, float a2, float *v)
{
    float t = a0 + a2;
    v[0] = t - a1;
    v[1] = fmaf(-0.5f, a2, a0);
    v[2] = t + a1;
}
// v[0..2] = a0 + a1*c at c = -1, 0, +1
__device__ __forceinline__ void herm2(float a0, float a1, float *v)
{
    v[0] = a0 - a1;
    v[1] = a0;
    v[2] = a0 + a1;
}

// Lattice weights, one float constant per population class, as the reference
// writes them (LbmConstants.hpp:28-35, :51-54): the number of non-zero
// velocity components selects 4/9, 1/9, 1/36 (D2Q9) or 8/27, 2/27, 1/54,
// 1/216 (D3Q27).  They equal the products of the 1D weights 2/3 and 1/6, but
// the products of the rounded 1D weights sum to 1 + 1.1e-7 over the 27
// directions, which would add that fraction of the mass every step; these
// sum to 1 + 7e-9.
__host__ __device__ constexpr float wgt2(int kx, int ky)
{
    return ((kx != 1) + (ky != 1)) == 0 ? 4.0f / 9.0f : ((kx != 1) + (ky != 1)) == 1 ? 1.0f / 9.0f : 1.0f / 36.0f;
}
__host__ __device__ constexpr float wgt3(int kx, int ky, int kz)
{
    return ((kx != 1) + (ky != 1) + (kz != 1)) == 0   ? 8.0f / 27.0f
           : ((kx != 1) + (ky != 1) + (kz != 1)) == 1 ? 2.0f / 27.0f
           : ((kx != 1) + (ky != 1) + (kz != 1)) == 2 ? 1.0f / 54.0f
                                                      : 1.0f / 216.0f;
}

// Hermite coefficients of one cell (the reference's m1, m2 and Q terms).
template <int DIM> struct Coef;

template <> struct Coef<2> {
    float rho, m1x, m1y, m2xx, m2yy, m2xy, qxxy, qxyy;
    // m = [rho, ux, uy, pixx, piyy, pixy]; the D2Q9 reference omits rho on
    // the pi terms of Q (LbmUtilsFunc.cu:488-490).
    __device__ __forceinline__ void make(const float *m)
    {
        float r = m[0], ux = m[1], uy = m[2], pxx = m[3], pyy = m[4], pxy = m[5];
        float r3 = 3.0f * r;
        rho = r;
        m1x = r3 * ux; m1y = r3 * uy;
        m2xx = r3 * pxx; m2yy = r3 * pyy; m2xy = 9.0f * r * pxy;
        float rux = r * ux, ruy = r * uy;
        qxxy = 9.0f * fmaf(pxx, uy, 2.0f * ux * (pxy - rux * uy));
        qxyy = 9.0f * fmaf(pyy, ux, 2.0f * uy * (pxy - ruy * ux));
    }
    // all nine populations, reference numbering
    __device__ __forceinline__ void populations(float *f) const
    {
        float C0[3], C1[3], C2[3];
        herm3(rho, m1y, m2yy, C0);
        herm3(m1x, m2xy, qxyy, C1);
        herm2(m2xx, qxxy, C2);
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            float F[3];
            herm3(C0[ky], C1[ky], C2[ky], F);
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const int i = dir_index<2>(kx, ky, 1);
                f[i] = wgt2(kx, ky) * F[kx];
            }
        }
    }
    // one population, direction given at run time
    __device__ __forceinline__ float population(int cx, int cy, int) const
    {
        float gx = cx ? 1.0f : -0.5f, gy = cy ? 1.0f : -0.5f;
        float fx = (float)cx, fy = (float)cy;
        float s = rho;
        s = fmaf(m1x, fx, s); s = fmaf(m1y, fy, s);
        s = fmaf(m2xx, gx, s); s = fmaf(m2yy, gy, s);
        s = fmaf(m2xy, fx * fy, s);
        s = fmaf(qxxy, gx * fy, s); s = fmaf(qxyy, fx * gy, s);
        const float w = wgt2(cx + 1, cy + 1);
        return w * s;
    }
};

template <> struct Coef<3> {
    float rho, m1x, m1y, m1z, m2xx, m2yy, m2zz, m2xy, m2yz, m2xz;
    float qxxy, qxyy, qxxz, qxzz, qyyz, qyzz, qxyz;
    // m = [rho, ux, uy, uz, pixx, piyy, pizz, pixy, piyz, pixz]
    __device__ __forceinline__ void make(const float *m)
    {
        float r = m[0], ux = m[1], uy = m[2], uz = m[3];
        float pxx = m[4], pyy = m[5], pzz = m[6], pxy = m[7], pyz = m[8], pxz = m[9];
        float r3 = 3.0f * r, r9 = 9.0f * r;
        rho = r;
        m1x = r3 * ux; m1y = r3 * uy; m1z = r3 * uz;
        m2xx = r3 * pxx; m2yy = r3 * pyy; m2zz = r3 * pzz;
        m2xy = r9 * pxy; m2yz = r9 * pyz; m2xz = r9 * pxz;
        // Q_aab = 9 rho (pi_aa u_b + 2 u_a (pi_ab - u_a u_b))
        float dxy = fmaf(-ux, uy, pxy), dyz = fmaf(-uy, uz, pyz), dxz = fmaf(-ux, uz, pxz);
        float r18 = 2.0f * r9;
        qxxy = fmaf(r9 * pxx, uy, r18 * ux * dxy);
        qxyy = fmaf(r9 * pyy, ux, r18 * uy * dxy);
        qxxz = fmaf(r9 * pxx, uz, r18 * ux * dxz);
        qxzz = fmaf(r9 * pzz, ux, r18 * uz * dxz);
        qyyz = fmaf(r9 * pyy, uz, r18 * uy * dyz);
        qyzz = fmaf(r9 * pzz, uy, r18 * uz * dyz);
        // Q_xyz = 27 rho (pi_xy uz + pi_yz ux + pi_xz uy - 2 ux uy uz)
        float t = fmaf(pxy, uz, fmaf(pyz, ux, pxz * uy));
        qxyz = 27.0f * r * fmaf(-2.0f * ux * uy, uz, t);
    }
    __device__ __forceinline__ float population(int cx, int cy, int cz) const
    {
        float gx = cx ? 1.0f : -0.5f, gy = cy ? 1.0f : -0.5f, gz = cz ? 1.0f : -0.5f;
        float fx = (float)cx, fy = (float)cy, fz = (float)cz;
        float s = rho;
        s = fmaf(m1x, fx, s); s = fmaf(m1y, fy, s); s = fmaf(m1z, fz, s);
        s = fmaf(m2xx, gx, s); s = fmaf(m2yy, gy, s); s = fmaf(m2zz, gz, s);
        s = fmaf(m2xy, fx * fy, s); s = fmaf(m2yz, fy * fz, s); s = fmaf(m2xz, fx * fz, s);
        s = fmaf(qxxy, gx * fy, s); s = fmaf(qxyy, fx * gy, s);
        s = fmaf(qxxz, gx * fz, s); s = fmaf(qxzz, fx * gz, s);
        s = fmaf(qyyz, gy * fz, s); s = fmaf(qyzz, fy * gz, s);
        s = fmaf(qxyz, fx * fy * fz, s);
        const float w = wgt3(cx + 1, cy + 1, cz + 1);
        return w * s;
    }
};

// D3Q27 reconstruction generic in the arithmetic type: V = float (one cell)
// or V = f2 (two cells per thread, packed FP32 pairs).
template <typename V> __device__ __forceinline__ void herm3v(V a0, V a1, V a2, V *v)
{
    V t = a0 + a2;
    v[0] = t - a1;
    v[1] = vfma(vconst<V>(-0.5f), a2, a0);
    v[2] = t + a1;
}
template <typename V> __device__ __forceinline__ void herm2v(V a0, V a1, V *v)
{
    v[0] = a0 - a1;
    v[1] = a0;
    v[2] = a0 + a1;
}

template <typename V> struct Coef3V {
    V rho, m1x, m1y, m1z, m2xx, m2yy, m2zz, m2xy, m2yz, m2xz;
    V qxxy, qxyy, qxxz, qxzz, qyyz, qyzz, qxyz;
    // same expressions as Coef<3>::make
    __device__ __forceinline__ void make(const V *m)
    {
        V r = m[0], ux = m[1], uy = m[2], uz = m[3];
        V pxx = m[4], pyy = m[5], pzz = m[6], pxy = m[7], pyz = m[8], pxz = m[9];
        V r3 = vconst<V>(3.0f) * r, r9 = vconst<V>(9.0f) * r;
        rho = r;
        m1x = r3 * ux; m1y = r3 * uy; m1z = r3 * uz;
        m2xx = r3 * pxx; m2yy = r3 * pyy; m2zz = r3 * pzz;
        m2xy = r9 * pxy; m2yz = r9 * pyz; m2xz = r9 * pxz;
        V zero = vconst<V>(0.0f);
        V dxy = vfma(zero - ux, uy, pxy), dyz = vfma(zero - uy, uz, pyz), dxz = vfma(zero - ux, uz, pxz);
        V r18 = vconst<V>(2.0f) * r9;
        qxxy = vfma(r9 * pxx, uy, r18 * ux * dxy);
        qxyy = vfma(r9 * pyy, ux, r18 * uy * dxy);
        qxxz = vfma(r9 * pxx, uz, r18 * ux * dxz);
        qxzz = vfma(r9 * pzz, ux, r18 * uz * dxz);
        qyyz = vfma(r9 * pyy, uz, r18 * uy * dyz);
        qyzz = vfma(r9 * pzz, uy, r18 * uz * dyz);
        V t = vfma(pxy, uz, vfma(pyz, ux, pxz * uy));
        qxyz = vconst<V>(27.0f) * r * vfma(vconst<V>(-2.0f) * ux * uy, uz, t);
    }
    // Evaluates the 27 populations slice by slice and hands each one to
    // sink(kz, ky, kx, value) as soon as it exists (k = c + 1), which keeps
    // register pressure low when the sink stores to shared memory.  With
    // WEIGHTED = false the values are the Hermite sums without their lattice
    // weights (the caller applies the weights).
    template <bool WEIGHTED = true, typename Sink> __device__ __forceinline__ void populations_each(Sink &&sink) const
    {
        V B00[3], B10[3], B01[3], B20[3], B02[3], B11[3];
        herm3v(rho, m1z, m2zz, B00);
        herm3v(m1x, m2xz, qxzz, B10);
        herm3v(m1y, m2yz, qyzz, B01);
        herm2v(m2xx, qxxz, B20);
        herm2v(m2yy, qyyz, B02);
        herm2v(m2xy, qxyz, B11);
#pragma unroll
        for (int kz = 0; kz < 3; ++kz) {
            V C0[3], C1[3], C2[3];
            herm3v(B00[kz], B01[kz], B02[kz], C0);
            herm3v(B10[kz], B11[kz], qxyy, C1);
            herm2v(B20[kz], qxxy, C2);
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                V F[3];
                herm3v(C0[ky], C1[ky], C2[ky], F);
#pragma unroll
                for (int kx = 0; kx < 3; ++kx) {
                    if constexpr (WEIGHTED) sink(kz, ky, kx, vconst<V>(wgt3(kx, ky, kz)) * F[kx]);
                    else sink(kz, ky, kx, F[kx]);
                }
            }
        }
    }
    // Only the 9 unweighted populations with c_y = KY - 1 (what a halo row
    // outside a tile feeds into it), as sink(kz, kx, value), each
    // bit-identical to populations_each<false>'s.
    template <int KY, typename Sink> __device__ __forceinline__ void populations_row(Sink &&sink) const
    {
        V B00[3], B10[3], B01[3], B20[3], B02[3], B11[3];
        herm3v(rho, m1z, m2zz, B00);
        herm3v(m1x, m2xz, qxzz, B10);
        herm3v(m1y, m2yz, qyzz, B01);
        herm2v(m2xx, qxxz, B20);
        herm2v(m2yy, qyyz, B02);
        herm2v(m2xy, qxyz, B11);
        // entry KY of herm3v / herm2v, with herm3v's operations
        auto h3 = [](V a0, V a1, V a2) {
            if constexpr (KY == 1) return vfma(vconst<V>(-0.5f), a2, a0);
            else if constexpr (KY == 0) return (a0 + a2) - a1;
            else return (a0 + a2) + a1;
        };
        auto h2 = [](V a0, V a1) {
            if constexpr (KY == 1) return a0;
            else if constexpr (KY == 0) return a0 - a1;
            else return a0 + a1;
        };
#pragma unroll
        for (int kz = 0; kz < 3; ++kz) {
            V F[3];
            herm3v(h3(B00[kz], B01[kz], B02[kz]), h3(B10[kz], B11[kz], qxyy), h2(B20[kz], qxxy), F);
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) sink(kz, kx, F[kx]);
        }
    }
    // Only the 9 unweighted populations with c_x = sx (+1 or -1, given at run
    // time: what a halo column outside a tile feeds into it), as
    // sink(kz, ky, value), each bit-identical to populations_each<false>'s
    // (herm3v's outer entries are (a0 + a2) -+ a1 = fma(-+1, a1, a0 + a2)).
    template <typename Sink> __device__ __forceinline__ void populations_col(V sx, Sink &&sink) const
    {
        V B00[3], B10[3], B01[3], B20[3], B02[3], B11[3];
        herm3v(rho, m1z, m2zz, B00);
        herm3v(m1x, m2xz, qxzz, B10);
        herm3v(m1y, m2yz, qyzz, B01);
        herm2v(m2xx, qxxz, B20);
        herm2v(m2yy, qyyz, B02);
        herm2v(m2xy, qxyz, B11);
#pragma unroll
        for (int kz = 0; kz < 3; ++kz) {
            V C0[3], C1[3], C2[3];
            herm3v(B00[kz], B01[kz], B02[kz], C0);
            herm3v(B10[kz], B11[kz], qxyy, C1);
            herm2v(B20[kz], qxxy, C2);
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) sink(kz, ky, vfma(sx, C1[ky], C0[ky] + C2[ky]));
        }
    }
};

// ------------------------------------------------------------ raw moments
// R = {rho, jx, jy[, jz], Pxx, Pyy[, Pzz], Pxy[, Pyz, Pxz]} (raw sums)
__device__ __forceinline__ void raw_moments2(const float *f, float *R)
{
    // rows by cy: (f(-1), f(0), f(+1))
    float s0 = f[1] + f[3], d0 = f[1] - f[3], x00 = f[0] + s0;   // cy = 0
    float s1 = f[5] + f[6], d1 = f[5] - f[6], x01 = f[2] + s1;   // cy = +1
    float sm = f[8] + f[7], dm = f[8] - f[7], x0m = f[4] + sm;   // cy = -1
    float sy = x01 + x0m;
    R[0] = x00 + sy;            // rho
    R[1] = d0 + (d1 + dm);      // jx
    R[2] = x01 - x0m;           // jy
    R[3] = s0 + (s1 + sm);      // Pxx
    R[4] = sy;                  // Pyy
    R[5] = d1 - dm;             // Pxy
}

// ------------------------------------------------------------- collision
// Input: raw moments R (see above).  Output: the stored moment vector
// [rho, u, pi] with pi = Pi'/rho - c_s^2 delta, where Pi' is the relaxed
// second moment of LbmUtilsFunc.cu:337-414 / :512-543 (body force is zero on
// this path: FsiCoupling2D.cu:227-228; the 3D body-force field is never set,
// LbmFlowField3D.cpp:85-86).  Written in the algebraically equal form
// pi' = (dev * (1 - omega) / rho) + equilibrium part, which avoids
// subtracting c_s^2 from a value near c_s^2.
// 1 / rho from the hardware approximation refined by one Newton step (within
// an ulp of the IEEE quotient, without the division's slow-path branch)
__device__ __forceinline__ float recip(float x)
{
    float r = __fdividef(1.0f, x);
    return r * fmaf(-x, r, 2.0f);
}

__device__ __forceinline__ void collide2(const float *R, float omega, float *m)
{
    float rho = R[0];
    float ir = recip(rho);
    float ux = R[1] * ir, uy = R[2] * ir;
    float omw = 1.0f - omega;
    float ux2 = ux * ux, uy2 = uy * uy;
    float half_u2 = 0.5f * (ux2 + uy2);
    float dev = 0.5f * (R[3] - R[4]) * omw * ir;
    float an = 0.5f * omega * (ux2 - uy2);
    m[0] = rho; m[1] = ux; m[2] = uy;
    m[3] = half_u2 + dev + an;
    m[4] = half_u2 - dev - an;
    m[5] = fmaf(omw * R[5], ir, omega * ux * uy);
}

__device__ __forceinline__ void collide3(const float *R, float omega, float *m)
{
    const float third = 1.0f / 3.0f;
    float rho = R[0];
    float ir = recip(rho);
    float ux = R[1] * ir, uy = R[2] * ir, uz = R[3] * ir;
    float omw = 1.0f - omega;
    float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    float u2_3 = (ux2 + uy2 + uz2) * third;
    float tr_3 = (R[4] + R[5] + R[6]) * third;
    float k = omw * ir;
    m[0] = rho; m[1] = ux; m[2] = uy; m[3] = uz;
    // pi'_aa = u^2/3 + (1-w)(P_aa - tr/3)/rho + w (u_a^2 - u^2/3)
    m[4] = fmaf(k, R[4] - tr_3, fmaf(omega, ux2 - u2_3, u2_3));
    m[5] = fmaf(k, R[5] - tr_3, fmaf(omega, uy2 - u2_3, u2_3));
    m[6] = fmaf(k, R[6] - tr_3, fmaf(omega, uz2 - u2_3, u2_3));
    // pi'_ab = (1-w) P_ab / rho + w u_a u_b
    m[7] = fmaf(k, R[7], omega * ux * uy);
    m[8] = fmaf(k, R[8], omega * uy * uz);
    m[9] = fmaf(k, R[9], omega * ux * uz);
}

__device__ __forceinline__ float round_half(float v) { return __half2float(__float2half_rn(v)); }

} // namespace fflbm
