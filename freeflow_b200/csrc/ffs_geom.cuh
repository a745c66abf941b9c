// Link geometry of the moving-boundary bounce-back: segment/segment (2D) and
// segment/triangle (3D) intersection, barycentric weights, bounding boxes and
// the (depth, element) link key.
//
// Reference: include/FSI_Simulator/core/SolidGeometryProxy_Device.cuh
//   depthIndexCompact :79-85, line_intersect :89-124, 2D intersectAtIndex
//   :211-227, getBoundingBox :198-209 / :424-440, barycentric_coordinates
//   :291-304, line_triangle_intersect :306-341 (tolerance 1e-6,
//   include/FSI_Simulator/utils/NumericUtils.cuh:24).
//
// Every operation is an explicitly rounded IEEE op (__f*_rn), so nothing is
// contracted into an FMA: the link set a surface produces is then a pure
// function of its float inputs, bit-identical to the CPU oracle compiled
// with -ffp-contract=off.  A link that flips between "hit" and "miss" would
// otherwise change a whole population, not just its last bit.
#pragma once
#include "ffs_common.cuh"

namespace fflbm {
namespace geom {

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float sqr(float a) { return __fsqrt_rn(a); }

struct Hit {
    bool hit;
    float depth;
    float b[3];
};

// line_intersect: returns 1 - t1 (the hit's fraction along p1 -> p2) or -1.
__device__ __forceinline__ float line_isect(float x1, float y1, float x2, float y2, float x3, float y3, float x4,
                                            float y4, float &xo, float &yo)
{
    float a1 = sub(mul(sub(x1, x2), sub(y3, y4)), mul(sub(y1, y2), sub(x3, x4)));
    float b1 = sub(mul(sub(x4, x2), sub(y3, y4)), mul(sub(y4, y2), sub(x3, x4)));
    // t1 = b1 / a1 can only land in (0, 1) when b1 and a1 have the same sign,
    // b1 != 0 and |b1| < |a1|; every other case (a1 = 0 and NaN included)
    // ends in the -1 below as well, so reject it before dividing
    if (!(fabsf(b1) < fabsf(a1)) || b1 == 0.0f || ((b1 < 0.0f) != (a1 < 0.0f))) return -1.0f;
    if (fabsf(a1) <= 0.0f) return -1.0f;
    float t1 = dvd(b1, a1);
    if (t1 <= 0.0f || t1 >= 1.0f) return -1.0f;
    xo = add(mul(t1, x1), mul(sub(1.0f, t1), x2));
    if (mul(sub(x3, xo), sub(x4, xo)) < 0.0f) {
        yo = add(mul(t1, y1), mul(sub(1.0f, t1), y2));
        return sub(1.0f, t1);
    }
    return -1.0f;
}

// 2D intersectAtIndex: segment p1 -> p2 against element e (vertices a, b).
__device__ __forceinline__ Hit isect2(const float *V, uint32_t a, uint32_t b, float p1x, float p1y, float p2x,
                                      float p2y)
{
    Hit r;
    r.hit = false; r.depth = 0.0f; r.b[0] = r.b[1] = r.b[2] = 0.0f;
    float x3 = V[2 * a], y3 = V[2 * a + 1], x4 = V[2 * b], y4 = V[2 * b + 1];
    float xo = 0.0f, yo = 0.0f;
    float d = line_isect(p1x, p1y, p2x, p2y, x3, y3, x4, y4, xo, yo);
    if (d > 0.0f && d < 1.0f) {
        float dxh = sub(x4, xo), dyh = sub(y4, yo), dx34 = sub(x4, x3), dy34 = sub(y4, y3);
        float l1 = sqr(add(mul(dxh, dxh), mul(dyh, dyh)));
        float l2 = sqr(add(mul(dx34, dx34), mul(dy34, dy34)));
        r.hit = true;
        r.depth = d;
        r.b[0] = dvd(l1, l2);
        r.b[1] = sub(1.0f, r.b[0]);
    }
    return r;
}

__device__ __forceinline__ float dot3(const float *a, const float *b)
{
    return add(add(mul(a[0], b[0]), mul(a[1], b[1])), mul(a[2], b[2]));
}
__device__ __forceinline__ void cross3(const float *a, const float *b, float *o)
{
    o[0] = sub(mul(a[1], b[2]), mul(b[1], a[2]));
    o[1] = sub(mul(a[2], b[0]), mul(b[2], a[0]));
    o[2] = sub(mul(a[0], b[1]), mul(b[0], a[1]));
}
__device__ __forceinline__ void normalize3(float *v)
{
    float inv = dvd(1.0f, sqr(dot3(v, v)));
    v[0] = mul(v[0], inv); v[1] = mul(v[1], inv); v[2] = mul(v[2], inv);
}

// line_triangle_intersect + barycentric_coordinates for triangle (a, b, c).
__device__ __forceinline__ Hit isect3(const float *V, uint32_t ia, uint32_t ib, uint32_t ic, const float *p1,
                                      const float *p2)
{
    Hit r;
    r.hit = false; r.depth = 0.0f; r.b[0] = r.b[1] = r.b[2] = 0.0f;
    float v0[3], v1[3], v2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { v0[k] = V[3 * (size_t)ia + k]; v1[k] = V[3 * (size_t)ib + k]; v2[k] = V[3 * (size_t)ic + k]; }
    float e1[3], e2[3], n[3], d[3], w0[3], pd[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { e1[k] = sub(v1[k], v0[k]); e2[k] = sub(v2[k], v0[k]); }
    cross3(e1, e2, n);
    normalize3(n);
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = sub(p2[k], p1[k]);
    normalize3(d);
    float nd = dot3(n, d);
    if (fabsf(nd) <= 1e-6f) return r;
#pragma unroll
    for (int k = 0; k < 3; ++k) { w0[k] = sub(v0[k], p1[k]); pd[k] = sub(p2[k], p1[k]); }
    float t = dvd(dot3(n, w0), dot3(n, pd));
    if (t < 0.0f || t > 1.0f) return r;
    float w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) w[k] = sub(add(p1[k], mul(t, pd[k])), v0[k]);
    float d00 = dot3(e1, e1), d01 = dot3(e1, e2), d11 = dot3(e2, e2);
    float d20 = dot3(w, e1), d21 = dot3(w, e2);
    float den = sub(mul(d00, d11), mul(d01, d01));
    float u0 = dvd(sub(mul(d11, d20), mul(d01, d21)), den);
    float vv = dvd(sub(mul(d00, d21), mul(d01, d20)), den);
    if (u0 >= -1e-6f && vv >= -1e-6f && add(u0, vv) <= 1.0f + 1e-6f) {
        r.hit = true;
        r.depth = t;
        r.b[0] = sub(sub(1.0f, u0), vv);
        r.b[1] = u0;
        r.b[2] = vv;
    }
    return r;
}

// Per-triangle part of isect3: everything that depends only on the
// triangle, evaluated with exactly the same operations, so isect3_pre()
// returns bit-identical results to isect3() while doing it once per triangle.
struct TriPre {
    float v0[3], e1[3], e2[3], n[3];
    float d00, d01, d11, den;
};

__device__ __forceinline__ TriPre tri_pre(const float *V, uint32_t ia, uint32_t ib, uint32_t ic)
{
    TriPre t;
    float v1[3], v2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { t.v0[k] = V[3 * (size_t)ia + k]; v1[k] = V[3 * (size_t)ib + k]; v2[k] = V[3 * (size_t)ic + k]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) { t.e1[k] = sub(v1[k], t.v0[k]); t.e2[k] = sub(v2[k], t.v0[k]); }
    cross3(t.e1, t.e2, t.n);
    normalize3(t.n);
    t.d00 = dot3(t.e1, t.e1);
    t.d01 = dot3(t.e1, t.e2);
    t.d11 = dot3(t.e2, t.e2);
    t.den = sub(mul(t.d00, t.d11), mul(t.d01, t.d01));
    return t;
}

__device__ __forceinline__ Hit isect3_pre(const TriPre &tr, const float *p1, const float *p2)
{
    Hit r;
    r.hit = false; r.depth = 0.0f; r.b[0] = r.b[1] = r.b[2] = 0.0f;
    float d[3], w0[3], pd[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = sub(p2[k], p1[k]);
    normalize3(d);
    float nd = dot3(tr.n, d);
    if (fabsf(nd) <= 1e-6f) return r;
#pragma unroll
    for (int k = 0; k < 3; ++k) { w0[k] = sub(tr.v0[k], p1[k]); pd[k] = sub(p2[k], p1[k]); }
    float t = dvd(dot3(tr.n, w0), dot3(tr.n, pd));
    if (t < 0.0f || t > 1.0f) return r;
    float w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) w[k] = sub(add(p1[k], mul(t, pd[k])), tr.v0[k]);
    float d20 = dot3(w, tr.e1), d21 = dot3(w, tr.e2);
    float u0 = dvd(sub(mul(tr.d11, d20), mul(tr.d01, d21)), tr.den);
    float vv = dvd(sub(mul(tr.d00, d21), mul(tr.d01, d20)), tr.den);
    if (u0 >= -1e-6f && vv >= -1e-6f && add(u0, vv) <= 1.0f + 1e-6f) {
        r.hit = true;
        r.depth = t;
        r.b[0] = sub(sub(1.0f, u0), vv);
        r.b[1] = u0;
        r.b[2] = vv;
    }
    return r;
}

// depthIndexCompact widened to 64 bits: (uint32(depth * 2^15) << 32) | element.
// Orders exactly like the reference's 32-bit key for up to 65536 elements.
__device__ __forceinline__ unsigned long long link_key(float depth, uint32_t e)
{
    uint32_t dq = __float2uint_rz(mul(depth, 32768.0f));
    return ((unsigned long long)dq << 32) | e;
}

} // namespace geom
} // namespace fflbm
