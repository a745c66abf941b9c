/*
 * CPU oracle for the moment-encoded LBM fluid step -- TEST INFRASTRUCTURE ONLY.
 * Only the tests, the smoke check and bench.py's CPU-baseline leg may load it;
 * the product path never does.  See ffs_oracle_impl.h for what it restates.
 *
 *   ffo32_*  reference-faithful FP32 build (R = float)
 *   ffo64_*  FP64 build of the same update (R = double)
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* LbmNodeFlag values, LbmDataTypes.cuh:17-56 */
enum {
    FL_INVALID = 0, FL_FLUID = 1, FL_FLUIDREST = 2, FL_SOLID = 3, FL_SOLIDDYN = 4, FL_WALL = 5,
    FL_WALL_L = 6, FL_WALL_R = 7, FL_WALL_F = 8, FL_WALL_B = 9, FL_WALL_D = 10, FL_WALL_U = 11,
    FL_WALL_C = 12, FL_IN_L = 13, FL_IN_R = 14, FL_IN_U = 15, FL_IN_D = 16, FL_IN_F = 17, FL_IN_B = 18,
    FL_OUT_L = 19, FL_OUT_R = 20, FL_OUT_U = 21, FL_OUT_D = 22, FL_OUT_F = 23, FL_OUT_B = 24
};

/* ---------------------------------------------------------------- geometry
 * FP32 restatement of the link geometry (SolidGeometryProxy_Device.cuh):
 * line_intersect :89-124, 2D intersectAtIndex :211-227, glm dot/cross/
 * normalize, barycentric_coordinates :291-304, line_triangle_intersect
 * :306-341 with the NumericUtils tolerance 1e-6 (NumericUtils.cuh:24).
 * Built with -ffp-contract=off: each operation rounds once, in order. */
typedef struct { int hit; float depth; float b[3]; } geo_hit;

static float geo_line(float x1, float y1, float x2, float y2, float x3, float y3, float x4, float y4, float *xo, float *yo)
{
    float a1 = (x1 - x2) * (y3 - y4) - (y1 - y2) * (x3 - x4);
    float b1 = (x4 - x2) * (y3 - y4) - (y4 - y2) * (x3 - x4);
    if (fabsf(a1) <= 0.0f) return -1.0f;
    float t1 = b1 / a1;
    if (t1 <= 0.0f || t1 >= 1.0f) return -1.0f;
    *xo = t1 * x1 + (1.0f - t1) * x2;
    if ((x3 - *xo) * (x4 - *xo) < 0.0f) {
        *yo = t1 * y1 + (1.0f - t1) * y2;
        return 1.0f - t1;
    }
    return -1.0f;
}

static geo_hit geo_isect2(const float *V, const uint32_t *E, int e, float p1x, float p1y, float p2x, float p2y)
{
    geo_hit r = {0, 0.0f, {0.0f, 0.0f, 0.0f}};
    uint32_t s = E[2 * e], t = E[2 * e + 1];
    float x3 = V[2 * s], y3 = V[2 * s + 1], x4 = V[2 * t], y4 = V[2 * t + 1];
    float xo = 0.0f, yo = 0.0f;
    float d = geo_line(p1x, p1y, p2x, p2y, x3, y3, x4, y4, &xo, &yo);
    if (d > 0.0f && d < 1.0f) {
        float dxh = x4 - xo, dyh = y4 - yo, dx34 = x4 - x3, dy34 = y4 - y3;
        float l1 = sqrtf(dxh * dxh + dyh * dyh);
        float l2 = sqrtf(dx34 * dx34 + dy34 * dy34);
        r.hit = 1; r.depth = d; r.b[0] = l1 / l2; r.b[1] = 1.0f - r.b[0];
    }
    return r;
}

static inline float geo_dot(const float *a, const float *b) { float x = a[0] * b[0], y = a[1] * b[1], z = a[2] * b[2]; return x + y + z; }
static inline void geo_cross(const float *a, const float *b, float *o)
{
    o[0] = a[1] * b[2] - b[1] * a[2];
    o[1] = a[2] * b[0] - b[2] * a[0];
    o[2] = a[0] * b[1] - b[0] * a[1];
}
static inline void geo_normalize(float *v)
{
    float inv = 1.0f / sqrtf(geo_dot(v, v));
    v[0] = v[0] * inv; v[1] = v[1] * inv; v[2] = v[2] * inv;
}

static geo_hit geo_isect3(const float *V, const uint32_t *E, int e, const float *p1, const float *p2)
{
    geo_hit r = {0, 0.0f, {0.0f, 0.0f, 0.0f}};
    float v[3][3];
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) v[j][k] = V[(size_t)E[3 * e + j] * 3 + k];
    float e1[3], e2[3], n[3], d[3], w0[3], pd[3];
    for (int k = 0; k < 3; ++k) { e1[k] = v[1][k] - v[0][k]; e2[k] = v[2][k] - v[0][k]; }
    geo_cross(e1, e2, n);
    geo_normalize(n);
    for (int k = 0; k < 3; ++k) d[k] = p2[k] - p1[k];
    geo_normalize(d);
    if (fabsf(geo_dot(n, d)) <= 1e-6f) return r;
    for (int k = 0; k < 3; ++k) { w0[k] = v[0][k] - p1[k]; pd[k] = p2[k] - p1[k]; }
    float t = geo_dot(n, w0) / geo_dot(n, pd);
    if (t < 0.0f || t > 1.0f) return r;
    float w[3];
    for (int k = 0; k < 3; ++k) w[k] = (p1[k] + t * pd[k]) - v[0][k];
    float d00 = geo_dot(e1, e1), d01 = geo_dot(e1, e2), d11 = geo_dot(e2, e2);
    float d20 = geo_dot(w, e1), d21 = geo_dot(w, e2);
    float den = d00 * d11 - d01 * d01;
    float u0 = (d11 * d20 - d01 * d21) / den;
    float v0 = (d00 * d21 - d01 * d20) / den;
    const float one_eps = 1.0f + 1e-6f;
    if (u0 >= -1e-6f && v0 >= -1e-6f && u0 + v0 <= one_eps) {
        r.hit = 1; r.depth = t; r.b[0] = (1.0f - u0) - v0; r.b[1] = u0; r.b[2] = v0;
    }
    return r;
}

/* ---------------------------------------------------------- 3D solid fill
 * The reference defines a 3D inside test, SolidGeometryProxy_Device<3>::
 * isInside (SolidGeometryProxy_Device.cuh:231-289: parity of the triangles
 * that the segment from the point to the origin crosses, with the
 * NumericUtils tolerances), but no 3D counterpart of fillSolidFlags2D.
 *
 * ffo_inside3_ref restates that test for one point.  ffo_fill_solid3 is the
 * product's 3D fill (ffs_lbm_fill_solid on a D3Q27 grid), restated with the
 * same float operations in the same order, so the two give the same flags:
 *   - rays run along +x through the (y, z) rows of cell centres;
 *   - a triangle is crossed by the row at (qy, qz) when the point lies in its
 *     (y, z) projection, by edge functions evaluated in vertex-index order
 *     (two triangles sharing an edge see exactly opposite values) with ties
 *     given to edges that point up in y (then z), so a row through a shared
 *     edge or vertex is counted once per sheet;
 *   - the crossing's x comes from the edge functions as barycentric weights,
 *     and it toggles the parity of every cell centre to its left;
 *   - Fluid and SolidDynamic cells become SolidDynamic where the parity is
 *     odd and Fluid elsewhere, like resetSolidFlagKernel +
 *     updateSolidFlagKernel (FsiCoupling2D.cu:318-354) in 2D. */
static float fs3_edge(const float *p, const float *s, float qy, float qz)
{
    return (s[1] - p[1]) * (qz - p[2]) - (s[2] - p[2]) * (qy - p[1]);
}

static float fs3_dir(const float *V, uint32_t iu, uint32_t iv, float qy, float qz, int *tie)
{
    const float *u = V + 3 * (size_t)iu, *v = V + 3 * (size_t)iv;
    *tie = (v[1] > u[1]) || (v[1] == u[1] && v[2] > u[2]);
    return iu < iv ? fs3_edge(u, v, qy, qz) : -fs3_edge(v, u, qy, qz);
}

static int fs3_incl(float e, int tie) { return e > 0.0f || (e == 0.0f && tie); }

static int fs3_cross(const float *V, uint32_t ia, uint32_t ib, uint32_t ic, float qy, float qz, float *xc)
{
    int t0, t1, t2;
    const float e0 = fs3_dir(V, ib, ic, qy, qz, &t0);
    const float e1 = fs3_dir(V, ic, ia, qy, qz, &t1);
    const float e2 = fs3_dir(V, ia, ib, qy, qz, &t2);
    if (e0 == 0.0f && e1 == 0.0f && e2 == 0.0f) return 0;
    const int pos = fs3_incl(e0, t0) && fs3_incl(e1, t1) && fs3_incl(e2, t2);
    const int neg = fs3_incl(-e0, !t0) && fs3_incl(-e1, !t1) && fs3_incl(-e2, !t2);
    if (!pos && !neg) return 0;
    const float ax = V[3 * (size_t)ia], bx = V[3 * (size_t)ib], cx = V[3 * (size_t)ic];
    *xc = ((e0 * ax + e1 * bx) + e2 * cx) / ((e0 + e1) + e2);
    return 1;
}

/* cells x in [0, nx) whose centre ((x + 0.5) cl) lies left of xc */
static int fs3_count_left(float xc, float cl, int nx)
{
    if (xc != xc) return 0;
    const float t = xc / cl - 0.5f;
    int k = !(t > 0.0f) ? 0 : (t >= (float)nx ? nx : (int)ceilf(t));
    while (k > 0 && ((float)(k - 1) + 0.5f) * cl >= xc) --k;
    while (k < nx && ((float)k + 0.5f) * cl < xc) ++k;
    return k;
}

/* first and last row index (clamped to [0, n)) whose centre can lie in
 * [lo, hi], padded by one row on each side */
static void fs3_rows(float lo, float hi, float cl, int n, int *r0, int *r1)
{
    float a = floorf(lo / cl - 0.5f) - 1.0f, b = ceilf(hi / cl - 0.5f) + 1.0f;
    a = fminf(fmaxf(a, 0.0f), (float)n);
    b = fminf(fmaxf(b, -1.0f), (float)(n - 1));
    *r0 = (int)a;
    *r1 = (int)b;
}

void ffo_fill_solid3(uint8_t *flags, int nx, int ny, int nz, float cl, const float *V, int nv, const uint32_t *E, int ne)
{
    const int words = (nx + 31) / 32;
    const size_t rows = (size_t)ny * nz;
    uint32_t *bits = (uint32_t *)calloc(rows * words, sizeof(uint32_t));
    if (!bits) return;
    for (int i = 0; i < ne; ++i) {
        const uint32_t ia = E[3 * (size_t)i], ib = E[3 * (size_t)i + 1], ic = E[3 * (size_t)i + 2];
        if (ia >= (uint32_t)nv || ib >= (uint32_t)nv || ic >= (uint32_t)nv) continue;
        int finite = 1;
        for (int k = 0; k < 3; ++k)
            finite &= isfinite(V[3 * (size_t)ia + k]) && isfinite(V[3 * (size_t)ib + k]) && isfinite(V[3 * (size_t)ic + k]);
        if (!finite) continue;
        const float *a = V + 3 * (size_t)ia, *b = V + 3 * (size_t)ib, *c = V + 3 * (size_t)ic;
        int y0, y1, z0, z1;
        fs3_rows(fminf(fminf(a[1], b[1]), c[1]), fmaxf(fmaxf(a[1], b[1]), c[1]), cl, ny, &y0, &y1);
        fs3_rows(fminf(fminf(a[2], b[2]), c[2]), fmaxf(fmaxf(a[2], b[2]), c[2]), cl, nz, &z0, &z1);
        for (int z = z0; z <= z1; ++z)
            for (int y = y0; y <= y1; ++y) {
                const float qy = ((float)y + 0.5f) * cl, qz = ((float)z + 0.5f) * cl;
                float xc;
                if (!fs3_cross(V, ia, ib, ic, qy, qz, &xc)) continue;
                const int k = fs3_count_left(xc, cl, nx);
                if (k < 1) continue;
                bits[((size_t)z * ny + y) * words + (size_t)((k - 1) >> 5)] ^= 1u << ((k - 1) & 31);
            }
    }
    for (size_t r = 0; r < rows; ++r) {
        uint32_t par = 0;
        for (int x = nx - 1; x >= 0; --x) {
            par ^= (bits[r * words + (size_t)(x >> 5)] >> (x & 31)) & 1u;
            uint8_t *f = flags + r * nx + x;
            if (*f == FL_FLUID || *f == FL_SOLIDDYN) *f = par ? FL_SOLIDDYN : FL_FLUID;
        }
    }
    free(bits);
}

/* SolidGeometryProxy_Device<3>::isInside (SolidGeometryProxy_Device.cuh:231-289) */
int ffo_inside3_ref(const float *V, const uint32_t *E, int ne, float px, float py, float pz)
{
    const float eps = 1e-6f;
    const float p[3] = {px, py, pz};
    int inside = 0;
    for (int i = 0; i < ne; ++i) {
        float v[3][3];
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) v[j][k] = V[(size_t)E[3 * (size_t)i + j] * 3 + k];
        float e1[3], e2[3], n[3], d[3];
        for (int k = 0; k < 3; ++k) { e1[k] = v[1][k] - v[0][k]; e2[k] = v[2][k] - v[0][k]; d[k] = p[k]; }
        geo_cross(e1, e2, n);
        geo_normalize(d);
        if (fabsf(geo_dot(n, d)) <= 0.0f + eps) continue;
        float w0[3], op[3];
        for (int k = 0; k < 3; ++k) { w0[k] = v[0][k] - p[k]; op[k] = -p[k]; }
        const float t = geo_dot(n, w0) / geo_dot(n, op);
        if (t <= 0.0f + eps || t > 1.0f + eps) continue;
        float hit[3];
        for (int k = 0; k < 3; ++k) hit[k] = p[k] + t * op[k];
        int same = 1;
        for (int j = 0; j < 3 && same; ++j) {
            const float *a = v[j], *b = v[(j + 1) % 3], *c = v[(j + 2) % 3];
            float ba[3], ca[3], ha[3], c1[3], c2[3];
            for (int k = 0; k < 3; ++k) { ba[k] = b[k] - a[k]; ca[k] = c[k] - a[k]; ha[k] = hit[k] - a[k]; }
            geo_cross(ba, ca, c1);
            const float vn = sqrtf(geo_dot(c1, c1));
            for (int k = 0; k < 3; ++k) c1[k] = c1[k] / vn;
            geo_cross(ba, ha, c2);
            for (int k = 0; k < 3; ++k) c2[k] = c2[k] / vn;
            if (geo_dot(c1, c2) <= 0.0f + eps) same = 0;
        }
        if (same) inside = !inside;
    }
    return inside;
}

#define R float
#define FN(x) ffo32_##x
#include "ffs_oracle_impl.h"
#undef R
#undef FN
#undef FN_THIRD
#undef FN_2THIRD
#undef FN_EPS

#define R double
#define FN(x) ffo64_##x
#include "ffs_oracle_impl.h"
#undef R
#undef FN

void ffo_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ffo_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* float -> binary16 -> float, round to nearest even (the rounding the
 * reference's __half shared-memory tile applies) */
float ffo_round_half(float v) { return (float)(_Float16)v; }
