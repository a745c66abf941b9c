/*
 * CPU oracle for the moment-encoded LBM fluid step -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is included twice by ffs_oracle.c: once with R = float (the
 * "ref32" build, which follows the reference's FP32 arithmetic, its op order,
 * its double-literal promotions and, for D2Q9, its binary16 shared-memory
 * population tile) and once with R = double (the "phys64" build: the same
 * update in FP64, used as the physics/precision yardstick).
 *
 * It restates these reference functions (paths relative to the FreeFlow repo):
 *   lattice tables        include/FSI_Simulator/lbm/LbmConstants.hpp:24-55
 *   Hermite reconstruction src/lbm/LbmUtilsFunc.cu:11-335 (D3Q27), :422-510 (D2Q9)
 *   collision             src/lbm/LbmUtilsFunc.cu:337-414 (D3Q27), :512-543 (D2Q9)
 *   fused step            src/core/FsiCoupling2D.cu:82-255, src/core/FsiCoupling3D.cu:83-334
 *   link detection        src/core/FsiCoupling2D.cu:31-80, src/core/FsiCoupling3D.cu:31-81
 *   outlets               src/core/FsiCoupling2D.cu:257-316, src/core/FsiCoupling3D.cu:336-420
 *   host step order       src/core/FsiCoupling2D.cu:358-432, src/core/FsiCoupling3D.cu:424-484
 *   geometry              include/FSI_Simulator/core/SolidGeometryProxy_Device.cuh:79-440
 *   initial state         src/lbm/LbmInitializer2D.cu:32-95, src/lbm/LbmInitializer3D.cu:33-113
 *   force scale Cf        include/FSI_Simulator/utils/Config.hpp:96-100,154-158
 *   fluid-solid fill      src/core/FsiCoupling2D.cu:318-354 (isInside, :126-144 of the proxy)
 *
 * Parity status: the reference ships no tests, golden vectors or fixtures for
 * this path, and its CUDA sources need glm/spdlog/nlohmann to compile, so the
 * reference itself cannot be run here.  Parity against the reference is
 * therefore UNPINNED; the oracle is pinned only by analytic known answers
 * (equilibrium fixed points, exact moment reproduction, conservation laws,
 * Taylor-Green decay) checked in the CPU test suite.
 *
 * Deliberate differences from the reference (documented, not bugs):
 *   - link keys are 64-bit (depth_q16 << 32 | element); ordering equals the
 *     reference's 32-bit (depth_q16 << 16 | element & 0xFFFF) key whenever the
 *     surface has at most 65536 elements;
 *   - surface forces are summed in double in a fixed (cell, direction) order
 *     instead of FP32 atomics;
 *   - the out-of-bounds shared-memory store of FsiCoupling2D.cu:129 is not
 *     reproduced (it has no defined result).
 */

#ifndef R
#error "include through ffs_oracle.c"
#endif

typedef struct {
    int dim, nx, ny, nz, Q, NM;
    long long ncell;
    int periodic;   /* bit0 x, bit1 y, bit2 z: halo wraps at both faces */
    int half_pops;  /* D2Q9: round the reconstructed tile to binary16 (reference smem) */
    int wall_stream;/* D2Q9: walls stream their moments (the reference's 2D kernel) */
    R vis, cl, ct, cf, omega;
    float clf;      /* lattice spacing as the reference's float (link geometry) */
    float bcvel[6];
    uint8_t *flags;
    R *mom[2];      /* AoS, NM values per cell, like the reference */
    int cur;
    R *rec;         /* 3 rolling z-planes x (nx*ny) x Q reconstructed populations */
    int rec_z[3];
    /* link state of the last step: sorted (cell*Q+dir, key) */
    long long nlinks, caplinks;
    uint64_t *link_cq, *link_key;
    uint8_t *linkcell; /* per-cell marker of the last step (1 bit used) */
} FN(grid);

/* ------------------------------------------------------------------ tables */

static R FN(w2)[9], FN(w3)[27];
static R FN(cs2);
static int FN(tables_ready) = 0;

static void FN(init_tables)(void)
{
    if (FN(tables_ready)) return;
    /* LbmConstants.hpp:51-54 and :28-35 (computed in R arithmetic) */
    FN(w2)[0] = (R)4 / (R)9;
    for (int i = 1; i <= 4; ++i) FN(w2)[i] = (R)1 / (R)9;
    for (int i = 5; i <= 8; ++i) FN(w2)[i] = (R)1 / (R)36;
    FN(w3)[0] = (R)8 / (R)27;
    for (int i = 1; i <= 6; ++i) FN(w3)[i] = (R)2 / (R)27;
    for (int i = 7; i <= 18; ++i) FN(w3)[i] = (R)1 / (R)54;
    for (int i = 19; i <= 26; ++i) FN(w3)[i] = (R)1 / (R)216;
    FN(cs2) = (R)1 / (R)3;
    FN(tables_ready) = 1;
}

/* --------------------------------------------------- Hermite reconstruction */

/* D2Q9 third-order coefficient; the 2D reference omits rho on the Pi terms
 * (LbmUtilsFunc.cu:439-441, :488-490). */
static inline R FN(q2)(R rho, R paa, R ub, R pab, R ua)
{
    return (R)9 * (paa * ub + (R)2 * pab * ua - (R)2 * rho * ua * ua * ub);
}

/* CalculateDistributionD2Q9ALL, LbmUtilsFunc.cu:476-510.  Arguments in the
 * reference's order (rho, ux, uy, pixx, pixy, piyy).  Populations 1..4 are
 * evaluated through double because the reference writes "0.5 * Q" with a
 * double literal. */
static void FN(rec2_all)(R rho, R ux, R uy, R pxx, R pxy, R pyy, R *f)
{
    const R *w = FN(w2);
    R m1x = (R)3 * rho * ux, m1y = (R)3 * rho * uy;
    R m2xx = (R)3 * rho * pxx, m2yy = (R)3 * rho * pyy, m2xy = (R)9 * rho * pxy;
    R qxxy = FN(q2)(rho, pxx, uy, pxy, ux);
    R qxyy = FN(q2)(rho, pyy, ux, pxy, uy);
    R bulk = rho - (R)0.5 * (m2xx + m2yy);
    f[0] = w[0] * bulk;
    f[1] = (R)((double)w[1] * ((double)(bulk + m1x + (R)1.5 * m2xx) - 0.5 * (double)qxyy));
    f[2] = (R)((double)w[2] * ((double)(bulk + m1y + (R)1.5 * m2yy) - 0.5 * (double)qxxy));
    f[3] = (R)((double)w[3] * ((double)(bulk - m1x + (R)1.5 * m2xx) + 0.5 * (double)qxyy));
    f[4] = (R)((double)w[4] * ((double)(bulk - m1y + (R)1.5 * m2yy) + 0.5 * (double)qxxy));
    R dbase = bulk + (R)1.5 * (m2xx + m2yy);
    f[5] = w[5] * (dbase + (m1x + m1y) + m2xy + (qxxy + qxyy));
    f[6] = w[6] * (dbase - m1x + m1y - m2xy + qxxy - qxyy);
    f[7] = w[7] * (dbase - m1x - m1y + m2xy - qxxy - qxyy);
    f[8] = w[8] * (dbase + m1x - m1y - m2xy - qxxy + qxyy);
}

/* CalculateDistributionD2Q9AtIndex, LbmUtilsFunc.cu:422-474 (all FP32). */
static R FN(rec2_at)(R rho, R ux, R uy, R pxx, R pxy, R pyy, int i)
{
    R m1x = (R)3 * rho * ux, m1y = (R)3 * rho * uy;
    R m2xx = (R)3 * rho * pxx, m2yy = (R)3 * rho * pyy, m2xy = (R)9 * rho * pxy;
    R qxxy = FN(q2)(rho, pxx, uy, pxy, ux);
    R qxyy = FN(q2)(rho, pyy, ux, pxy, uy);
    R bulk = rho - (R)0.5 * (m2xx + m2yy);
    R dbase = bulk + (R)1.5 * (m2xx + m2yy);
    R s = 0;
    switch (i) {
    case 0: s = bulk; break;
    case 1: s = bulk + m1x + (R)1.5 * m2xx - (R)0.5 * qxyy; break;
    case 2: s = bulk + m1y + (R)1.5 * m2yy - (R)0.5 * qxxy; break;
    case 3: s = bulk - m1x + (R)1.5 * m2xx + (R)0.5 * qxyy; break;
    case 4: s = bulk - m1y + (R)1.5 * m2yy + (R)0.5 * qxxy; break;
    case 5: s = dbase + (m1x + m1y) + m2xy + (qxxy + qxyy); break;
    case 6: s = dbase - m1x + m1y - m2xy + qxxy - qxyy; break;
    case 7: s = dbase - m1x - m1y + m2xy - qxxy - qxyy; break;
    case 8: s = dbase + m1x - m1y - m2xy - qxxy + qxyy; break;
    }
    return FN(w2)[i] * s;
}

/* D3Q27 coefficients shared by both reconstructions (LbmUtilsFunc.cu:27-68). */
typedef struct {
    R rho, m1x, m1y, m1z, m2xx, m2yy, m2zz, m2xy, m2yz, m2xz;
    R qxxy, qxyy, qxxz, qxzz, qyyz, qyzz, qxyz;
} FN(coef3);

static inline R FN(q3)(R rho, R paa, R ub, R pab, R ua)
{
    return (R)9 * (rho * paa * ub + (R)2 * rho * pab * ua - (R)2 * rho * ua * ua * ub);
}

static void FN(coef3_make)(R rho, R ux, R uy, R uz, R pxx, R pyy, R pzz,
                           R pxy, R pyz, R pxz, FN(coef3) *c)
{
    c->rho = rho;
    c->m1x = (R)3 * rho * ux; c->m1y = (R)3 * rho * uy; c->m1z = (R)3 * rho * uz;
    c->m2xx = (R)3 * rho * pxx; c->m2yy = (R)3 * rho * pyy; c->m2zz = (R)3 * rho * pzz;
    c->m2xy = (R)9 * rho * pxy; c->m2yz = (R)9 * rho * pyz; c->m2xz = (R)9 * rho * pxz;
    c->qxxy = FN(q3)(rho, pxx, uy, pxy, ux);
    c->qxyy = FN(q3)(rho, pyy, ux, pxy, uy);
    c->qxxz = FN(q3)(rho, pxx, uz, pxz, ux);
    c->qxzz = FN(q3)(rho, pzz, ux, pxz, uz);
    c->qyyz = FN(q3)(rho, pyy, uz, pyz, uy);
    c->qyzz = FN(q3)(rho, pzz, uy, pyz, uz);
    c->qxyz = (R)27 * (rho * (pxy * uz + pyz * ux + pxz * uy - (R)2 * ux * uy * uz));
}

/* CalculateDistributionD3Q27All, LbmUtilsFunc.cu:212-335. */
static void FN(rec3_all)(const FN(coef3) *c, R *f)
{
    const R *W = FN(w3);
    R w0 = W[0], w1 = W[1], w2 = W[7], w3 = W[19];
    R rho = c->rho, m1x = c->m1x, m1y = c->m1y, m1z = c->m1z;
    R m2xx = c->m2xx, m2yy = c->m2yy, m2zz = c->m2zz, m2xy = c->m2xy, m2yz = c->m2yz, m2xz = c->m2xz;
    R qxxy = c->qxxy, qxyy = c->qxyy, qxxz = c->qxxz, qxzz = c->qxzz, qyyz = c->qyyz, qyzz = c->qyzz, qxyz = c->qxyz;
    R bulk = rho - (R)0.5 * (m2xx + m2yy + m2zz);
    f[0] = w0 * bulk;
    R ax = bulk + (R)1.5 * m2xx;
    f[1] = w1 * (ax + m1x - (R)0.5 * (qxyy + qxzz));
    f[2] = w1 * (ax - m1x + (R)0.5 * (qxyy + qxzz));
    R ay = bulk + (R)1.5 * m2yy;
    f[3] = w1 * (ay + m1y - (R)0.5 * (qxxy + qyzz));
    f[4] = w1 * (ay - m1y + (R)0.5 * (qxxy + qyzz));
    R az = bulk + (R)1.5 * m2zz;
    f[5] = w1 * (az + m1z - (R)0.5 * (qxxz + qyyz));
    f[6] = w1 * (az - m1z + (R)0.5 * (qxxz + qyyz));
    R exy = rho + m2xx + m2yy - (R)0.5 * m2zz, qxy = qxxy + qxyy, oxy = (R)0.5 * (qxzz + qyzz);
    f[7] = w2 * (exy + (m1x + m1y) + m2xy + qxy - oxy);
    f[8] = w2 * (exy - (m1x + m1y) + m2xy - qxy + oxy);
    f[13] = w2 * (exy + (m1x - m1y) - m2xy - (qxxy - qxyy) - (R)0.5 * (qxzz - qyzz));
    f[14] = w2 * (exy - (m1x - m1y) - m2xy + (qxxy - qxyy) + (R)0.5 * (qxzz - qyzz));
    R exz = rho + m2xx + m2zz - (R)0.5 * m2yy, qxz = qxxz + qxzz, oxz = (R)0.5 * (qxyy + qyyz);
    f[9] = w2 * (exz + (m1x + m1z) + m2xz + qxz - oxz);
    f[10] = w2 * (exz - (m1x + m1z) + m2xz - qxz + oxz);
    f[15] = w2 * (exz + (m1x - m1z) - m2xz - (qxxz - qxzz) - (R)0.5 * (qxyy - qyyz));
    f[16] = w2 * (exz - (m1x - m1z) - m2xz + (qxxz - qxzz) + (R)0.5 * (qxyy - qyyz));
    R eyz = rho + m2yy + m2zz - (R)0.5 * m2xx, qyz = qyyz + qyzz, oyz = (R)0.5 * (qxxy + qxxz);
    f[11] = w2 * (eyz + (m1y + m1z) + m2yz + qyz - oyz);
    f[12] = w2 * (eyz - (m1y + m1z) + m2yz - qyz + oyz);
    f[17] = w2 * (eyz + (m1y - m1z) - m2yz - (qyyz - qyzz) - (R)0.5 * (qxxy - qxxz));
    f[18] = w2 * (eyz - (m1y - m1z) - m2yz + (qyyz - qyzz) + (R)0.5 * (qxxy - qxxz));
    R cM1 = m1x + m1y + m1z, cS = m2xx + m2yy + m2zz, cO = m2xy + m2yz + m2xz;
    R cQ = qxxy + qxxz + qxyy + qyyz + qxzz + qyzz;
    R cc = rho + cS;
    f[19] = w3 * (cc + cM1 + cO + cQ + qxyz);
    f[20] = w3 * (cc - cM1 + cO - cQ - qxyz);
    f[21] = w3 * (cc + (m1x + m1y - m1z) + (m2xy - m2yz - m2xz) + (qxxy - qxxz + qxyy - qyyz + qxzz + qyzz) - qxyz);
    f[22] = w3 * (cc - (m1x + m1y - m1z) + (m2xy - m2yz - m2xz) - (qxxy - qxxz + qxyy - qyyz + qxzz + qyzz) + qxyz);
    f[23] = w3 * (cc + (m1x - m1y + m1z) + (-m2xy - m2yz + m2xz) + (-qxxy + qxxz + qxyy + qyyz + qxzz - qyzz) - qxyz);
    f[24] = w3 * (cc - (m1x - m1y + m1z) + (-m2xy - m2yz + m2xz) - (-qxxy + qxxz + qxyy + qyyz + qxzz - qyzz) + qxyz);
    f[25] = w3 * (cc + (-m1x + m1y + m1z) + (-m2xy + m2yz - m2xz) + (qxxy + qxxz - qxyy + qyyz - qxzz + qyzz) - qxyz);
    f[26] = w3 * (cc - (-m1x + m1y + m1z) + (-m2xy + m2yz - m2xz) - (qxxy + qxxz - qxyy + qyyz - qxzz + qyzz) + qxyz);
}

/* CalculateDistributionD3Q27AtIndex, LbmUtilsFunc.cu:11-210. */
static R FN(rec3_at)(const FN(coef3) *c, int i)
{
    R rho = c->rho, m1x = c->m1x, m1y = c->m1y, m1z = c->m1z;
    R m2xx = c->m2xx, m2yy = c->m2yy, m2zz = c->m2zz, m2xy = c->m2xy, m2yz = c->m2yz, m2xz = c->m2xz;
    R qxxy = c->qxxy, qxyy = c->qxyy, qxxz = c->qxxz, qxzz = c->qxzz, qyyz = c->qyyz, qyzz = c->qyzz, qxyz = c->qxyz;
    R bulk = rho - (R)0.5 * (m2xx + m2yy + m2zz);
    R bulk2 = rho + (m2xx + m2yy + m2zz);
    R h = (R)0.5, t = (R)1.5, s = 0;
    switch (i) {
    case 0: s = bulk; break;
    case 1: s = bulk + m1x + t * m2xx - h * (qxyy + qxzz); break;
    case 2: s = bulk - m1x + t * m2xx + h * (qxyy + qxzz); break;
    case 3: s = bulk + m1y + t * m2yy - h * (qxxy + qyzz); break;
    case 4: s = bulk - m1y + t * m2yy + h * (qxxy + qyzz); break;
    case 5: s = bulk + m1z + t * m2zz - h * (qxxz + qyyz); break;
    case 6: s = bulk - m1z + t * m2zz + h * (qxxz + qyyz); break;
    case 7: s = rho + (m1x + m1y) + (m2xx + m2yy - h * m2zz) + m2xy + (qxxy + qxyy) - h * (qxzz + qyzz); break;
    case 8: s = rho - (m1x + m1y) + (m2xx + m2yy - h * m2zz) + m2xy - (qxxy + qxyy) + h * (qxzz + qyzz); break;
    case 9: s = rho + (m1x + m1z) + (m2xx + m2zz - h * m2yy) + m2xz + (qxxz + qxzz) - h * (qxyy + qyyz); break;
    case 10: s = rho - (m1x + m1z) + (m2xx + m2zz - h * m2yy) + m2xz - (qxxz + qxzz) + h * (qxyy + qyyz); break;
    case 11: s = rho + (m1y + m1z) + (m2yy + m2zz - h * m2xx) + m2yz + (qyyz + qyzz) - h * (qxxy + qxxz); break;
    case 12: s = rho - (m1y + m1z) + (m2yy + m2zz - h * m2xx) + m2yz - (qyyz + qyzz) + h * (qxxy + qxxz); break;
    case 13: s = rho + (m1x - m1y) + (m2xx + m2yy - h * m2zz) - m2xy - (qxxy - qxyy) - h * (qxzz - qyzz); break;
    case 14: s = rho - (m1x - m1y) + (m2xx + m2yy - h * m2zz) - m2xy + (qxxy - qxyy) + h * (qxzz - qyzz); break;
    case 15: s = rho + (m1x - m1z) + (m2xx + m2zz - h * m2yy) - m2xz - (qxxz - qxzz) - h * (qxyy - qyyz); break;
    case 16: s = rho - (m1x - m1z) + (m2xx + m2zz - h * m2yy) - m2xz + (qxxz - qxzz) + h * (qxyy - qyyz); break;
    case 17: s = rho + (m1y - m1z) + (m2yy + m2zz - h * m2xx) - m2yz - (qyyz - qyzz) - h * (qxxy - qxxz); break;
    case 18: s = rho - (m1y - m1z) + (m2yy + m2zz - h * m2xx) - m2yz + (qyyz - qyzz) + h * (qxxy - qxxz); break;
    case 19: s = bulk2 + (m1x + m1y + m1z) + (m2xy + m2yz + m2xz) + (qxxy + qxxz + qxyy + qyyz + qxzz + qyzz) + qxyz; break;
    case 20: s = bulk2 - (m1x + m1y + m1z) + (m2xy + m2yz + m2xz) - (qxxy + qxxz + qxyy + qyyz + qxzz + qyzz) - qxyz; break;
    case 21: s = bulk2 + (m1x + m1y - m1z) + (m2xy - m2yz - m2xz) + (qxxy - qxxz + qxyy - qyyz + qxzz + qyzz) - qxyz; break;
    case 22: s = bulk2 - (m1x + m1y - m1z) + (m2xy - m2yz - m2xz) - (qxxy - qxxz + qxyy - qyyz + qxzz + qyzz) + qxyz; break;
    case 23: s = bulk2 + (m1x - m1y + m1z) + (-m2xy - m2yz + m2xz) + (-qxxy + qxxz + qxyy + qyyz + qxzz - qyzz) - qxyz; break;
    case 24: s = bulk2 - (m1x - m1y + m1z) + (-m2xy - m2yz + m2xz) - (-qxxy + qxxz + qxyy + qyyz + qxzz - qyzz) + qxyz; break;
    case 25: s = bulk2 + (-m1x + m1y + m1z) + (-m2xy + m2yz - m2xz) + (qxxy + qxxz - qxyy + qyyz - qxzz + qyzz) - qxyz; break;
    case 26: s = bulk2 - (-m1x + m1y + m1z) + (-m2xy + m2yz - m2xz) - (qxxy + qxxz - qxyy + qyyz - qxzz + qyzz) + qxyz; break;
    }
    return FN(w3)[i] * s;
}

/* ---------------------------------------------------------------- collision */

/* LbmUtilsFuncGpu2D::Collision, LbmUtilsFunc.cu:512-543 (F = 0 on this path). */
static void FN(collide2)(R rho, R ux, R uy, R fx, R fy, R om, R *pxx, R *pyy, R *pxy)
{
    R omw = (R)1 - om;
    R p = rho / (R)3;
    R ru2 = rho * ux * ux, rv2 = rho * uy * uy;
    R dev = (*pxx - *pyy) * (R)0.5;
    R be = p + (R)0.5 * (ru2 + rv2);
    R an = (R)0.5 * om * (ru2 - rv2);
    R ff = (R)0.5 * omw;
    R ftx = fx * ux + ff * (fx * ux - fy * uy);
    R fty = fy * uy + ff * (fy * uy - fx * ux);
    R nxx = be + dev * omw + an + ftx;
    R nyy = be - dev * omw - an + fty;
    R nxy = *pxy * omw + (om * rho * ux * uy) + ((R)1 - (R)0.5 * om) * (fy * ux + fx * uy);
    *pxx = nxx; *pyy = nyy; *pxy = nxy;
}

#define FN_THIRD ((sizeof(R) == 4) ? (R)0.33333333f : (R)1 / (R)3)
#define FN_2THIRD ((sizeof(R) == 4) ? (R)0.6666667f : (R)2 / (R)3)

/* LbmUtilsFuncGpu3D::Collision, LbmUtilsFunc.cu:337-414.  The FP32 build keeps
 * the reference's rounded 0.33333333f / 0.6666667f literals; the FP64 build
 * uses exact thirds. */
static void FN(collide3)(R rho, R ux, R uy, R uz, R Fx, R Fy, R Fz, R om, R *m)
{
    /* m = {pxx, pyy, pzz, pxy, pyz, pxz} raw second moments in, relaxed out */
    const R third = FN_THIRD, two3 = FN_2THIRD;
    R omw = (R)1 - om;
    R dfc = omw * (R)0.5;
    R odc = (R)1 - (R)0.5 * om;
    R r3 = rho * third;
    R rux = rho * ux * ux, ruy = rho * uy * uy, ruz = rho * uz * uz;
    R wr = om * rho;
    m[3] = omw * m[3] + wr * (ux * uy) + odc * (Fx * uy + Fy * ux);
    m[5] = omw * m[5] + wr * (ux * uz) + odc * (Fx * uz + Fz * ux);
    m[4] = omw * m[4] + wr * (uy * uz) + odc * (Fy * uz + Fz * uy);
    R sxx = m[0], syy = m[1], szz = m[2];
    R dxx = ((R)2 * sxx - syy - szz) * third;
    R dyy = ((R)2 * syy - sxx - szz) * third;
    R dzz = ((R)2 * szz - sxx - syy) * third;
    R fux = Fx * ux, fuy = Fy * uy, fuz = Fz * uz;
    R fdc = dfc * two3;
    R en = (rux + ruy + ruz) * third;
    R rx = (om * third) * ((R)2 * rux - ruy - ruz);
    R fxx = fux + fdc * ((R)2 * fux - fuy - fuz);
    m[0] = r3 + en + omw * dxx + rx + fxx;
    R ry = (om * third) * ((R)2 * ruy - rux - ruz);
    R fyy = fuy + fdc * ((R)2 * fuy - fux - fuz);
    m[1] = r3 + en + omw * dyy + ry + fyy;
    R rz = (om * third) * ((R)2 * ruz - rux - ruy);
    R fzz = fuz + fdc * ((R)2 * fuz - fux - fuy);
    m[2] = r3 + en + omw * dzz + rz + fzz;
}

/* -------------------------------------------------------------- binary16 */

static inline R FN(round_pop)(const FN(grid) *g, R v)
{
    if (!g->half_pops) return v;
    return (R)(float)(_Float16)(float)v; /* round-to-nearest-even, as __float2half */
}

/* ----------------------------------------------------------------- geometry
 * Restated from SolidGeometryProxy_Device.cuh in ffs_oracle.c (geo_* below),
 * in FP32 for BOTH builds: the surface arrays are FP32 in the reference and
 * the link set is a discrete function of them, so the FP64 build uses the very
 * same links and differs from the FP32 build only in the fluid arithmetic. */

typedef struct { int hit; R depth; R b[3]; } FN(isect);

static FN(isect) FN(isect2)(const float *V, const uint32_t *E, int e, R p1x, R p1y, R p2x, R p2y)
{
    geo_hit h = geo_isect2(V, E, e, (float)p1x, (float)p1y, (float)p2x, (float)p2y);
    FN(isect) r; r.hit = h.hit; r.depth = (R)h.depth; r.b[0] = (R)h.b[0]; r.b[1] = (R)h.b[1]; r.b[2] = (R)h.b[2];
    return r;
}

static FN(isect) FN(isect3)(const float *V, const uint32_t *E, int e, const R *p1, const R *p2)
{
    float a[3] = {(float)p1[0], (float)p1[1], (float)p1[2]}, b[3] = {(float)p2[0], (float)p2[1], (float)p2[2]};
    geo_hit h = geo_isect3(V, E, e, a, b);
    FN(isect) r; r.hit = h.hit; r.depth = (R)h.depth; r.b[0] = (R)h.b[0]; r.b[1] = (R)h.b[1]; r.b[2] = (R)h.b[2];
    return r;
}

/* depthIndexCompact, :79-85, widened to 64 bits (see file header). */
static inline uint64_t FN(link_key)(R depth, int e)
{
    uint32_t dq = (uint32_t)((float)depth * 32768.0f);
    return ((uint64_t)dq << 32) | (uint32_t)e;
}

/* ------------------------------------------------------------ grid helpers */

/* node flags (LbmDataTypes.cuh:17-56) are defined once in ffs_oracle.c */

/* bounce-back flag sets: FsiCoupling2D.cu:171-176 and FsiCoupling3D.cu:209-216 */
static inline int FN(is_bb)(int dim, uint8_t f)
{
    if (f == FL_SOLID || f == FL_WALL || f == FL_WALL_L || f == FL_WALL_R || f == FL_WALL_U || f == FL_WALL_D)
        return 1;
    if (dim == 3 && (f == FL_WALL_F || f == FL_WALL_B)) return 1;
    return 0;
}

static const int FN(ex2)[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int FN(ey2)[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int FN(inv2)[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const int FN(ex3)[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
static const int FN(ey3)[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
static const int FN(ez3)[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
static const int FN(inv3)[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};

static inline void FN(dirs)(const FN(grid) *g, const int **ex, const int **ey, const int **ez, const int **inv)
{
    static const int zero9[9] = {0};
    if (g->dim == 2) { *ex = FN(ex2); *ey = FN(ey2); *ez = zero9; *inv = FN(inv2); }
    else { *ex = FN(ex3); *ey = FN(ey3); *ez = FN(ez3); *inv = FN(inv3); }
}

/* Halo index of a non-periodic axis as the reference's shared-memory fill
 * forms it (FsiCoupling2D.cu:104-105, FsiCoupling3D.cu:106-108):
 * min(n - 1, max(0, (s - 1) + blockDim * blockIdx)) with an unsigned
 * blockDim * blockIdx, so -1 becomes a huge unsigned value and then n - 1
 * (the low face wraps) while n is clamped to n - 1 (the high face clamps). */
static inline int FN(haloi)(int v, int n) { return (v < 0 || v >= n) ? n - 1 : v; }
static inline int FN(wrapi)(int v, int n) { return ((v % n) + n) % n; }

/* ------------------------------------------------------------- life cycle */

FN(grid) *FN(create)(int dim, int nx, int ny, int nz, double viscosity, double density,
                     double dx, double dt, const float *bcvel, int periodic, int half_pops)
{
    FN(init_tables)();
    if ((dim != 2 && dim != 3) || nx <= 0 || ny <= 0) return NULL;
    if (dim == 2) nz = 1;
    if (nz <= 0) return NULL;
    FN(grid) *g = (FN(grid) *)calloc(1, sizeof(FN(grid)));
    g->dim = dim; g->nx = nx; g->ny = ny; g->nz = nz;
    g->Q = dim == 2 ? 9 : 27; g->NM = dim == 2 ? 6 : 10;
    g->ncell = (long long)nx * ny * nz;
    /* half_pops bit 0: binary16 tile; bit 1: 2D walls stream (both 2D only) */
    g->periodic = periodic;
    g->half_pops = (dim == 2) ? (half_pops & 1) : 0;
    g->wall_stream = (dim == 2) ? ((half_pops >> 1) & 1) : 0;
    /* m_viscosity is a float (LbmFlowField2D.hpp:177); omega is formed in double
     * (FsiCoupling2D.cu:236, FsiCoupling3D.cu:303) and rounded to R. */
    float visf = (float)viscosity;
    g->vis = (R)visf;
    g->omega = (sizeof(R) == 4) ? (R)(1.0 / ((double)visf * 3.0 + 0.5)) : (R)(1.0 / (viscosity * 3.0 + 0.5));
    g->cl = (sizeof(R) == 4) ? (R)(float)dx : (R)dx;
    g->clf = (float)dx;
    g->ct = (sizeof(R) == 4) ? (R)(float)dt : (R)dt;
    /* getCf, Config.hpp:96-100 (2D) and :154-158 (3D) */
    if (sizeof(R) == 4) {
        float cm = (float)(dim == 2 ? density * dx * dx : density * dx * dx * dx);
        g->cf = (R)(float)((double)cm * dx / (dt * dt));
    } else {
        double cm = dim == 2 ? density * dx * dx : density * dx * dx * dx;
        g->cf = (R)(cm * dx / (dt * dt));
    }
    for (int i = 0; i < 6; ++i) g->bcvel[i] = bcvel ? bcvel[i] : 0.0f;
    g->flags = (uint8_t *)calloc((size_t)g->ncell, 1);
    for (long long c = 0; c < g->ncell; ++c) g->flags[c] = FL_FLUID;
    g->mom[0] = (R *)calloc((size_t)g->ncell * g->NM, sizeof(R));
    g->mom[1] = (R *)calloc((size_t)g->ncell * g->NM, sizeof(R));
    g->rec = (R *)malloc(sizeof(R) * (size_t)4 * nx * ny * g->Q);
    g->linkcell = (uint8_t *)calloc((size_t)g->ncell, 1);
    g->cur = 0;
    return g;
}

void FN(destroy)(FN(grid) *g)
{
    if (!g) return;
    free(g->flags); free(g->mom[0]); free(g->mom[1]); free(g->rec);
    free(g->link_cq); free(g->link_key); free(g->linkcell);
    free(g);
}

void FN(set_flags)(FN(grid) *g, const uint8_t *f) { memcpy(g->flags, f, (size_t)g->ncell); }
void FN(get_flags)(const FN(grid) *g, uint8_t *f) { memcpy(f, g->flags, (size_t)g->ncell); }
double FN(get_cf)(const FN(grid) *g) { return (double)g->cf; }
double FN(get_omega)(const FN(grid) *g) { return (double)g->omega; }

/* which: 0 = current, 1 = next, 2 = buffer A (reference m_fMom / m_moments_pre),
 * 3 = buffer B, 4 = both (set only) */
static R *FN(buf)(FN(grid) *g, int which)
{
    switch (which) {
    case 0: return g->mom[g->cur];
    case 1: return g->mom[1 - g->cur];
    case 2: return g->mom[0];
    default: return g->mom[1];
    }
}

void FN(set_moments)(FN(grid) *g, const double *aos, int which)
{
    size_t n = (size_t)g->ncell * g->NM;
    if (which == 4) {
        for (size_t i = 0; i < n; ++i) g->mom[0][i] = g->mom[1][i] = (R)aos[i];
        return;
    }
    R *b = FN(buf)(g, which);
    for (size_t i = 0; i < n; ++i) b[i] = (R)aos[i];
}

void FN(get_moments)(FN(grid) *g, double *aos, int which)
{
    size_t n = (size_t)g->ncell * g->NM;
    R *b = FN(buf)(g, which);
    for (size_t i = 0; i < n; ++i) aos[i] = (double)b[i];
}

/* initialize_state_kernel_2d/3d (LbmInitializer2D.cu:32-95, LbmInitializer3D.cu:33-113):
 * rho = 1, u from the inlet flag, moments of the 2nd-order equilibrium, written
 * to both buffers; the current buffer becomes buffer A (LbmFlowField*::reset). */
void FN(initialize)(FN(grid) *g)
{
    const int *ex, *ey, *ez, *inv;
    FN(dirs)(g, &ex, &ey, &ez, &inv);
    const R *W = g->dim == 2 ? FN(w2) : FN(w3);
    const float *bc = g->bcvel;
    g->cur = 0;
    for (long long c = 0; c < g->ncell; ++c) {
        uint8_t f = g->flags[c];
        R ux = 0, uy = 0, uz = 0, rho = 1;
        if (g->dim == 2) {
            if (f == FL_IN_L) ux = bc[0];
            else if (f == FL_IN_D) uy = bc[1];
            else if (f == FL_IN_R) ux = -bc[2];
            else if (f == FL_IN_U) uy = -bc[3];
        } else {
            if (f == FL_IN_L) ux = bc[0];
            else if (f == FL_IN_D) uz = bc[1];
            else if (f == FL_IN_R) ux = -bc[2];
            else if (f == FL_IN_U) uz = -bc[3];
            else if (f == FL_IN_F) uy = bc[4];
            else if (f == FL_IN_B) uy = -bc[5];
        }
        R usq = ux * ux + uy * uy + (g->dim == 3 ? uz * uz : 0);
        if (g->dim == 2) usq = ux * ux + uy * uy;
        R feq[27];
        for (int k = 0; k < g->Q; ++k) {
            R cu = (R)ex[k] * ux + (R)ey[k] * uy;
            if (g->dim == 3) cu = cu + (R)ez[k] * uz;
            feq[k] = W[k] * rho * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
        }
        R invr = (R)1 / rho;
        R *m0 = g->mom[0] + (size_t)c * g->NM, *m1 = g->mom[1] + (size_t)c * g->NM;
        R v[10];
        if (g->dim == 2) {
            R pxx = feq[1] + feq[3] + feq[5] + feq[6] + feq[7] + feq[8];
            R pyy = feq[2] + feq[4] + feq[5] + feq[6] + feq[7] + feq[8];
            R pxy = feq[5] - feq[6] + feq[7] - feq[8];
            v[0] = rho; v[1] = ux; v[2] = uy;
            v[3] = pxx * invr - FN(cs2); v[4] = pyy * invr - FN(cs2); v[5] = pxy * invr;
        } else {
            const R *q = feq;
            R pxx = (q[1] + q[2] + q[7] + q[8] + q[9] + q[10] + q[13] + q[14] + q[15] + q[16] + q[19] + q[20] + q[21] + q[22] + q[23] + q[24] + q[25] + q[26]);
            R pyy = (q[3] + q[4] + q[7] + q[8] + q[11] + q[12] + q[13] + q[14] + q[17] + q[18] + q[19] + q[20] + q[21] + q[22] + q[23] + q[24] + q[25] + q[26]);
            R pzz = (q[5] + q[6] + q[9] + q[10] + q[11] + q[12] + q[15] + q[16] + q[17] + q[18] + q[19] + q[20] + q[21] + q[22] + q[23] + q[24] + q[25] + q[26]);
            R pxy = ((q[7] + q[8] + q[19] + q[20] + q[21] + q[22]) - (q[13] + q[14] + q[23] + q[24] + q[25] + q[26]));
            R pyz = ((q[11] + q[12] + q[19] + q[20] + q[25] + q[26]) - (q[17] + q[18] + q[21] + q[22] + q[23] + q[24]));
            R pxz = ((q[9] + q[10] + q[19] + q[20] + q[23] + q[24]) - (q[15] + q[16] + q[21] + q[22] + q[25] + q[26]));
            v[0] = rho; v[1] = ux; v[2] = uy; v[3] = uz;
            v[4] = (R)((double)(pxx * invr) - (double)FN(cs2));
            v[5] = (R)((double)(pyy * invr) - (double)FN(cs2));
            v[6] = (R)((double)(pzz * invr) - (double)FN(cs2));
            v[7] = pxy * invr; v[8] = pyz * invr; v[9] = pxz * invr;
        }
        for (int k = 0; k < g->NM; ++k) m0[k] = m1[k] = v[k];
    }
}

/* --------------------------------------------------- reconstructed z-planes */

static void FN(rec_cell)(const FN(grid) *g, const R *m, R *f)
{
    if (g->dim == 2) {
        /* FsiCoupling2D.cu:110-117 passes (rho, ux, uy, pixx, pixy, piyy) */
        FN(rec2_all)(m[0], m[1], m[2], m[3], m[5], m[4], f);
        for (int i = 0; i < 9; ++i) f[i] = FN(round_pop)(g, f[i]);
    } else {
        FN(coef3) c;
        FN(coef3_make)(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8], m[9], &c);
        FN(rec3_all)(&c, f);
    }
}

/* slot cache of 4 planes (3 are needed at a time, clamped or wrapped in z) */
typedef struct { int z[4]; R *p[4]; } FN(planes);

static R *FN(plane_get)(FN(grid) *g, FN(planes) *pl, const R *src, int z, const int *keep)
{
    for (int s = 0; s < 4; ++s)
        if (pl->z[s] == z) return pl->p[s];
    int s = 0;
    for (; s < 4; ++s) {
        int used = 0;
        for (int k = 0; k < 3; ++k) if (pl->z[s] == keep[k]) used = 1;
        if (!used) break;
    }
    pl->z[s] = z;
    R *dst = pl->p[s];
    long long nxy = (long long)g->nx * g->ny;
    const R *m = src + (size_t)z * nxy * g->NM;
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < nxy; ++c) FN(rec_cell)(g, m + (size_t)c * g->NM, dst + (size_t)c * g->Q);
    return dst;
}

/* ---------------------------------------------------------------- one cell */

static long long FN(find_link)(const FN(grid) *g, uint64_t cq)
{
    long long lo = 0, hi = g->nlinks - 1;
    while (lo <= hi) {
        long long mid = (lo + hi) / 2;
        if (g->link_cq[mid] == cq) return mid;
        if (g->link_cq[mid] < cq) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

typedef struct {
    const float *V, *U;
    const uint32_t *E;
    int nv, ne;
    double *forces;
} FN(surface);

/* The per-cell body of mrDeformableSolver2DKernel_Shrd (FsiCoupling2D.cu:139-253)
 * and mrDeformableSolver3DKernel_ShrdM (FsiCoupling3D.cu:174-333).
 * P[3] = reconstructed planes for z-1, z, z+1 (after clamping / wrapping). */
static void FN(update_cell)(FN(grid) *g, const R *src, R *dst, int x, int y, int z,
                            R *const *P, const FN(surface) *S, int with_links)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz, Q = g->Q, NM = g->NM, dim = g->dim;
    const int *ex, *ey, *ez, *inv;
    FN(dirs)(g, &ex, &ey, &ez, &inv);
    long long cid = ((long long)z * ny + y) * nx + x;
    const R *mc = src + (size_t)cid * NM;
    const R *own = P[1] + ((size_t)y * nx + x) * Q;
    R pop[27];
    for (int i = 0; i < Q; ++i) {
        int cx = ex[i], cy = ey[i], cz = ez[i];
        int x1 = x - cx, y1 = y - cy, z1 = z - cz;
        int notCross = x1 >= 0 && x1 < nx && y1 >= 0 && y1 < ny && z1 >= 0 && z1 < nz;
        int wx = FN(wrapi)(x1, nx), wy = FN(wrapi)(y1, ny), wz = FN(wrapi)(z1, nz);
        long long ib = ((long long)wz * ny + wy) * nx + wx;
        const int bb = FN(is_bb)(dim, g->flags[ib]);
        if (bb && !(dim == 2 && g->wall_stream)) {
            R v = own[inv[i]];
            pop[i] = v > 0 ? v : (R)0;
            continue;
        }
        /* wall_stream, 2D: the reference's kernel computes the bounce-back value
         * but, is_blocked being set only on the moving-wall path, overwrites it
         * with the ordinary pull and skips the link (FsiCoupling2D.cu:171-224) */
        int blocked = 0;
        if (with_links && notCross && !bb) {
            long long li = FN(find_link)(g, (uint64_t)cid * Q + i);
            if (li >= 0) {
                int e = (int)(g->link_key[li] & 0xFFFFFFFFu);
                FN(isect) in;
                const float cl = g->clf;
                if (dim == 2) {
                    in = FN(isect2)(S->V, S->E, e, (float)x * cl, (float)y * cl, (float)x1 * cl, (float)y1 * cl);
                } else {
                    R p1[3] = {(float)x * cl, (float)y * cl, (float)z * cl};
                    R p2[3] = {(float)x1 * cl, (float)y1 * cl, (float)z1 * cl};
                    in = FN(isect3)(S->V, S->E, e, p1, p2);
                }
                if (in.hit) {
                    blocked = 1;
                    R vfin = own[inv[i]];
                    R fin = vfin > 0 ? vfin : (R)0;
                    R fout, F[3];
                    if (dim == 2) {
                        /* FsiCoupling2D.cu:193-214 */
                        uint32_t a = S->E[2 * e], b = S->E[2 * e + 1];
                        R ux = (R)S->U[2 * a] * in.b[0] + (R)S->U[2 * b] * in.b[1];
                        R uy = (R)S->U[2 * a + 1] * in.b[0] + (R)S->U[2 * b + 1] * in.b[1];
                        R sc = g->ct / g->cl;
                        ux = ux * sc; uy = uy * sc;
                        R pxx = mc[3] + ux * ux - mc[1] * mc[1];
                        R pyy = mc[4] + uy * uy - mc[2] * mc[2];
                        R pxy = mc[5] + uy * ux - mc[1] * mc[2];
                        fout = FN(rec2_at)(mc[0], ux, uy, pxx, pxy, pyy, i);
                        F[0] = (fin * ((R)(-cx) - ux) - fout * ((R)cx - ux)) * g->cf;
                        F[1] = (fin * ((R)(-cy) - uy) - fout * ((R)cy - uy)) * g->cf;
                        if (S->forces) {
                            S->forces[2 * a] += (double)(F[0] * in.b[0]);
                            S->forces[2 * a + 1] += (double)(F[1] * in.b[0]);
                            S->forces[2 * b] += (double)(F[0] * in.b[1]);
                            S->forces[2 * b + 1] += (double)(F[1] * in.b[1]);
                        }
                    } else {
                        /* FsiCoupling3D.cu:229-269 */
                        uint32_t vv[3] = {S->E[3 * e], S->E[3 * e + 1], S->E[3 * e + 2]};
                        R u[3];
                        for (int k = 0; k < 3; ++k) {
                            R s = (R)S->U[3 * vv[0] + k] * in.b[0] + (R)S->U[3 * vv[1] + k] * in.b[1];
                            u[k] = s + (R)S->U[3 * vv[2] + k] * in.b[2];
                        }
                        for (int k = 0; k < 3; ++k) u[k] = u[k] * g->ct / g->cl;
                        R pxx = mc[4] + u[0] * u[0] - mc[1] * mc[1];
                        R pyy = mc[5] + u[1] * u[1] - mc[2] * mc[2];
                        R pzz = mc[6] + u[2] * u[2] - mc[3] * mc[3];
                        R pxy = mc[7] + u[0] * u[1] - mc[1] * mc[2];
                        R pyz = mc[8] + u[1] * u[2] - mc[2] * mc[3];
                        R pxz = mc[9] + u[0] * u[2] - mc[1] * mc[3];
                        FN(coef3) cc;
                        FN(coef3_make)(mc[0], u[0], u[1], u[2], pxx, pyy, pzz, pxy, pyz, pxz, &cc);
                        fout = FN(rec3_at)(&cc, i);
                        int cv[3] = {cx, cy, cz};
                        for (int k = 0; k < 3; ++k)
                            F[k] = (fin * ((R)(-cv[k]) - u[k]) - fout * ((R)cv[k] - u[k])) * g->cf;
                        if (S->forces)
                            for (int k = 0; k < 3; ++k) {
                                S->forces[3 * vv[0] + k] += (double)(F[k] * in.b[0]);
                                S->forces[3 * vv[1] + k] += (double)(F[k] * in.b[1]);
                                S->forces[3 * vv[2] + k] += (double)(F[k] * in.b[2]);
                            }
                    }
                    pop[i] = fout;
                }
            }
        }
        if (!blocked) {
            int sx, sy, sz;
            if (g->periodic & 1) sx = wx; else sx = FN(haloi)(x1, nx);
            if (g->periodic & 2) sy = wy; else sy = FN(haloi)(y1, ny);
            (void)sz;
            const R *pl = P[1 - cz]; /* plane z - cz */
            R v = pl[((size_t)sy * nx + sx) * Q + i];
            pop[i] = v > 0 ? v : (R)0;
        }
    }
    R *o = dst + (size_t)cid * NM;
    if (dim == 2) {
        /* FsiCoupling2D.cu:226-252 */
        const R *p = pop;
        R rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
        R ir = (R)1 / rho;
        R ux = (p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) * ir;
        R uy = (p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) * ir;
        R pxx = p[1] + p[3] + p[5] + p[6] + p[7] + p[8];
        R pyy = p[2] + p[4] + p[5] + p[6] + p[7] + p[8];
        R pxy = p[5] - p[6] + p[7] - p[8];
        FN(collide2)(rho, ux, uy, 0, 0, g->omega, &pxx, &pyy, &pxy);
        o[0] = rho; o[1] = ux; o[2] = uy;
        o[3] = pxx * ir - FN(cs2); o[4] = pyy * ir - FN(cs2); o[5] = pxy * ir;
    } else {
        /* FsiCoupling3D.cu:287-320 (the body-force field is identically zero) */
        const R *p = pop;
        R rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] + p[9] + p[10] + p[11] + p[12] + p[13] + p[14] + p[15] + p[16] + p[17] + p[18] + p[19] + p[20] + p[21] + p[22] + p[23] + p[24] + p[25] + p[26];
        R ir = (R)1 / rho;
        R ux = ((p[1] + p[7] + p[9] + p[13] + p[15] + p[19] + p[21] + p[23] + p[26]) - (p[2] + p[8] + p[10] + p[14] + p[16] + p[20] + p[22] + p[24] + p[25])) * ir;
        R uy = ((p[3] + p[7] + p[11] + p[14] + p[17] + p[19] + p[21] + p[24] + p[25]) - (p[4] + p[8] + p[12] + p[13] + p[18] + p[20] + p[22] + p[23] + p[26])) * ir;
        R uz = ((p[5] + p[9] + p[11] + p[16] + p[18] + p[19] + p[22] + p[23] + p[25]) - (p[6] + p[10] + p[12] + p[15] + p[17] + p[20] + p[21] + p[24] + p[26])) * ir;
        R m[6];
        m[0] = (p[1] + p[2] + p[7] + p[8] + p[9] + p[10] + p[13] + p[14] + p[15] + p[16] + p[19] + p[20] + p[21] + p[22] + p[23] + p[24] + p[25] + p[26]);
        m[1] = (p[3] + p[4] + p[7] + p[8] + p[11] + p[12] + p[13] + p[14] + p[17] + p[18] + p[19] + p[20] + p[21] + p[22] + p[23] + p[24] + p[25] + p[26]);
        m[2] = (p[5] + p[6] + p[9] + p[10] + p[11] + p[12] + p[15] + p[16] + p[17] + p[18] + p[19] + p[20] + p[21] + p[22] + p[23] + p[24] + p[25] + p[26]);
        m[3] = ((p[7] + p[8] + p[19] + p[20] + p[21] + p[22]) - (p[13] + p[14] + p[23] + p[24] + p[25] + p[26]));
        m[4] = ((p[11] + p[12] + p[19] + p[20] + p[25] + p[26]) - (p[17] + p[18] + p[21] + p[22] + p[23] + p[24]));
        m[5] = ((p[9] + p[10] + p[19] + p[20] + p[23] + p[24]) - (p[15] + p[16] + p[21] + p[22] + p[25] + p[26]));
        FN(collide3)(rho, ux, uy, uz, 0, 0, 0, g->omega, m);
        o[0] = rho; o[1] = ux; o[2] = uy; o[3] = uz;
        o[4] = m[0] * ir - FN(cs2); o[5] = m[1] * ir - FN(cs2); o[6] = m[2] * ir - FN(cs2);
        o[7] = m[3] * ir; o[8] = m[4] * ir; o[9] = m[5] * ir;
    }
}

/* ------------------------------------------------------------- link build */

typedef struct { uint64_t cq, key; } FN(cand);

static int FN(cand_cmp)(const void *a, const void *b)
{
    const FN(cand) *x = (const FN(cand) *)a, *y = (const FN(cand) *)b;
    if (x->cq != y->cq) return x->cq < y->cq ? -1 : 1;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return 0;
}

/* mrSolver2DComputeOccupancyFlagKernel_v3 / mrSolver3DComputeOccupancyFlagKernel_v3:
 * every surface element tests every lattice link whose cell lies in its
 * bounding box grown by one cell; per (cell, direction) the smallest
 * (depth, element) key wins. */
static void FN(build_links)(FN(grid) *g, const FN(surface) *S)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz, Q = g->Q, dim = g->dim;
    const int *ex, *ey, *ez, *inv;
    FN(dirs)(g, &ex, &ey, &ez, &inv);
    for (long long i = 0; i < g->nlinks; ++i) g->linkcell[g->link_cq[i] / Q] = 0;
    g->nlinks = 0;
    long long ncand = 0, capc = 1024;
    FN(cand) *cand = (FN(cand) *)malloc(sizeof(FN(cand)) * capc);
    for (int e = 0; e < S->ne; ++e) {
        /* getBoundingBox: min starts at FLT_MAX, max at FLT_MIN (:198-209, :424-440) */
        float bmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bmax[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
        for (int j = 0; j < dim; ++j) {
            uint32_t v = S->E[dim * e + j];
            for (int k = 0; k < dim; ++k) {
                float c = S->V[(size_t)v * dim + k];
                if (c < bmin[k]) bmin[k] = c;
                if (bmax[k] < c) bmax[k] = c;
            }
        }
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) {
            lo[k] = (int)(bmin[k] / g->clf) - 1;
            hi[k] = (int)(bmax[k] / g->clf) + 1;
        }
        for (int l = 1; l < Q; ++l) {
            for (int k3 = (dim == 3 ? lo[2] : 0); k3 <= (dim == 3 ? hi[2] : 0); ++k3) {
                if (k3 < 0 || k3 >= nz) continue;
                for (int j = lo[1]; j <= hi[1]; ++j) {
                    if (j < 0 || j >= ny) continue;
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        if (i < 0 || i >= nx) continue;
                        FN(isect) in;
                        const float cl = g->clf;
                        if (dim == 2) {
                            in = FN(isect2)(S->V, S->E, e, (float)i * cl, (float)j * cl,
                                            ((float)i - (float)ex[l]) * cl, ((float)j - (float)ey[l]) * cl);
                        } else {
                            R p1[3] = {(float)i * cl, (float)j * cl, (float)k3 * cl};
                            R p2[3] = {((float)i - (float)ex[l]) * cl, ((float)j - (float)ey[l]) * cl, ((float)k3 - (float)ez[l]) * cl};
                            in = FN(isect3)(S->V, S->E, e, p1, p2);
                        }
                        if (!in.hit) continue;
                        if (ncand == capc) { capc *= 2; cand = (FN(cand) *)realloc(cand, sizeof(FN(cand)) * capc); }
                        long long cell = ((long long)k3 * ny + j) * nx + i;
                        cand[ncand].cq = (uint64_t)cell * Q + l;
                        cand[ncand].key = FN(link_key)(in.depth, e);
                        ncand++;
                    }
                }
            }
        }
    }
    qsort(cand, (size_t)ncand, sizeof(FN(cand)), FN(cand_cmp));
    if (g->caplinks < ncand) {
        g->caplinks = ncand + 16;
        g->link_cq = (uint64_t *)realloc(g->link_cq, sizeof(uint64_t) * g->caplinks);
        g->link_key = (uint64_t *)realloc(g->link_key, sizeof(uint64_t) * g->caplinks);
    }
    long long n = 0;
    for (long long i = 0; i < ncand; ++i) {
        if (n > 0 && g->link_cq[n - 1] == cand[i].cq) continue; /* sorted: first key is the min */
        g->link_cq[n] = cand[i].cq;
        g->link_key[n] = cand[i].key;
        g->linkcell[cand[i].cq / Q] = 1;
        n++;
    }
    g->nlinks = n;
    free(cand);
}

long long FN(num_links)(const FN(grid) *g) { return g->nlinks; }
void FN(get_links)(const FN(grid) *g, uint64_t *cq, uint64_t *key)
{
    memcpy(cq, g->link_cq, sizeof(uint64_t) * (size_t)g->nlinks);
    memcpy(key, g->link_key, sizeof(uint64_t) * (size_t)g->nlinks);
}

/* ---------------------------------------------------------------- outlets */

/* mrApplyOutlet2DKernel / mrApplyOutlet3DKernel, in place on the new current
 * buffer; a neighbour index outside the grid is skipped (the reference reads
 * out of bounds there). */
static void FN(outlets)(FN(grid) *g, R *m)
{
    const long long N = g->ncell, nx = g->nx, nxy = (long long)g->nx * g->ny;
    const int NM = g->NM, d3 = g->dim == 3;
    for (long long c = 0; c < N; ++c) {
        uint8_t f = g->flags[c];
        long long ip; int comp, pcomp, sign;
        if (f == FL_OUT_U) { ip = c - (d3 ? nxy : nx); comp = d3 ? 3 : 2; pcomp = d3 ? 6 : 4; sign = 1; }
        else if (f == FL_OUT_D) { ip = c + (d3 ? nxy : nx); comp = d3 ? 3 : 2; pcomp = d3 ? 6 : 4; sign = -1; }
        else if (f == FL_OUT_L) { ip = c + 1; comp = 1; pcomp = d3 ? 4 : 3; sign = -1; }
        else if (f == FL_OUT_R) { ip = c - 1; comp = 1; pcomp = d3 ? 4 : 3; sign = 1; }
        else if (d3 && f == FL_OUT_F) { ip = c + nx; comp = 2; pcomp = 5; sign = -1; }
        else if (d3 && f == FL_OUT_B) { ip = c - nx; comp = 2; pcomp = 5; sign = 1; }
        else continue;
        if (ip < 0 || ip >= N) continue;
        if (g->flags[ip] != FL_FLUID) continue;
        R up = m[(size_t)ip * NM + comp];
        if ((sign > 0 && up > 0) || (sign < 0 && up < 0)) m[(size_t)c * NM + comp] = up;
        m[(size_t)c * NM + pcomp] = up * up;
    }
}

/* ------------------------------------------------------------------ step */

static void FN(zset)(const FN(grid) *g, int z, int *zs)
{
    for (int k = 0; k < 3; ++k) {
        int zz = z - 1 + k;
        if (g->dim == 2) zz = 0;
        else if (g->periodic & 4) zz = FN(wrapi)(zz, g->nz);
        else zz = FN(haloi)(zz, g->nz);
        zs[k] = zz;
    }
}

/* solveLbmAndFsiStep2D/3D: links -> fused update -> swap -> outlets.
 * forces (DIM x nv, double) is accumulated (+=), like the proxy's force
 * array. */
int FN(step)(FN(grid) *g, const float *V, const float *U, const uint32_t *E, int nv, int ne, double *forces)
{
    FN(surface) S = {V, U, E, nv, ne, forces};
    if (ne > 0 && V && E) FN(build_links)(g, &S);
    else {
        for (long long i = 0; i < g->nlinks; ++i) g->linkcell[g->link_cq[i] / g->Q] = 0;
        g->nlinks = 0;
    }
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const R *src = g->mom[g->cur];
    R *dst = g->mom[1 - g->cur];
    long long nxy = (long long)nx * ny;
    FN(planes) pl;
    for (int s = 0; s < 4; ++s) { pl.z[s] = -1; pl.p[s] = g->rec + (size_t)s * nxy * g->Q; }
    for (int z = 0; z < nz; ++z) {
        int zs[3];
        FN(zset)(g, z, zs);
        R *P[3];
        for (int k = 0; k < 3; ++k) P[k] = FN(plane_get)(g, &pl, src, zs[k], zs);
        long long base = (long long)z * nxy;
#pragma omp parallel for schedule(static)
        for (long long c = 0; c < nxy; ++c) {
            long long cid = base + c;
            uint8_t f = g->flags[cid];
            if (f != FL_FLUID && f != FL_SOLIDDYN) continue;
            if (g->linkcell[cid]) continue;
            FN(update_cell)(g, src, dst, (int)(c % nx), (int)(c / nx), z, P, &S, 0);
        }
        /* cells with links: sequential, fixed order, so force sums are reproducible */
        for (long long c = 0; c < nxy; ++c) {
            long long cid = base + c;
            uint8_t f = g->flags[cid];
            if (f != FL_FLUID && f != FL_SOLIDDYN) continue;
            if (!g->linkcell[cid]) continue;
            FN(update_cell)(g, src, dst, (int)(c % nx), (int)(c / nx), z, P, &S, 1);
        }
    }
    g->cur = 1 - g->cur;
    FN(outlets)(g, g->mom[g->cur]);
    return 0;
}

/* ------------------------------------------------------------ fill solid */

/* resetSolidFlagKernel + updateSolidFlagKernel with the 2D even-odd isInside
 * test (FsiCoupling2D.cu:318-354; SolidGeometryProxy_Device.cuh:126-144). */
void FN(fill_solid2)(FN(grid) *g, const float *V, const uint32_t *E, int ne)
{
    if (g->dim != 2) return;
    for (long long c = 0; c < g->ncell; ++c)
        if (g->flags[c] == FL_FLUID || g->flags[c] == FL_SOLIDDYN) g->flags[c] = FL_FLUID;
    for (int y = 0; y < g->ny; ++y)
        for (int x = 0; x < g->nx; ++x) {
            long long c = (long long)y * g->nx + x;
            if (g->flags[c] != FL_FLUID) continue;
            float px = ((float)x + 0.5f) * g->clf, py = ((float)y + 0.5f) * g->clf;
            int in = 0;
            for (int i = 0; i < ne; ++i) {
                uint32_t a = E[2 * i], b = E[2 * i + 1];
                float sx = V[2 * a], sy = V[2 * a + 1], tx = V[2 * b], ty = V[2 * b + 1];
                if ((sy < py && ty >= py) || (sy >= py && ty < py))
                    in ^= (sx + (py - sy) * (tx - sx) / (ty - sy) > px);
            }
            if (in) g->flags[c] = FL_SOLIDDYN;
        }
}

/* ----------------------------------------------- single-cell math (tests) */

void FN(reconstruct)(int dim, const double *m, double *f, int half_pops)
{
    FN(init_tables)();
    R mm[10], ff[27];
    int NM = dim == 2 ? 6 : 10, Q = dim == 2 ? 9 : 27;
    for (int k = 0; k < NM; ++k) mm[k] = (R)m[k];
    FN(grid) g; memset(&g, 0, sizeof(g)); g.dim = dim; g.half_pops = half_pops;
    FN(rec_cell)(&g, mm, ff);
    for (int k = 0; k < Q; ++k) f[k] = (double)ff[k];
}

double FN(reconstruct_at)(int dim, const double *m, int i)
{
    FN(init_tables)();
    if (dim == 2) return (double)FN(rec2_at)((R)m[0], (R)m[1], (R)m[2], (R)m[3], (R)m[5], (R)m[4], i);
    FN(coef3) c;
    FN(coef3_make)((R)m[0], (R)m[1], (R)m[2], (R)m[3], (R)m[4], (R)m[5], (R)m[6], (R)m[7], (R)m[8], (R)m[9], &c);
    return (double)FN(rec3_at)(&c, i);
}

/* moments of a population set followed by collision and re-encode, i.e. the
 * tail of the fused kernel for one cell with the pulled populations given. */
void FN(collide_pops)(int dim, const double *pops, double omega, double *out)
{
    FN(init_tables)();
    FN(grid) g; memset(&g, 0, sizeof(g));
    g.dim = dim; g.nx = g.ny = g.nz = 1; g.Q = dim == 2 ? 9 : 27; g.NM = dim == 2 ? 6 : 10;
    g.omega = (R)omega;
    /* reuse update_cell's tail through a one-cell grid whose pulls come from a
     * plane holding exactly the given populations (uniform, no walls) */
    R plane[27], src[10] = {0}, dst[10];
    for (int k = 0; k < g.Q; ++k) plane[k] = (R)pops[k];
    uint8_t fl = FL_FLUID; g.flags = &fl;
    R *P[3] = {plane, plane, plane};
    FN(surface) S; memset(&S, 0, sizeof(S));
    FN(update_cell)(&g, src, dst, 0, 0, 0, P, &S, 0);
    for (int k = 0; k < g.NM; ++k) out[k] = (double)dst[k];
}
