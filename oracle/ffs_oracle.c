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
