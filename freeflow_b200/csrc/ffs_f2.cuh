// Packed FP32 pairs for sm_100: add/sub/mul/fma.rn.f32x2 issue two IEEE FP32
// operations per instruction.  Each lane of a pair rounds exactly like the
// scalar instruction, so results are bit-identical to scalar code with the
// same operation order.
#pragma once
#include <cuda_runtime.h>

namespace fflbm {

struct f2 {
    unsigned long long v;
};

__device__ __forceinline__ f2 f2make(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f2 f2splat(float a) { return f2make(a, a); }
__device__ __forceinline__ void f2split(f2 x, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x.v));
}
__device__ __forceinline__ f2 operator+(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f2 operator-(f2 a, f2 b)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f2 operator*(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
// a * b + c
__device__ __forceinline__ f2 vfma(f2 a, f2 b, f2 c)
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }

template <typename V> __device__ __forceinline__ V vconst(float a);
template <> __device__ __forceinline__ float vconst<float>(float a) { return a; }
template <> __device__ __forceinline__ f2 vconst<f2>(float a) { return f2splat(a); }

} // namespace fflbm
