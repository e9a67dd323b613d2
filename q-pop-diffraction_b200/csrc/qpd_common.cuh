// Common types for the B200 diffraction kernels: precision traits and complex arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qpd {

// Complex storage type for each real precision.  The float path keeps fields as
// complex64 (8 B per value), the double path as complex128 (16 B).
template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };
template <typename T> using C_t = typename Cplx<T>::type;

template <typename C> __host__ __device__ __forceinline__ C cmake(decltype(C::x) re, decltype(C::x) im) {
    C c;
    c.x = re;
    c.y = im;
    return c;
}
// The intensity floor max(v, 1e-50) as numpy.maximum computes it (src/python/diffraction.py:111): a NaN
// propagates, where fmax would return the floor.
__device__ __forceinline__ double floor_1e50(double v) { return v < 1e-50 ? 1e-50 : v; }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmake<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmake<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a += b * c
template <typename C> __device__ __forceinline__ void cfma(C& a, C b, C c) {
    a.x = fma(b.x, c.x, fma(-b.y, c.y, a.x));
    a.y = fma(b.x, c.y, fma(b.y, c.x, a.y));
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return cmake<C>(a.x * s, a.y * s); }
// -i * a
template <typename C> __device__ __forceinline__ C cmul_mi(C a) { return cmake<C>(a.y, -a.x); }
// +i * a
template <typename C> __device__ __forceinline__ C cmul_pi(C a) { return cmake<C>(-a.y, a.x); }
// a - i b and a + i b (the swap stays in the scalar operands)
template <typename C> __device__ __forceinline__ C cadd_mi(C a, C b) { return cmake<C>(a.x + b.y, a.y - b.x); }
template <typename C> __device__ __forceinline__ C cadd_pi(C a, C b) { return cmake<C>(a.x - b.y, a.y + b.x); }
// a += s * b, s real
template <typename C> __device__ __forceinline__ void caxpy(C& a, decltype(C::x) s, C b) {
    a.x = fma(s, b.x, a.x);
    a.y = fma(s, b.y, a.y);
}

#ifndef QPD_F32X2
#define QPD_F32X2 1
#endif
#if QPD_F32X2 && defined(__CUDA_ARCH__)
// complex64 on the packed two-lane float32 instructions of sm_100 (add/sub/mul/fma .f32x2): one
// instruction per complex add or real-scaled multiply-add instead of two.  Same IEEE round-to-
// nearest results per lane as the scalar forms.
__device__ __forceinline__ unsigned long long f2_pk(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 f2_up(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pk(a)), "l"(f2_pk(b)));
    return f2_up(d);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pk(a)), "l"(f2_pk(b)));
    return f2_up(d);
}
template <> __device__ __forceinline__ float2 cscale<float2>(float2 a, float s) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pk(a)), "l"(f2_pk(make_float2(s, s))));
    return f2_up(d);
}
template <> __device__ __forceinline__ void caxpy<float2>(float2& a, float s, float2 b) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_pk(make_float2(s, s))), "l"(f2_pk(b)), "l"(f2_pk(a)));
    a = f2_up(d);
}
// a += b * c: the b.x products as one packed fma, the b.y cross terms scalar
template <> __device__ __forceinline__ void cfma<float2>(float2& a, float2 b, float2 c) {
    caxpy(a, b.x, c);
    a.x = fmaf(-b.y, c.y, a.x);
    a.y = fmaf(b.y, c.x, a.y);
}
template <> __device__ __forceinline__ float2 cmul<float2>(float2 a, float2 b) {
    float2 t = cscale(b, a.x);
    t.x = fmaf(-a.y, b.y, t.x);
    t.y = fmaf(a.y, b.x, t.y);
    return t;
}
#endif


}  // namespace qpd
