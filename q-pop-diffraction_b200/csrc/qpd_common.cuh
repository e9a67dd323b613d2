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


}  // namespace qpd
