// Unit roots exp(-2 pi i m / R) of the odd radices that have a register butterfly, in constant
// memory.  Butterflies index them with offsets that are compile-time constants after unrolling,
// so every use is a constant-bank operand rather than a register.  The host fills both tables
// once per device (qpd_roots_init), from double-precision cos / sin.
#pragma once

#include "qpd_common.cuh"

namespace qpd {

// Odd radices with a register butterfly and their offsets in the tables.
constexpr int kOddRadices[] = {3, 5, 7, 11, 13, 17};
__host__ __device__ constexpr int root_offset(int R) {
    return R == 3 ? 0 : R == 5 ? 3 : R == 7 ? 8 : R == 11 ? 15 : R == 13 ? 26 : R == 17 ? 39 : -1;
}
constexpr int kRootsTotal = 3 + 5 + 7 + 11 + 13 + 17;

// internal linkage: each translation unit that launches butterflies fills its own copy
static __constant__ float2 c_roots_f[kRootsTotal];
static __constant__ double2 c_roots_d[kRootsTotal];

template <typename T> __device__ __forceinline__ C_t<T> unit_root(int idx);
template <> __device__ __forceinline__ float2 unit_root<float>(int idx) { return c_roots_f[idx]; }
template <> __device__ __forceinline__ double2 unit_root<double>(int idx) { return c_roots_d[idx]; }

}  // namespace qpd
