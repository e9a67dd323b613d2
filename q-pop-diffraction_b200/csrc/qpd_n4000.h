// Register-resident 4000-point axis passes (qpd_n4000.cu), used for every 4000-point axis of the
// float32 fused schedule: the y pass over contiguous pencils of the (x, k_z, y) layout, and strided
// y and x passes over pairs of neighbouring inner values.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "qpd_kernels.cuh"

namespace qpd {

constexpr int kPass4kMax = 48;

// One fused pass over 4000-point pencils: its inputs, in segment order, and how they fold.
//   field[fl]   field of input fl (an index into the field array of AxisArgs::in);
//   u, V, ik    the fold coefficient of input fl, factored: for the frequency index m = t + 200 r
//               (t < 200, r < 20), exp(-i (k_m + G) R) = u[t] V[r] exactly, with
//               u[t] = exp(-2 pi i t R / (N h)) and V[r] = exp(-i (2 pi (200 r - N [r >= 10]) R / (N h) + G R)),
//               each rounded from float64; with bit fl of ik set the coefficient also carries -i k_m,
//               k_m = kscale (m - N [r >= 10]), kscale = 2 pi / (N h);
//   last        bit fl: input fl closes a segment, whose folded sum is stored as field out[fl]
//               (AxisArgs::out), or, in the x pass, becomes the intensity.
struct Pass4k {
    const float2* u[kPass4kMax];  // 200 values per input
    const float2* V[kPass4kMax];  // 20 values per input
    int field[kPass4kMax];
    int out[kPass4kMax];
    unsigned long long ik;
    unsigned long long last;
    float kscale;
    int n;  // inputs
};

// y pass over y-fastest fields: one contiguous 4000-point pencil of every field at a time (npencils =
// nx * nz, in any order of x and k_z), the folded outputs written back in place.
cudaError_t launch_ypass4000(const AxisArgs<float>& a, const Pass4k& p, long long npencils, cudaStream_t st);

// Strided passes over pencils of 4000 values, in pairs of neighbouring inner values (a.nz even, nouter
// outer values), loaded as tensor tiles through `map`, a float32 view (2 inner, middle, nfields * rows)
// of the field array with boxes of (4, 200, 1) rows along the middle dimension or (4, 1, 200) along the
// outer one:
//   YPassZFast  the y pass over (x, y, z) fields (map (2 nz, ny, nfields nx), box (4, 200, 1), nouter = nx),
//               outputs written in place;
//   XPassZFast  the x pass with the |S Amp|^2 + fftshift epilogue over (x, y, z) fields (map (2 nz, ny,
//               nfields nx), box (4, 1, 200), a.nz = nz, nouter = ny);
//   XPassYFast  the same over (k_z, x, y) fields (map (2 ny, nx, nfields nz), box (4, 200, 1), a.nz = ny,
//               nouter = nz).
enum class Strided4k { YPassZFast, XPassZFast, XPassYFast };
cudaError_t launch_strided4000(const CUtensorMap& map, const AxisArgs<float>& a, const Pass4k& p, int nouter,
                               Strided4k kind, cudaStream_t st);

// I[shift(k_x)][shift(k_y)][shift(k_z)] = T[k_z][k_y][k_x] for the intensity the y-fastest x pass staged in
// AxisArgs::Istage (T and I distinct, nz <= 256).
cudaError_t launch_unstage_intensity(const double* T, double* I, long long nx, long long ny, long long nz,
                                     cudaStream_t st);

}  // namespace qpd
