// Boundary-input preparation on the GPU: Q-POP-FerroDyn fields in their file order become the
// packed kernel inputs in one pass.
//
// The reference does this on the host in float64 (src/python/cli.py:174-217, loaders in
// src/python/io_utils.py:30-92) and, in its native program, partly in the `columns` kernel
// (src/heffte/kernels.cuh:34-50): transpose (nz, ny, nx) -> (x, y, z), scale P and u, one-hot
// phases of the FE materials, region = (cell is FE) x region file, and the u_z reference ramp
// (cumsum_z dc[mat] - dc[mat] / 2) dz summed over the FULL material stack, then cropped.
//
// Layout: a block owns 32 columns x at one row y.  It walks the full stack in chunks of 32
// layers.  Each chunk is read with x fastest (coalesced in the file order), the ramp is scanned
// serially per column in float64 in the same order as numpy.cumsum, and the cropped layers are
// written transposed with z fastest (coalesced in the kernel order) through padded shared tiles.
#pragma once

#include "qpd_kernels.cuh"

namespace qpd {

constexpr int kMaxMaterials = 64;
constexpr unsigned kFlagBadMaterial = 4u;  // a material index outside the dc / phase_of tables

template <typename T> struct FieldsArgs {
    const float* P[3];        // nStruc planes, (nz, ny, nx)
    const float* u[3];        // null -> 0
    const float* phase;       // nPhase planes of phase fractions, or null: one-hot from the material
    const float* region;      // null -> 1
    const signed char* mat;   // (nz_full, ny, nx)
    long long nx, ny, nz, z0; // crop size and its first layer in the material stack
    int nStruc, nPhase, nMat;
    double dz, p_scale, u_scale;
    double dc[kMaxMaterials];
    signed char phase_of[kMaxMaterials];
    T* Pout;                  // 3 planes of n, (x, y, z)
    T* Uout;
    signed char* phase_idx;   // single mode
    T* weight;
    T* wdense;                // dense mode: nPhase planes
    unsigned int* flags;
};

constexpr int kFT = 32;        // tile edge (x and z)
constexpr int kFRows = 8;      // threadIdx.y extent
constexpr int kFPitch = kFT + 1;

// Dynamic shared memory: ramp (double) + phase index (char) + one float tile per input plane.
inline size_t fields_smem_bytes(int planes) {
    return sizeof(double) * kFT * kFPitch + sizeof(float) * (size_t)planes * kFT * kFPitch + kFT * kFPitch;
}

template <typename T> __global__ void __launch_bounds__(kFT * kFRows) fields_kernel(FieldsArgs<T> a) {
    extern __shared__ __align__(128) unsigned char fsm[];
    double* ramp = reinterpret_cast<double*>(fsm);                        // [z][x]
    float* tiles = reinterpret_cast<float*>(ramp + kFT * kFPitch);        // [plane][z][x]
    const int nU = a.u[0] ? 3 : 0, nW = a.phase ? a.nPhase : 0, nR = a.region ? 1 : 0;
    const int planes = a.nStruc + nU + nW + nR;
    signed char* pidx = reinterpret_cast<signed char*>(tiles + (size_t)planes * kFT * kFPitch);

    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long x0 = (long long)blockIdx.x * kFT, y = blockIdx.y;
    const long long n = a.nx * a.ny * a.nz;
    const long long plane_in = a.nz * a.ny * a.nx;
    double run = 0.0;          // running column sum (lanes of warp 0)
    unsigned int f = 0;

    for (long long zc = 0; zc < a.z0 + a.nz; zc += kFT) {
        // 1. materials of the chunk: dc and phase index, x fastest
        for (int zz = ty; zz < kFT; zz += kFRows) {
            const long long z = zc + zz, x = x0 + tx;
            double d = 0.0;
            signed char p = -1;
            if (z < a.z0 + a.nz && x < a.nx) {
                const int m = a.mat[(z * a.ny + y) * a.nx + x];
                if (m >= 0 && m < a.nMat) {
                    d = a.dc[m];
                    p = a.phase_of[m];
                } else {
                    f |= kFlagBadMaterial;
                }
            }
            ramp[zz * kFPitch + tx] = d;
            pidx[zz * kFPitch + tx] = p;
        }
        // 2. cropped input planes of the chunk, x fastest
        const bool crop = zc + kFT > a.z0;
        if (crop) {
            for (int zz = ty; zz < kFT; zz += kFRows) {
                const long long zl = zc + zz - a.z0, x = x0 + tx;
                const bool in = zl >= 0 && zl < a.nz && x < a.nx;
                const long long off = (zl * a.ny + y) * a.nx + x;
                int q = 0;
                for (int k = 0; k < a.nStruc; k++, q++) tiles[(q * kFT + zz) * kFPitch + tx] = in ? a.P[k][off] : 0.f;
                for (int k = 0; k < nU; k++, q++) tiles[(q * kFT + zz) * kFPitch + tx] = in ? a.u[k][off] : 0.f;
                for (int k = 0; k < nW; k++, q++)
                    tiles[(q * kFT + zz) * kFPitch + tx] = in ? a.phase[k * plane_in + off] : 0.f;
                if (nR) tiles[(q * kFT + zz) * kFPitch + tx] = in ? a.region[off] : 0.f;
            }
        }
        __syncthreads();
        // 3. ramp: one lane per column, layers in order (numpy.cumsum's summation order)
        if (ty == 0) {
            for (int zz = 0; zz < kFT && zc + zz < a.z0 + a.nz; zz++) {
                const double d = ramp[zz * kFPitch + tx];
                run = __dadd_rn(run, d);
                ramp[zz * kFPitch + tx] = __dmul_rn(__dadd_rn(run, -0.5 * d), a.dz);
            }
        }
        __syncthreads();
        // 4. cropped layers, z fastest: lane = layer, rows = columns
        if (crop) {
            const int zz = tx;
            const long long zl = zc + zz - a.z0;
            for (int xx = ty; xx < kFT; xx += kFRows) {
                const long long x = x0 + xx;
                if (zl < 0 || zl >= a.nz || x >= a.nx) continue;
                const long long g = (x * a.ny + y) * a.nz + zl;
                const int t = zz * kFPitch + xx;
                int q = 0;
                for (int k = 0; k < 3; k++)
                    a.Pout[k * n + g] = k < a.nStruc ? T(__dmul_rn(a.p_scale, (double)tiles[(q + k) * kFT * kFPitch + t])) : T(0);
                q += a.nStruc;
                for (int k = 0; k < 3; k++) {  // rounded products and sums, no contraction: as numpy
                    double v = nU ? __dmul_rn((double)tiles[(q + k) * kFT * kFPitch + t], a.u_scale) : 0.0;
                    if (k == 2) v = __dadd_rn(v, ramp[t]);
                    a.Uout[k * n + g] = T(v);
                }
                q += nU;
                const int p = pidx[t];
                const double r = p >= 0 ? (nR ? (double)tiles[(q + nW) * kFT * kFPitch + t] : 1.0) : 0.0;
                if (a.wdense) {
                    for (int k = 0; k < a.nPhase; k++) {
                        const double o = nW ? (double)tiles[(q + k) * kFT * kFPitch + t] : (k == p ? 1.0 : 0.0);
                        a.wdense[k * n + g] = T(o * r);
                    }
                } else {
                    int which = -1;
                    double w = 0.0;
                    for (int k = 0; k < a.nPhase; k++) {
                        const double o = nW ? (double)tiles[(q + k) * kFT * kFPitch + t] : (k == p ? 1.0 : 0.0);
                        const double wp = o * r;
                        if (wp != 0.0) {
                            if (which >= 0) f |= 1u;
                            else {
                                which = k;
                                w = wp;
                            }
                        }
                    }
                    if (which >= 0 && w != 1.0) f |= 2u;
                    a.phase_idx[g] = (signed char)which;
                    a.weight[g] = T(w);
                }
            }
        }
        __syncthreads();
    }
    if (f) atomicOr(a.flags, f);
}

}  // namespace qpd
