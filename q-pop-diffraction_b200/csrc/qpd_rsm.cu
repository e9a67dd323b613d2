// Reciprocal-space-map projections of a device-resident intensity volume.
//
// The reference bins every voxel with numpy.histogram2d over pairs of broadcast q components
// (src/python/rsm.py:88-104).  Its q grid is the tensor product of three 1-D axes, so each of the
// three maps is a projection of I along the third axis followed by a re-binning of the 1-D axes;
// the projections are the only part that touches the n voxels, and they run here:
//
//   xy[x, y] = sum_z I[x, y, z],  xz[x, z] = sum_y I[x, y, z],  yz[y, z] = sum_x I[x, y, z]
//
// with I (nx, ny, nz) float64, z fastest (the layout the hot path writes).  Two passes over I,
// both coalesced, both deterministic (fixed summation order, no atomics):
//   rsm_x_kernel: one block per x slab (ny, nz): xz by columns of 32 z, xy by warp sums over z;
//   rsm_yz_kernel: one thread per (y, z), summing over x with the loads of consecutive threads
//   adjacent in memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "qpopdiff.h"

void qpd_internal_set_error(const char* msg);

namespace {

constexpr int kRT = 32;    // z columns per chunk (lanes)
constexpr int kRRows = 8;  // warps per block
constexpr long long kMaxRsmNy = 16384;  // shared xy row sums: 8 * ny bytes

__global__ void __launch_bounds__(kRT * kRRows) rsm_x_kernel(const double* __restrict__ I, long long ny, long long nz,
                                                          double* __restrict__ xy, double* __restrict__ xz) {
    extern __shared__ double rows[];            // ny partial row sums of this slab
    __shared__ double part[kRRows][kRT + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long x = blockIdx.x;
    const double* slab = I + x * ny * nz;
    for (long long y = ty * kRT + tx; y < ny; y += kRT * kRRows) rows[y] = 0.0;
    __syncthreads();
    for (long long zc = 0; zc < nz; zc += kRT) {
        const long long z = zc + tx;
        double col = 0.0;
        for (long long y = ty; y < ny; y += kRRows) {   // warp ty owns rows y = ty (mod 8): no races on rows[y]
            const double v = z < nz ? slab[y * nz + z] : 0.0;
            col += v;
            double s = v;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (tx == 0) rows[y] += s;
        }
        part[ty][tx] = col;
        __syncthreads();
        if (ty == 0 && z < nz) {
            double t = 0.0;
            for (int r = 0; r < kRRows; r++) t += part[r][tx];
            if (xz) xz[x * nz + z] = t;
        }
        __syncthreads();
    }
    if (xy)
        for (long long y = ty * kRT + tx; y < ny; y += kRT * kRRows) xy[x * ny + y] = rows[y];
}

__global__ void rsm_yz_kernel(const double* __restrict__ I, long long nx, long long plane, double* __restrict__ yz) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= plane) return;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};         // four independent chains keep loads in flight
    long long x = 0;
    for (; x + 4 <= nx; x += 4)
        for (int k = 0; k < 4; k++) acc[k] += I[(x + k) * plane + j];
    for (; x < nx; x++) acc[0] += I[x * plane + j];
    yz[j] = (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

int fail(const std::string& msg, int code) {
    qpd_internal_set_error(msg.c_str());
    return code;
}

}  // namespace

extern "C" {

int qpd_rsm_project(const double* I, int64_t nx, int64_t ny, int64_t nz, double* xy, double* xz, double* yz,
                    void* stream) {
    if (!I || nx < 1 || ny < 1 || nz < 1) return fail("qpd_rsm_project: NULL intensity or empty grid", QPD_ERR_ARG);
    if (ny > kMaxRsmNy || nx > 0x7fffffff) return fail("qpd_rsm_project: ny > 16384 or nx > 2^31 - 1", QPD_ERR_UNSUPPORTED);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (xy || xz) {
        const size_t smem = sizeof(double) * (size_t)ny;
        cudaError_t e = cudaFuncSetAttribute(rsm_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return fail(std::string("qpd_rsm_project: ") + cudaGetErrorString(e), QPD_ERR_CUDA);
        rsm_x_kernel<<<(unsigned)nx, dim3(kRT, kRRows), smem, st>>>(I, ny, nz, xy, xz);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(std::string("qpd_rsm_project: ") + cudaGetErrorString(e), QPD_ERR_CUDA);
    }
    if (yz) {
        const long long plane = ny * nz;
        rsm_yz_kernel<<<(unsigned)((plane + 255) / 256), 256, 0, st>>>(I, nx, plane, yz);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(std::string("qpd_rsm_project: ") + cudaGetErrorString(e), QPD_ERR_CUDA);
    }
    return QPD_OK;
}

}  // extern "C"
